"""Host-side parts of the product on CPU: the C ABI loads and exports every
declared symbol, the Field contract, p-values, generators and CLI argument
handling (no GPU call is made here)."""
import ctypes
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import M61, PKG, ROOT

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
CLI = os.path.join(PKG, "bin", "modlin")


def declared_functions():
    src = open(os.path.join(ROOT, "include", "modlin.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(modlin_[a-z0-9_]+)\s*\(", src)) - {"modlin_progress_fn"})


def test_library_exports_every_declared_symbol(built_lib):
    names = declared_functions()
    assert len(names) >= 25
    L = ctypes.CDLL(built_lib)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(modlin_[a-z0-9_]+)\b", out))
    assert set(names) <= exported


def test_binding_lists_all_exports(M):
    from modlin import _lib
    assert set(declared_functions()) <= set(_lib.EXPORTED) | {"modlin_rank_batch"}


def test_field_contract(M, O):
    """src/fp.rs:49-113 through the C ABI vs the oracle."""
    rng = np.random.default_rng(5)
    for p in [2, 3, 97, 65537, (1 << 31) - 1, M61, (1 << 62) + 135, (1 << 63) - 25]:
        f, g = M.Field(p), O.Field(p)
        assert f.safe_batch == g.safe_batch
        assert f.mu == (2**128 - 1) // p
        for t in [0, 1, p - 1, p, 2**128 - 1, 1 << 127] + [int(x) << 64 | int(y) for x, y in
                                                          rng.integers(0, 2**63, (64, 2))]:
            assert f.reduce_u128(t) == t % p
        for x in [0, p - 1, 2**64 - 1]:
            assert f.reduce(x) == x % p
        for a, b in rng.integers(0, p, (64, 2), dtype=np.uint64):
            assert f.mul(int(a), int(b)) == int(a) * int(b) % p


def test_field_rejects_bad_modulus(M):
    for p in [0, 1, 1 << 63, 2**64 - 1]:
        with pytest.raises(M.ModlinError):
            M.Field(p)


def test_pvalues_bit_exact_vs_golden(M):
    for p, n, c, hc, hl in GOLD["oracle"]["pvalues"]:
        assert M.corank_tail_pvalue(p, n, c) == float.fromhex(hc), (p, n, c)
        assert M.lc_left_tail_pvalue(p, n, c) == float.fromhex(hl), (p, n, c)


def test_pvalues_vs_live_oracle(M, O):
    for p in [2, 11, 65521, M61]:
        for n in [3, 50, 500]:
            for d in range(0, n + 1, max(1, n // 25)):
                assert M.corank_prob(p, n, d) == O.corank_prob(p, n, d)
                assert M.corank_tail_pvalue(p, n, d) == O.corank_tail_pvalue(p, n, d)
                assert M.lc_left_tail_pvalue(p, n, d) == O.lc_left_tail_pvalue(p, n, d)


def test_stats_reference_values(M):
    """tests/test_stats.rs:25-37 on the product's p-values."""
    assert M.corank_tail_pvalue(M61, 305, 0) == 1.0
    assert M.corank_tail_pvalue(M61, 305, 33) == 1e-307
    assert M.lc_left_tail_pvalue(M61, 10_000, 5000) == 1.0
    assert M.lc_left_tail_pvalue(M61, 10_000, 272) == 1e-307
    assert M.lc_left_tail_pvalue(2, 1000, 503) == 0.9947916666666666


def test_pretty_p_value(M):
    for hx, s in GOLD["oracle"]["pretty"]:
        assert M.pretty_p_value(float.fromhex(hx)) == s, s
    assert M.pretty_p_value(0.0) == "0"
    assert M.pretty_p_value(1.0) == "1"
    rng = np.random.default_rng(3)
    import oracle
    for x in list(10.0 ** rng.uniform(-320, 20, 300)) + list(rng.uniform(0, 1, 300)):
        assert M.pretty_p_value(float(x)) == oracle.pretty_p_value(float(x)), x


@pytest.mark.parametrize("kind,key", [("mixmax17", "mixmax17"), ("mixmax", "mixmax240"), ("mixmax256", "mixmax256")])
def test_product_mixmax_golden(M, kind, key):
    g = M.prng.Prng(kind, GOLD["reference"]["mixmax_seed"])
    assert [int(x) >> 3 for x in g.fill(10)] == GOLD["reference"][key]


def test_product_prng_streams_match_oracle(M, O):
    for kind in ["xoroshiro128pp", "mixmax17", "mixmax", "mixmax256"]:
        for seed in [1, 2, 0xDEADBEEF]:
            g = M.prng.Prng(kind, seed)
            a = np.concatenate([g.fill(1000), g.fill(777)])
            assert np.array_equal(a, O.prng(kind, seed, 1777)), (kind, seed)
    assert [int(x) for x in M.prng.Prng("xoroshiro128pp", 0).fill(10)] == GOLD["reference"]["xoroshiro_seed0"]


def test_prng_names_and_zero_seed(M):
    assert M.prng.Prng("mixmax17", 1).name == "MIXMAX (TRandomMixMax17, N=17)"
    assert M.prng.Prng("mixmax256", 1).name == "MIXMAX (TRandomMixMax256, N=256, skip=2)"
    assert M.prng.Prng("mixmax", 1).name == "MIXMAX (TRandomMixMax, N=240, s=487013230256099140)"
    assert M.prng.Prng("xoroshiro128pp", 0).name == "xoroshiro128++"
    with pytest.raises(M.ModlinError):
        M.prng.Prng("mixmax17", 0)


def test_generators_match_oracle(M, O):
    for p in [2, 3, 127, 65521, (1 << 31) - 1, M61, (1 << 63) - 25]:
        assert np.array_equal(M.gen.uniform(p, 11, 5000), O.gen_uniform(p, 11, 5000))
    for p, L in [(127, 5), (65521, 40), (M61, 64), (2, 9)]:
        assert np.array_equal(M.gen.planted(p, L, 8, 3000), O.gen_planted(p, L, 8, 3000))
    for p, head in GOLD["oracle"]["uniform_heads"].items():
        assert [int(x) for x in M.gen.uniform(int(p), 7, 16)] == head


def run_cli(*args):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    return subprocess.run([CLI, *args], capture_output=True, text=True, env=env, timeout=60)


@pytest.mark.parametrize("args,msg", [
    (["-R", "1", "-p", "7"], "SIDE/LENGTH must be at least 2"),
    (["-L", "1", "-p", "7"], "SIDE/LENGTH must be at least 2"),
    (["-R", "5000000000", "-p", "7"], "SIDE is too large"),
    (["-R", "4", "-p", "7", "0"], "reps must be at least 1"),
    (["-R", "4", "-p", "1"], "modulus must be at least 2"),
    (["-R", "4", "-p", "9223372036854775808"], "modulus must be below"),
    (["-R", "4", "-p", "91"], "modulus must be prime"),
    (["-R", "4", "-L", "4", "-p", "7"], ""),
    (["-p", "7"], ""),
    (["-R", "4"], ""),
    (["-R", "4", "-p", "7", "-S", "0xZZ"], ""),
])
def test_cli_validation_exit_2(built_lib, args, msg):
    """src/cli.rs:161-189: argument errors exit with status 2."""
    r = run_cli(*args)
    assert r.returncode == 2, (args, r.stderr)
    assert msg in r.stderr
    assert r.stdout == ""


def test_cli_zero_seed_mixmax_exit_1(built_lib):
    """src/main.rs:29-35: header printed, then the generator error, exit 1."""
    r = run_cli("-R", "4", "-p", "7", "--prng", "mixmax17", "-S", "0")
    assert r.returncode == 1
    assert r.stdout == "Generator: MIXMAX (TRandomMixMax17, N=17)\nSeed: 0x0000000000000000\n"
    assert "Error initializing the generator" in r.stderr


def test_cli_seed_parsing(built_lib):
    """src/cli.rs:53-66 and src/main.rs:26: 0x/0o/0b prefixes, underscores,
    `{:#018x}` echo. Without a GPU the run stops after the header lines."""
    for s, v in [("0xDEAD_BEEF", 0xDEADBEEF), ("0o17", 15), ("0B101", 5), ("1_000", 1000), (" 42 ", 42)]:
        r = run_cli("-R", "2", "-p", "7", "--prng", "xoroshiro128pp", "-S", s)
        lines = r.stdout.splitlines()
        assert lines[:2] == ["Generator: xoroshiro128++", "Seed: 0x%016x" % v], r.stdout
        assert lines[2] == ("Running a modular rank test using 0.000 MiB of RAM: 1 2\u00d72 matrix "
                            "over the field of size 7")


def test_prng_state_roundtrip(M):
    """modlin_prng_get_state / set_state: a saved position replays the stream."""
    for kind, words in [("xoroshiro128pp", 2), ("mixmax17", 19), ("mixmax", 242), ("mixmax256", 258)]:
        g = M.prng.Prng(kind, 9)
        g.fill(1234)
        s = g.get_state()
        assert s.size == words
        a = g.fill(777)
        g.set_state(s)
        assert np.array_equal(g.fill(777), a)
    g = M.prng.Prng("mixmax17", 9)
    s = g.get_state()
    for i, bad in [(3, 1 << 61), (17, 1 << 62), (18, 0), (18, 18)]:
        t = s.copy()
        t[i] = bad
        with pytest.raises(M.ModlinError):
            g.set_state(t)
    with pytest.raises(M.ModlinError):
        g.set_state(s[:-1])


@pytest.mark.parametrize("kind", ["mixmax17", "mixmax", "mixmax256"])
def test_mixmax_is_linear_over_fp(M, kind):
    """The device fill's jump-ahead rests on this: block b of the stream is
    (skip + 1) linear iterations of block b - 1 over F_p (outputs >> 3 are
    the raw state entries v[1..N-1])."""
    from mixmax_model import MIX, mix_step
    N, _, skip, _ = MIX[kind]
    g = M.prng.Prng(kind, 5)
    st = g.get_state()
    y = [int(st[N])] + [int(v) for v in st[1:N]]
    out = g.fill(6 * (N - 1))
    for b in range(6):
        for _ in range(skip + 1):
            y = mix_step(kind, y)
        got = [(int(v) >> 3) % M61 for v in out[b * (N - 1):(b + 1) * (N - 1)]]
        assert got == y[1:], (kind, b)


@pytest.mark.parametrize("kind", ["mixmax17", "mixmax256"])
def test_mixmax_folds_keep_p_for_zero(M, kind):
    """ROOT's single fold leaves 2^61 - 1 (not 0) where a sum of nonzero
    residues is = 0, and that reaches the output as (2^61 - 1) << 3: states
    planted to hit such sums produce it, so a fill that computes canonical
    residues alone would differ there."""
    from mixmax_model import MIX, plant, set_mix_state
    N, _, skip, _ = MIX[kind]
    per = skip + 1
    x = plant(kind, np.random.default_rng(1), [(per, 5), (2 * per, N - 1)])
    g = M.prng.Prng(kind, 1)
    set_mix_state(g, kind, x, N)
    out = g.fill(2 * (N - 1))
    p3 = np.uint64((M61 << 3) & ((1 << 64) - 1))
    assert out[4] == p3 and out[N - 1 + N - 2] == p3


def test_timeout_hook_rejects_bad_arguments(M):
    """The failure-detection hook validates its arguments on the host."""
    L = M.lib()
    assert L.modlin_testing_grid_timeout_once(0, 0) == -8
    assert L.modlin_testing_grid_timeout_once(1000, -1) == -8
    assert L.modlin_testing_grid_timeout_once(5_000_000_000, 0) == -8
