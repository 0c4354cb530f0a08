"""The `modlin` CLI on the GPU: stdout byte-identical to the reference's
(README.md:61-158, src/main.rs:23-26, :74-78, :121-125, :142-148, :170-174)."""
import json
import os
import subprocess

import pytest

from conftest import M61, PKG

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
CLI = os.path.join(PKG, "bin", "modlin")


def run(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout.splitlines()


def test_readme_rank_500():
    out = run("-R", "500", "-p", str(M61), "-S", "1", "--prng", "mixmax17")
    assert out == GOLD["reference"]["readme_rank500_stdout"]


def test_readme_lc_1000():
    out = run("-L", "1000", "-p", str(M61), "-S", "1", "--prng", "mixmax17")
    assert out == GOLD["reference"]["readme_lc1000_stdout"]


@pytest.mark.parametrize("kernel", ["plain", "tc"])
def test_readme_xoroshiro_rank(kernel):
    out = run("-R", "1000", "-p", "2", "--prng", "xoroshiro128pp", "--kernel", kernel)
    assert out == ["Generator: xoroshiro128++", "Seed: 0x0000000000000000",
                   "Running a modular rank test using 7.629 MiB of RAM: 1 1000×1000 matrix over the field of size 2",
                   "Matrix 1/1\tcorank=0\tp=1"]
    out = run("-R", "1000", "-p", str(M61), "--prng", "xoroshiro128pp", "--kernel", kernel)
    assert out[-1] == "Matrix 1/1\tcorank=0\tp=1"


def test_readme_xoroshiro_lc():
    out = run("-L", "1000", "-p", "2", "--prng", "xoroshiro128pp")
    assert out[2:] == ["Running a modular linear-complexity test using 0.031 MiB of RAM: 1 sequence of length 1000 "
                       "over the field of size 2",
                       "Sequence 1/1\tlinear complexity=503\tp=0.9947916666666666"]
    out = run("-L", "10000", "-p", str(M61), "--prng", "xoroshiro128pp")
    assert out[-1] == "Sequence 1/1\tlinear complexity=5000\tp=1"


def test_reps_match_one_at_a_time(O):
    """`reps` runs on disjoint stretches of the orbit (src/main.rs:82, :152)."""
    out = run("-L", "300", "-p", "65521", "-S", "5", "--prng", "mixmax256", "4")
    assert out[2].startswith("Running a modular linear-complexity test using 0.009 MiB of RAM: 4 sequences")
    x = [int(v) % 65521 for v in O.prng("mixmax256", 5, 1200)]
    for t in range(4):
        lc = O.linear_complexity(65521, x[300 * t:300 * (t + 1)])
        p = O.pretty_p_value(O.lc_left_tail_pvalue(65521, 300, lc))
        assert out[3 + t] == f"Sequence {t + 1}/4\tlinear complexity={lc}\tp={p}"
    out = run("-R", "40", "-p", "97", "-S", "3", "--prng", "mixmax17", "3")
    x = [int(v) % 97 for v in O.prng("mixmax17", 3, 4800)]
    for t in range(3):
        c = 40 - O.rank(97, x[1600 * t:1600 * (t + 1)], 40)
        p = O.pretty_p_value(O.corank_tail_pvalue(97, 40, c))
        assert out[3 + t] == f"Matrix {t + 1}/3\tcorank={c}\tp={p}"


def test_readme_headline_mixmax256_rank_65536():
    """README.md:110-113: MIXMAX-256 fails the rank test once the side
    exceeds its linear complexity 65280 (README.md:98-107). The largest run
    here: a 65536 x 65536 matrix (32 GiB) over 2^61-1 from MIXMAX-256 seed 1
    has corank 65536 - 65280 = 256."""
    out = run("-R", "65536", "-p", str(M61), "-S", "1", "--prng", "mixmax256")
    assert out[0] == "Generator: MIXMAX (TRandomMixMax256, N=256, skip=2)"
    assert out[-1] == "Matrix 1/1\tcorank=256\tp=1e-307"


def test_rank_reps_batched_equal_one_at_a_time(M, O):
    """-R with several reps runs them in batched launches; every matrix is
    the next n*n outputs of the generator, so the results equal the oracle's
    ranks of consecutive slices of the host stream (src/main.rs:82-125)."""
    n, reps = 120, 5
    want = {}
    for p in (M61, 2, 97):
        out = run("-R", str(n), "-p", str(p), "-S", "7", "--prng", "mixmax17", str(reps))
        stream = O.prng("mixmax17", 7, reps * n * n)
        F = O.Field(p)
        want[p] = []
        for i in range(reps):
            m = [F.reduce(int(x)) for x in stream[i * n * n:(i + 1) * n * n]]
            want[p].append(O.rank(p, m, n))
            corank = n - want[p][-1]
            assert out[3 + i].startswith(f"Matrix {i + 1}/{reps}\tcorank={corank}\tp="), (p, i, out[3 + i])
    # MIXMAX is linear over F_(2^61-1): its 120 x 120 matrices there have rank 34.
    g = M.prng.Prng("mixmax17", 7)
    assert M.fp.rank_prng_batch(M61, g, n, reps) == want[M61]
