"""GPU rank through the C ABI vs the CPU oracle (bit-exact ranks and column
profiles). Mirrors tests/test_rank.rs of the reference and adds the README's
500x500 MIXMAX-17 run, edge cases and large-size properties."""
import json
import os

import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
KERNELS = ["plain", "tc"]


def kernels_available(M):
    ks = ["plain"]
    try:
        M.rank(M61, np.eye(130, dtype=np.uint64), 130, kernel="tc")
        ks.append("tc")
    except M.ModlinError:
        pass
    return ks


@pytest.fixture(scope="module")
def ks(M):
    return kernels_available(M)


def test_tc_kernel_present(ks):
    assert "tc" in ks, "the tensor-core trailing update is not built"


@pytest.mark.parametrize("kernel", KERNELS)
def test_rank_of_known_matrices(M, ks, kernel):
    """tests/test_rank.rs:74-97."""
    if kernel not in ks:
        pytest.skip("kernel not built")
    assert M.rank(M61, np.eye(3, dtype=np.uint64), 3, kernel=kernel) == 3
    assert M.rank(M61, [1, 2, 3, 4, 5, 6, 5, 7, 9], 3, kernel=kernel) == 2
    assert M.rank(M61, np.zeros(16, dtype=np.uint64), 4, kernel=kernel) == 0
    assert M.rank(2, [1, 1, 0, 0, 1, 1, 1, 0, 1], 3, kernel=kernel) == 2


@pytest.mark.parametrize("kernel", KERNELS)
def test_blocked_matches_reference(M, O, ks, kernel):
    """tests/test_rank.rs:99-149 — the whole panel-boundary grid, ranks and
    column profiles equal to the oracle's."""
    if kernel not in ks:
        pytest.skip("kernel not built")
    ts = O.TestStream()
    for p in [2, 97, M61]:
        for n in [1, 2, 5, 63, 64, 65, 129, 200, 257, 300]:
            for target in [n, n // 2, n // 3, 1, 0]:
                a = ts.rank_case(p, n, target)
                expected = O.rank_naive(p, a, n)
                r, pc = M.rank(p, a, n, kernel=kernel, pivot_cols=True)
                er, epc = O.rank(p, a, n, with_pcols=True)
                assert r == expected == er, (p, n, target)
                assert pc == epc, (p, n, target)


def test_golden_ranks(M, ks):
    for case in GOLD["oracle"]["ranks"]:
        p, n, L, seed = case["p"], case["n"], case["L"], case["seed"]
        m = M.gen.planted(p, L, seed, n * n) if L else M.gen.uniform(p, seed, n * n)
        for kernel in ks:
            r, pc = M.rank(p, m, n, kernel=kernel, pivot_cols=True)
            assert r == case["rank"] and pc == case["pcols"], (case, kernel)


def test_readme_mixmax17_500(M, ks):
    """README.md:61-71: -R 500 -p 2^61-1 -S 1 -> corank 432, p = 1e-307."""
    g = M.prng.Prng("mixmax17", 1)
    f = M.Field(M61)
    x = g.fill(250000)
    m = np.array([f.reduce(int(v)) for v in x], dtype=np.uint64)
    for kernel in ks:
        r = M.rank(M61, m, 500, kernel=kernel)
        assert 500 - r == 432
        assert M.pretty_p_value(M.corank_tail_pvalue(M61, 500, 500 - r)) == "1e-307"


@pytest.mark.parametrize("p", [2, 3, 127, 65521, 2147483647, M61, (1 << 62) + 135, (1 << 63) - 25])
def test_primes_and_sizes_vs_oracle(M, O, ks, p):
    """Every field policy (Mersenne, Barrett with safe_batch 4..2^64) on
    uniform and planted matrices across panel boundaries."""
    for n, L, seed in [(1, 0, 1), (3, 0, 2), (64, 0, 3), (65, 30, 4), (191, 0, 5), (256, 100, 6), (333, 333, 7)]:
        m = O.gen_planted(p, L, seed, n * n) if L else O.gen_uniform(p, seed, n * n)
        er, epc = O.rank(p, m, n, with_pcols=True)
        for kernel in ks:
            r, pc = M.rank(p, m, n, kernel=kernel, pivot_cols=True)
            assert (r, pc) == (er, epc), (p, n, L, kernel)


def test_degenerate_structures(M, O, ks):
    """Zero columns, zero rows, duplicated rows, a window of zero rows (forces
    later window rounds), rank concentrated in the last rows."""
    p = M61
    rng = np.random.default_rng(9)
    n = 200
    cases = []
    a = rng.integers(0, p, (n, n), dtype=np.uint64)
    a[:, :70] = 0
    cases.append(a)
    b = rng.integers(0, p, (n, n), dtype=np.uint64)
    b[:150] = 0
    cases.append(b)
    c = rng.integers(0, p, (n, n), dtype=np.uint64)
    c[1::2] = c[0::2]
    cases.append(c)
    d = np.zeros((n, n), dtype=np.uint64)
    d[-3:] = rng.integers(0, p, (3, n), dtype=np.uint64)
    cases.append(d)
    e = rng.integers(0, 2, (n, n), dtype=np.uint64)
    e[:64] = 0
    cases.append(e)
    for x in cases:
        er, epc = O.rank(p, x, n, with_pcols=True)
        for kernel in ks:
            assert M.rank(p, x, n, kernel=kernel, pivot_cols=True) == (er, epc)
    for x in cases[-1:]:
        er = O.rank(2, x, n)
        for kernel in ks:
            assert M.rank(2, x, n, kernel=kernel) == er


def test_mid_size_vs_oracle(M, O, ks):
    for p, n, L in [(M61, 1024, 0), (M61, 1100, 300), (65521, 777, 500), (127, 640, 0)]:
        m = O.gen_planted(p, L, 12, n * n) if L else O.gen_uniform(p, 12, n * n)
        er, epc = O.rank(p, m, n, with_pcols=True)
        for kernel in ks:
            assert M.rank(p, m, n, kernel=kernel, pivot_cols=True) == (er, epc), (p, n, L, kernel)


def test_large_iid_full_rank_property(M, ks):
    """At large sides the oracle is too slow: a uniform matrix over 2^61-1 has
    full rank and the identity column profile (up to probability ~1/p)."""
    import torch
    n = 8192
    t = torch.empty(n * n, dtype=torch.int64, device="cuda")
    for kernel in ks:
        M.gen.uniform_device(M61, 7, t.data_ptr(), n * n)
        r, pc = M.fp.rank_device(M61, t.data_ptr(), n, kernel=kernel, pivot_cols=True)
        assert r == n and pc == list(range(n)), kernel


def test_device_generator_matches_host(M):
    import torch
    for p in [2, 127, 65521, 2147483647, M61, (1 << 63) - 25]:
        count = 300_000
        t = torch.empty(count, dtype=torch.int64, device="cuda")
        M.gen.uniform_device(p, 11, t.data_ptr(), count)
        got = t.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, M.gen.uniform(p, 11, count)), p


def test_input_validation(M):
    with pytest.raises(M.ModlinError) as e:
        M.rank(7, [1, 2, 3, 9], 2, check_input=True)
    assert e.value.code == -3
    with pytest.raises(M.ModlinError) as e:
        M.rank(1, [1], 1)
    assert e.value.code == -1
    with pytest.raises(M.ModlinError) as e:
        M.rank(7, [], 0)
    assert e.value.code == -2


def test_host_matrix_untouched(M):
    a = np.arange(1, 26, dtype=np.uint64).reshape(5, 5) % 13
    b = a.copy()
    M.rank(13, a, 5)
    assert np.array_equal(a, b)
