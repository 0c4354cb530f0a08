"""GPU Berlekamp-Massey through the C ABI vs the CPU oracle. Mirrors
tests/test_linear_complexity.rs and adds the README's runs, the persistent
cooperative kernel, batches of uneven sequences and the bounded-wait path."""
import json
import os

import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


KINDS = ("block", "grid", "cluster")


def lcs_all(M, p, s):
    return {k: M.linear_complexity(p, s, kernel=k) for k in KINDS}


def each(e):
    return {k: e for k in KINDS}


def test_linear_complexity_of_lfsr_sequence(M):
    """tests/test_linear_complexity.rs:72-91."""
    s = [1, 2, 3]
    for i in range(3, 40):
        s.append((3 * s[i - 1] + 5 * s[i - 2] + 7 * s[i - 3]) % M61)
    for k in KINDS:
        assert M.linear_complexity(M61, s, kernel=k) == 3
        assert M.linear_complexity(M61, [4] * 20, kernel=k) == 1
        assert M.linear_complexity(M61, [0] * 20, kernel=k) == 0
    assert M.linear_complexity(M61, []) == 0


def test_matches_reference(M, O):
    """tests/test_linear_complexity.rs:93-133."""
    ts = O.TestStream()
    for p in [2, 3, 97, 65537, M61]:
        for n in [1, 2, 3, 5, 16, 50, 100, 200]:
            s = ts.lc_random(p, n)
            e = O.lc_naive(p, s)
            assert lcs_all(M, p, s) == each(e), (p, n)
        for k in [1, 4, 10, 25]:
            s = ts.lc_lfsr(p, k)
            e = O.lc_naive(p, s)
            assert e <= k
            assert lcs_all(M, p, s) == each(e), (p, k)


def test_golden_lcs(M):
    for c in GOLD["oracle"]["lcs"]:
        p, n, L, seed = c["p"], c["n"], c["L"], c["seed"]
        s = M.gen.planted(p, L, seed, n) if L else M.gen.uniform(p, seed, n)
        assert lcs_all(M, p, s) == each(c["lc"]), c


@pytest.mark.parametrize("p", [2, 127, 65521, 2147483647, M61, (1 << 62) + 135, (1 << 63) - 25])
def test_primes_vs_oracle(M, O, p):
    for n, L, seed in [(700, 0, 1), (1500, 90, 2), (4000, 1999, 3), (5000, 0, 4)]:
        s = O.gen_planted(p, L, seed, n) if L else O.gen_uniform(p, seed, n)
        e = O.linear_complexity(p, s)
        assert lcs_all(M, p, s) == each(e), (p, n, L)


def test_grid_kernel_cta_counts(M, O):
    s = O.gen_uniform(M61, 5, 30000)
    e = O.linear_complexity(M61, s)
    for ctas in [1, 7, 64, 148]:
        assert M.linear_complexity(M61, s, kernel="grid", grid_ctas=ctas) == e


def test_readme_runs(M):
    """README.md:81-88, :98-107, :131-137, :151-158."""
    cases = [("mixmax17", 1, 1000, M61, 272, "1e-307"), ("xoroshiro128pp", 0, 1000, 2, 503, "0.9947916666666666"),
             ("xoroshiro128pp", 0, 10000, M61, 5000, "1"), ("mixmax256", 1, 200000, M61, 65280, "1e-307")]
    for kind, seed, n, p, lc, ps in cases:
        f = M.Field(p)
        x = M.prng.Prng(kind, seed).fill(n)
        s = np.array([f.reduce(int(v)) for v in x], dtype=np.uint64)
        got = M.linear_complexity(p, s)
        assert got == lc, (kind, n)
        assert M.pretty_p_value(M.lc_left_tail_pvalue(p, n, got)) == ps


def test_batch_uneven_mixed_primes(M, O):
    rng = np.random.default_rng(31)
    items, want = [], []
    for i in range(300):
        p = [65521, 2147483647, M61, 2, 97][i % 5]
        n = int(rng.integers(1, 1200))
        if i % 2:
            s = O.gen_uniform(p, 100 + i, n)
        else:
            s = O.gen_planted(p, int(rng.integers(1, max(2, n // 4))), 100 + i, n)
        items.append((p, s))
        want.append(O.linear_complexity(p, s))
    assert M.lc_batch(items) == want


def test_batch_large_sequences_global_workspace(M, O):
    items = [(M61, O.gen_uniform(M61, 40 + i, 9000 + 1000 * i)) for i in range(3)]
    items.append((65521, O.gen_planted(65521, 2500, 7, 12000)))
    assert M.lc_batch(items) == [O.linear_complexity(p, s) for p, s in items]


def test_batch_empty_and_trivial(M):
    assert M.lc_batch([]) == []
    assert M.lc_batch([(7, [])]) == [0]
    assert M.lc_batch([(7, [0, 0, 0]), (7, [1])]) == [0, 1]


def test_input_validation(M):
    with pytest.raises(M.ModlinError) as e:
        M.linear_complexity(7, [1, 2, 7], check_input=True)
    assert e.value.code == -3
    with pytest.raises(M.ModlinError):
        M.linear_complexity(0, [1])


def test_cluster_kernel_long_sequences(M, O):
    """The one-cluster kernel (16 CTAs, one cluster barrier per step) on long
    sequences: equal to the oracle and to the grid kernel, for every field
    policy, up to its length limit."""
    for p, n, L, seed in [(M61, 40000, 0, 1), (65521, 30000, 7000, 2), ((1 << 63) - 25, 20000, 0, 3),
                          (2147483647, 36000, 17000, 4)]:
        s = O.gen_planted(p, L, seed, n) if L else O.gen_uniform(p, seed, n)
        e = O.linear_complexity(p, s)
        assert M.linear_complexity(p, s, kernel="cluster") == e, (p, n, L)
        assert M.linear_complexity(p, s, kernel="grid") == e, (p, n, L)
    import torch
    n = 409600
    t = torch.empty(n, dtype=torch.int64, device="cuda")
    M.gen.planted_device(M61, 100000, 5, t.data_ptr(), n)
    assert M.fp.linear_complexity_device(M61, t.data_ptr(), n, kernel="cluster") == 100000
    with pytest.raises(M.ModlinError) as ex:
        M.fp.linear_complexity_device(M61, t.data_ptr(), n + 1, kernel="cluster")
    assert ex.value.code == -2


def test_shared_memory_boundary_lengths(M, O):
    """Lengths whose c, b, t arrays need just under 48 KiB of dynamic shared
    memory: with the kernels' static shared memory the total passes 48 KiB
    (the launch must opt in)."""
    for n in [2027, 2040, 2047, 2048]:
        s = O.gen_uniform(65521, n, n)
        e = O.linear_complexity(65521, s)
        assert M.linear_complexity(65521, s, kernel="block") == e, n
        assert M.lc_batch([(65521, s), (M61, O.gen_uniform(M61, 1, 100))])[0] == e, n
