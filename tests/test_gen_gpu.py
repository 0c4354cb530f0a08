"""Device workload generators vs their host forms (bit-identical streams) and
the oracle's planted generator."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

PRIMES = [2, 3, 127, 65521, 2**31 - 1, M61, 2**63 - 25]


def test_planted_device_matches_host(M, O):
    import torch
    for p in PRIMES:
        for L, count in [(0, 5), (1, 40), (3, 2), (17, 300), (200, 1500), (1500, 4000)]:
            t = torch.empty(max(count, 1), dtype=torch.int64, device="cuda")
            M.gen.planted_device(p, L, 5 + L, t.data_ptr(), count)
            got = t.cpu().numpy().view(np.uint64)[:count]
            want = M.gen.planted(p, L, 5 + L, count)
            assert np.array_equal(got, want), (p, L, count)
            if count <= 300:
                assert np.array_equal(want, O.gen_planted(p, L, 5 + L, count)), (p, L)


def test_planted_batch_device_matches_host(M):
    import torch
    rng = np.random.default_rng(3)
    ps, Ls, seeds, counts, bufs = [], [], [], [], []
    for i in range(300):
        p = PRIMES[i % len(PRIMES)]
        n = int(rng.integers(1, 2000))
        L = int(rng.integers(0, n // 2 + 2))
        ps.append(p)
        Ls.append(L)
        seeds.append(1000 + i)
        counts.append(n)
        bufs.append(torch.empty(n, dtype=torch.int64, device="cuda"))
    M.gen.planted_batch_device(ps, Ls, seeds, [b.data_ptr() for b in bufs], counts)
    for i in range(len(bufs)):
        got = bufs[i].cpu().numpy().view(np.uint64)
        assert np.array_equal(got, M.gen.planted(ps[i], Ls[i], seeds[i], counts[i])), i


def test_planted_device_linear_complexity(M):
    """A planted order-L stream of length >= 2L has linear complexity L
    (a_L != 0 and the initial state generic with overwhelming probability)."""
    import torch
    for p, L, n in [(M61, 1000, 4000), (65521, 777, 3000), (2**31 - 1, 64, 1000)]:
        t = torch.empty(n, dtype=torch.int64, device="cuda")
        M.gen.planted_device(p, L, 9, t.data_ptr(), n)
        assert M.fp.linear_complexity_device(p, t.data_ptr(), n) == L


@pytest.mark.parametrize("p,L,count", [(M61, 64, 1 << 22), (65521, 300, (1 << 22) + 777), (2**63 - 25, 128, 1 << 22)])
def test_planted_device_jump_ahead_matches_host(M, p, L, count):
    """Long streams go through the jump-ahead segments (x^T mod f states,
    segments extended in parallel): every value equals the sequential
    stream's."""
    import torch
    t = torch.empty(count, dtype=torch.int64, device="cuda")
    M.gen.planted_device(p, L, 77, t.data_ptr(), count)
    got = t.cpu().numpy().view(np.uint64)
    want = M.gen.planted(p, L, 77, count)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, (bad[:5], bad.size)
