"""Batched rank (one persistent launch over uneven sides and primes) vs the
CPU oracle. Mirrors tests/test_rank.rs's grid with every matrix in one batch,
and adds mixed-prime batches of iid and recurrence-planted matrices."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

PRIMES = [2, 3, 127, 65521, 2**31 - 1, M61, 2**63 - 25]


def test_batch_matches_reference_grid(M, O):
    """tests/test_rank.rs:99-149's whole grid as one batch."""
    ts = O.TestStream()
    items, want = [], []
    for p in [2, 97, M61]:
        for n in [1, 2, 5, 63, 64, 65, 129, 200, 257, 300]:
            for target in [n, n // 2, n // 3, 1, 0]:
                a = ts.rank_case(p, n, target)
                items.append((p, a))
                want.append(O.rank_naive(p, a, n))
    assert M.rank_batch(items) == want


def test_batch_known_and_degenerate(M):
    """tests/test_rank.rs:74-97 plus zero, identity, constant and 1x1 cases."""
    items = [
        (M61, np.eye(3, dtype=np.uint64)),
        (M61, np.array([1, 2, 3, 4, 5, 6, 5, 7, 9], dtype=np.uint64)),
        (M61, np.zeros(16, dtype=np.uint64)),
        (2, np.array([1, 1, 0, 0, 1, 1, 1, 0, 1], dtype=np.uint64)),
        (127, np.zeros(1, dtype=np.uint64)),
        (127, np.array([5], dtype=np.uint64)),
        (65521, np.eye(200, dtype=np.uint64)),
        (65521, np.full(150 * 150, 7, dtype=np.uint64)),
        (2**63 - 25, np.eye(65, dtype=np.uint64)[::-1].copy()),
    ]
    assert M.rank_batch(items) == [3, 2, 0, 2, 0, 1, 200, 1, 65]


def _mixed(M, count, nmax, seed):
    rng = np.random.default_rng(seed)
    items = []
    for i in range(count):
        p = PRIMES[i % len(PRIMES)]
        n = int(rng.integers(1, nmax + 1))
        if i % 2:
            L = int(rng.integers(max(1, n // 4), n + 1))
            a = M.gen.planted(p, L, 1000 + i, n * n)
        else:
            a = M.gen.uniform(p, 1000 + i, n * n)
        items.append((p, a))
    return items


def test_batch_mixed_vs_oracle(M, O):
    items = _mixed(M, 160, 300, 5)
    got = M.rank_batch(items)
    for (p, a), r in zip(items, got):
        n = int(round(a.size ** 0.5))
        assert r == O.rank(p, a, n), (p, n)


def test_batch_device_matches_host_form(M):
    import torch
    items = _mixed(M, 64, 520, 9)
    host = M.rank_batch(items)
    bufs = [torch.from_numpy(a.view(np.int64)).cuda() for _, a in items]
    dev = M.fp.rank_batch_device([p for p, _ in items], [b.data_ptr() for b in bufs],
                                 [int(round(a.size ** 0.5)) for _, a in items])
    assert dev == host
    # The single-matrix engine agrees on the largest ones.
    for (p, a), r in list(zip(items, host))[:8]:
        n = int(round(a.size ** 0.5))
        assert M.rank(p, a, n) == r


def test_batch_empty_and_zero_side(M):
    assert M.rank_batch([]) == []
    assert M.rank_batch([(M61, np.zeros(0, dtype=np.uint64)), (M61, np.eye(2, dtype=np.uint64))]) == [0, 2]


def test_batch_tensor_core_variant_matches_oracle(M, O):
    """The tensor-core batch kernel (one CTA per matrix, trailing updates as
    limb GEMMs on its SM), forced for every job, on every limb count: the
    oracle's ranks, as the integer-pipe kernel's."""
    import torch
    rng = np.random.default_rng(77)
    items = []
    for i in range(42):
        p = PRIMES[i % len(PRIMES)]
        n = int(rng.integers(1, 420))
        a = M.gen.uniform(p, 300 + i, n * n) if i % 2 else M.gen.planted(p, max(1, n // 2), 300 + i, n * n)
        items.append((p, n, a))
    want = [O.rank(p, a, n) for p, n, a in items]
    for kernel in ("tc", "plain"):
        bufs = [torch.from_numpy(a.view(np.int64).copy()).cuda() for _, _, a in items]
        got = M.fp.rank_batch_device([p for p, _, _ in items], [b.data_ptr() for b in bufs],
                                     [n for _, n, _ in items], kernel=kernel)
        assert got == want, kernel
