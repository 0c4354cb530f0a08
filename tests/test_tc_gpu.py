"""The tensor-core trailing update (tcgen05 kind::i8 limb GEMMs) on its own:
C -= L*U mod p through the C ABI, compared with exact Python integers and
with the u64 Barrett kernel, for every limb count (1, 2, 4, 8 limbs)."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

PRIMES = [127, 251, 65521, 2147483647, 4294967291, M61, (1 << 62) + 135, (1 << 63) - 25]


def rand_res(rng, p, shape):
    return (rng.integers(0, 2**63, shape, dtype=np.uint64) % np.uint64(p)).astype(np.uint64)


def run(M, p, C, L, U, kernel):
    import torch
    Mr, N = C.shape
    K = U.shape[0]
    Lp = np.zeros((Mr, 64 if K <= 64 else 128), dtype=np.uint64)
    Lp[:, :K] = L
    dC = torch.from_numpy(C.view(np.int64).copy()).cuda()
    dL = torch.from_numpy(Lp.view(np.int64).copy()).cuda()
    dU = torch.from_numpy(np.ascontiguousarray(U).view(np.int64).copy()).cuda()
    M.fp.trailing_update_device(p, dC.data_ptr(), N, Mr, N, dL.data_ptr(), dU.data_ptr(), N, K, kernel=kernel)
    torch.cuda.synchronize()
    return dC.cpu().numpy().view(np.uint64)


def exact(p, C, L, U):
    Co = C.astype(object)
    prod = L.astype(object).dot(U.astype(object))
    return ((Co - prod) % p).astype(np.uint64)


@pytest.mark.parametrize("p", PRIMES)
def test_small_exact(M, p):
    rng = np.random.default_rng(p % 1000)
    for Mr, N, K in [(128, 16, 64), (130, 70, 64), (5, 3, 1), (200, 129, 33)]:
        C, L, U = rand_res(rng, p, (Mr, N)), rand_res(rng, p, (Mr, K)), rand_res(rng, p, (K, N))
        want = exact(p, C, L, U)
        assert np.array_equal(run(M, p, C, L, U, "plain"), want), (p, Mr, N, K, "plain")
        assert np.array_equal(run(M, p, C, L, U, "tc"), want), (p, Mr, N, K, "tc")


@pytest.mark.parametrize("p", PRIMES)
def test_extreme_values(M, p):
    """All entries p-1: the largest limb products and accumulator sums."""
    for Mr, N, K in [(256, 256, 64), (129, 33, 64)]:
        C = np.full((Mr, N), p - 1, dtype=np.uint64)
        L = np.full((Mr, K), p - 1, dtype=np.uint64)
        U = np.full((K, N), p - 1, dtype=np.uint64)
        want = exact(p, C[:4, :4], L[:4], U[:, :4])
        got = run(M, p, C, L, U, "tc")
        assert np.array_equal(got[:4, :4], want)
        assert np.array_equal(got, run(M, p, C, L, U, "plain"))


@pytest.mark.parametrize("p", [M61, 2147483647, 65521, 127, (1 << 63) - 25])
def test_large_tc_equals_plain(M, p):
    rng = np.random.default_rng(7)
    for Mr, N, K in [(2048, 1536, 64), (1000, 3001, 17), (4096, 512, 64)]:
        C, L, U = rand_res(rng, p, (Mr, N)), rand_res(rng, p, (Mr, K)), rand_res(rng, p, (K, N))
        assert np.array_equal(run(M, p, C, L, U, "tc"), run(M, p, C, L, U, "plain")), (p, Mr, N, K)


@pytest.mark.parametrize("p", PRIMES)
def test_two_panel_depth_exact(M, p):
    """K up to 128 (two panels per pass, 128-byte limb rows): exact, and the
    largest sums (all entries p-1) still fit the 32-bit accumulators."""
    rng = np.random.default_rng(p % 977)
    for Mr, N, K in [(128, 16, 128), (300, 130, 128), (131, 45, 65), (257, 200, 100)]:
        C, L, U = rand_res(rng, p, (Mr, N)), rand_res(rng, p, (Mr, K)), rand_res(rng, p, (K, N))
        assert np.array_equal(run(M, p, C, L, U, "tc"), exact(p, C, L, U)), (p, Mr, N, K)
    Mr, N, K = 129, 33, 128
    C = np.full((Mr, N), p - 1, dtype=np.uint64)
    L = np.full((Mr, K), p - 1, dtype=np.uint64)
    U = np.full((K, N), p - 1, dtype=np.uint64)
    got = run(M, p, C, L, U, "tc")
    assert np.array_equal(got[:4, :4], exact(p, C[:4, :4], L[:4], U[:, :4]))
    assert (got == got[0, 0]).all()


def test_two_panel_depth_large(M):
    """A K = 128 update equals two K = 64 updates in a row."""
    rng = np.random.default_rng(11)
    for p in [M61, 65521]:
        Mr, N = 3000, 2500
        C, L, U = rand_res(rng, p, (Mr, N)), rand_res(rng, p, (Mr, 128)), rand_res(rng, p, (128, N))
        one = run(M, p, C, L, U, "tc")
        two = run(M, p, run(M, p, C, L[:, :64], U[:64], "tc"), L[:, 64:], U[64:], "tc")
        assert np.array_equal(one, two)
        assert np.array_equal(two, run(M, p, run(M, p, C, L[:, :64], U[:64], "plain"), L[:, 64:], U[64:], "plain"))


@pytest.mark.parametrize("K", [128, 64, 100, 17])
def test_cta_pairs_equal_single_ctas(M, K):
    """Updates over 2^61-1 on CTA pairs (M = 256 MMAs over two SMs, each
    holding half of every B tile) equal the single-CTA kernel's and exact
    Python integers, for row counts that leave the pair's second half partly
    or wholly past the end."""
    p = M61
    L = M.lib()
    rng = np.random.default_rng(K)
    prev = L.modlin_set_tc_pairs(-1)
    try:
        for Mr, N in [(129, 16), (300, 130), (257, 64), (1000, 3000), (2048, 1536)]:
            C, Lm, U = rand_res(rng, p, (Mr, N)), rand_res(rng, p, (Mr, K)), rand_res(rng, p, (K, N))
            L.modlin_set_tc_pairs(1)
            pair = run(M, p, C, Lm, U, "tc")
            L.modlin_set_tc_pairs(0)
            single = run(M, p, C, Lm, U, "tc")
            assert np.array_equal(pair, single), (Mr, N, K)
            if Mr * N <= 40000:
                assert np.array_equal(pair, exact(p, C, Lm, U)), (Mr, N, K)
    finally:
        L.modlin_set_tc_pairs(prev)
