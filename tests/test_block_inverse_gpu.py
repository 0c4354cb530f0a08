"""modlin_block_inverse_device: -P^-1 of a 64 x 64 block (the multiplier
block of a rank block step) against exact Python Gauss-Jordan, on every field
policy, on the recursive path (large p) and the pivoting one (small p, and
blocks whose leading 16- or 32-block or Schur complement is singular, where
the recursive path hands over)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

M61 = (1 << 61) - 1
PRIMES = [M61, (1 << 62) - 57, (1 << 63) - 25, 2147483647, 1048583, 65521, 7, 2]


def inv_mod(P, p):
    n = len(P)
    A = [[int(x) % p for x in row] + [1 if i == j else 0 for j in range(n)] for i, row in enumerate(P)]
    for c in range(n):
        r = next((r for r in range(c, n) if A[r][c]), None)
        if r is None:
            return None
        A[c], A[r] = A[r], A[c]
        inv = pow(A[c][c], p - 2, p)
        A[c] = [x * inv % p for x in A[c]]
        for r in range(n):
            if r != c and A[r][c]:
                f = A[r][c]
                A[r] = [(x - f * y) % p for x, y in zip(A[r], A[c])]
    return [row[n:] for row in A]


def device_inverse(M, p, P, ld=64):
    buf = np.zeros((64, ld), dtype=np.uint64)
    buf[:, :64] = np.array(P, dtype=np.uint64)
    t = torch.from_numpy(buf.reshape(-1).view(np.int64)).cuda()
    out = torch.empty(64 * 64, dtype=torch.int64, device="cuda")
    ok = M.fp.block_inverse_device(p, t.data_ptr(), ld, out.data_ptr())
    torch.cuda.synchronize()
    return ok, out.cpu().numpy().view(np.uint64).reshape(64, 64)


def cases(p, rng):
    def rand():
        return [[int(x) for x in rng.integers(0, p, 64, dtype=np.uint64)] for _ in range(64)]
    P = rand()
    yield "random", P, 64
    Q = rand()
    for i in range(8):
        Q[i][0] = 0  # pivot of column 0 below the first rows
    yield "leading-zeros", Q, 64
    Q = rand()
    for j in range(16):
        Q[0][j] = 0  # leading 16 x 16 block singular
    yield "lead16-singular", Q, 64
    Q = rand()
    for j in range(32):
        Q[20][j] = Q[3][j] * 5 % p  # leading 32 x 32 block singular
    yield "lead32-singular", Q, 64
    yield "strided", rand(), 100
    Q = rand()
    Q[10] = [x * 3 % p for x in Q[3]]
    yield "singular", Q, 64


@pytest.mark.parametrize("p", PRIMES)
def test_block_inverse(M, p):
    rng = np.random.default_rng(p % 1000003)
    for name, P, ld in cases(p, rng):
        ref = inv_mod(P, p)
        ok, got = device_inverse(M, p, P, ld)
        assert ok == (ref is not None), (p, name)
        if ref is None:
            continue
        want = np.array([[(p - x) % p for x in row] for row in ref], dtype=np.uint64)
        assert np.array_equal(got, want), (p, name)
