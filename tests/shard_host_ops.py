"""Exact host arithmetic for the column-sharded rank's per-process compute
(test infrastructure: the CPU multi-process tests plug it into
modlin.shard.rank_sharded in place of the GPU backend)."""
import numpy as np
import torch

PANEL = 64


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


def _obj(t):
    return t.contiguous().numpy().view(np.uint64).astype(object)


def _tensor(a):
    return torch.from_numpy(np.array(a, dtype=object).astype(np.uint64).view(np.int64))


class HostOps:
    def __init__(self, p, oracle):
        self.p, self.O = p, oracle

    def block_inverse(self, local, r0, c0):
        inv = inv_mod(_obj(local[r0:r0 + PANEL, c0:c0 + PANEL]).tolist(), self.p)
        if inv is None:
            return None
        return _tensor([[(-x) % self.p for x in row] for row in inv]).reshape(-1)

    def multipliers(self, local, r0, c0, Vneg):
        X = _obj(local[r0 + PANEL:, c0:c0 + PANEL])
        Pinv = (-_obj(Vneg).reshape(PANEL, PANEL)) % self.p
        return _tensor(X.dot(Pinv) % self.p).reshape(X.shape[0], PANEL)

    def empty_h(self, rows, like):
        return torch.empty((rows, PANEL), dtype=torch.int64)

    def update(self, local, r0, cstart, H):
        if local.shape[0] - r0 - PANEL <= 0 or local.shape[1] - cstart <= 0:
            return
        C = _obj(local[r0 + PANEL:, cstart:])
        U = _obj(local[r0:r0 + PANEL, cstart:])
        local[r0 + PANEL:, cstart:] = _tensor((C - _obj(H).dot(U)) % self.p).reshape(C.shape)

    def rank(self, block):
        n = block.shape[0]
        return self.O.rank(self.p, block.contiguous().numpy().view(np.uint64).ravel(), n) if n else 0
