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

    def zeros(self, *shape):
        return torch.zeros(shape, dtype=torch.int64)

    def block_inverse(self, local, r0, c0):
        inv = inv_mod(_obj(local[r0:r0 + PANEL, c0:c0 + PANEL]).tolist(), self.p)
        if inv is None:
            return None
        return _tensor([[(-x) % self.p for x in row] for row in inv]).reshape(-1)

    def panel_pivots(self, local, r0, c0, W):
        """Gaussian elimination of local[r0:, c0:c0+W] in row order: per
        column the first non-pivot row that is nonzero there."""
        p = self.p
        B = [list(row) for row in _obj(local[r0:, c0:c0 + W]).tolist()]
        used = [False] * len(B)
        prow, pcol = [], []
        for c in range(W):
            r = next((i for i in range(len(B)) if not used[i] and B[i][c] % p), None)
            if r is None:
                continue
            used[r] = True
            prow.append(r)
            pcol.append(c)
            inv = pow(B[r][c], p - 2, p)
            for i in range(len(B)):
                if not used[i] and B[i][c] % p:
                    f = B[i][c] * inv % p
                    B[i] = [(x - f * y) % p for x, y in zip(B[i], B[r])]
        return prow, pcol

    def sub_inverse(self, local, rows, cols):
        p, pb = self.p, len(rows)
        P = _obj(local[rows][:, cols]).tolist()
        inv = inv_mod(P, p)
        assert inv is not None
        V = [[0] * PANEL for _ in range(PANEL)]
        for i in range(PANEL):
            for j in range(PANEL):
                if i < pb and j < pb:
                    V[i][j] = (-inv[i][j]) % p
                elif i == j:
                    V[i][j] = p - 1
        return _tensor(V).reshape(-1)

    def multipliers(self, local, r0, rows_below, cols, V, out):
        m = len(rows_below)
        H = out[:m]
        H.zero_()
        if m:
            X = np.zeros((m, PANEL), dtype=object)
            X[:, :len(cols)] = _obj(local[list(rows_below)][:, cols])
            Pinv = (-_obj(V).reshape(PANEL, PANEL)) % self.p
            H.copy_(_tensor(X.dot(Pinv) % self.p).reshape(m, PANEL))
        return H

    def move_rows(self, local, r0, perm):
        local[r0:] = local[perm].clone()

    def update(self, local, r0, pb, c_from, c_to, H):
        if local.shape[0] - r0 - pb <= 0 or c_to <= c_from or pb == 0:
            return
        C = _obj(local[r0 + pb:, c_from:c_to])
        U = _obj(local[r0:r0 + pb, c_from:c_to])
        local[r0 + pb:, c_from:c_to] = _tensor((C - _obj(H[:, :pb]).dot(U)) % self.p).reshape(C.shape)
