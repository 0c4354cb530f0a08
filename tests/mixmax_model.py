"""MIXMAX as the linear map over F_p, p = 2^61 - 1, that one iteration is
(src/prng.rs:191-222 with canonical residues), and states planted through
it: test helpers for the jump-ahead device fill."""
import numpy as np

M61 = (1 << 61) - 1
# kind: (N, SPECIALMUL, SKIP, SPECIAL) (src/prng.rs:284, :305, :326); -1 is ROOT's -1.
MIX = {"mixmax17": (17, 36, 0, None), "mixmax": (240, 51, 0, 487013230256099140), "mixmax256": (256, 0, 2, -1)}


def mix_step(kind, x):
    """One MIXMAX iteration as the linear map over F_p it is (canonical
    residues, state [sumtot, v1..v_{N-1}])."""
    N, sm, _, special = MIX[kind]
    y = [0] * N
    tp, tv, tot = 0, x[0], x[0]
    for i in range(1, N):
        tpo = (tp << sm) % M61 if sm else 0
        tp = (tp + x[i]) % M61
        tv = (tv + tp + tpo) % M61
        y[i] = tv
        tot = (tot + tv) % M61
    if special is not None:
        t2 = (-x[1]) % M61 if special == -1 else special * x[1] % M61
        y[2] = (y[2] + t2) % M61
        tot = (tot + t2) % M61
    y[0] = tot
    return y


def plant(kind, rng, zeros):
    """A state [sumtot, v1..] with, for each (k, i) in zeros, entry i of the
    state after k iterations = 0 (mod p): the conditions are linear, solved
    together over one free coordinate each."""
    N = MIX[kind][0]
    x = [int(rng.integers(1, M61)) for _ in range(N)]
    js = [3 + 3 * m for m in range(len(zeros))]

    def after(v, k):
        for _ in range(k):
            v = mix_step(kind, v)
        return v

    K = len(zeros)
    A = [[0] * K for _ in range(K)]
    for n, j in enumerate(js):
        e = [0] * N
        e[j] = 1
        for m, (k, i) in enumerate(zeros):
            A[m][n] = after(e, k)[i]
    rhs = [(-after(x, k)[i]) % M61 for k, i in zeros]
    # Gauss-Jordan mod p on the K x K system A d = rhs
    for c in range(K):
        r = next(r for r in range(c, K) if A[r][c])
        A[c], A[r], rhs[c], rhs[r] = A[r], A[c], rhs[r], rhs[c]
        inv = pow(A[c][c], M61 - 2, M61)
        A[c] = [a * inv % M61 for a in A[c]]
        rhs[c] = rhs[c] * inv % M61
        for r in range(K):
            if r != c and A[r][c]:
                f = A[r][c]
                A[r] = [(a - f * b) % M61 for a, b in zip(A[r], A[c])]
                rhs[r] = (rhs[r] - f * rhs[c]) % M61
    for n, j in enumerate(js):
        x[j] = (x[j] + rhs[n]) % M61
    for k, i in zeros:
        assert after(x, k)[i] == 0
    return x


def set_mix_state(g, kind, x, counter):
    N = MIX[kind][0]
    words = np.zeros(N + 2, dtype=np.uint64)
    words[0] = x[0]  # v[0]: never read
    words[1:N] = x[1:]
    words[N] = x[0]
    words[N + 1] = counter
    g.set_state(words)
