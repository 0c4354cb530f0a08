"""Batch plans: built once, launched without host synchronisation, captured in
a CUDA graph and replayed; every replay gives the oracle's ranks and linear
complexities."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu

PRIMES = [2, 127, 65521, 2**31 - 1, M61, 2**63 - 25]


def _arena(torch, arrays):
    total = sum(a.size for a in arrays)
    host = np.zeros(max(total, 1), dtype=np.uint64)
    offs, o = [], 0
    for a in arrays:
        host[o:o + a.size] = a
        offs.append(o)
        o += a.size
    dev = torch.from_numpy(host.view(np.int64)).cuda()
    return dev, [dev.data_ptr() + 8 * x for x in offs]


def test_rank_plan_graph_replay(M, O):
    import torch
    rng = np.random.default_rng(17)
    items = []
    for i in range(60):
        p = PRIMES[i % len(PRIMES)]
        n = int(rng.integers(1, 400))
        a = M.gen.planted(p, int(rng.integers(1, n + 1)), 50 + i, n * n) if i % 3 == 0 else M.gen.uniform(p, 50 + i, n * n)
        items.append((p, n, a))
    want = [O.rank(p, a, n) for p, n, a in items]
    pristine, _ = _arena(torch, [a for _, _, a in items])
    work = pristine.clone()
    ptrs = []
    o = 0
    for _, n, _ in items:
        ptrs.append(work.data_ptr() + 8 * o)
        o += n * n
    out = torch.full((len(items),), -1, dtype=torch.int64, device="cuda")
    plan = M.fp.BatchPlan("rank", [p for p, _, _ in items], ptrs, [n for _, n, _ in items], out.data_ptr())
    # Plain launch first (on the default stream).
    plan.launch()
    torch.cuda.synchronize()
    assert out.cpu().tolist() == want
    # Captured: restore the matrices, then rank them all.
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            work.copy_(pristine)
            plan.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        out.fill_(-1)
        g.replay()
        torch.cuda.synchronize()
        assert out.cpu().tolist() == want
    plan.free()


def test_lc_plan_graph_replay(M, O):
    import torch
    rng = np.random.default_rng(23)
    items = []
    for i in range(80):
        p = PRIMES[i % len(PRIMES)]
        n = int(rng.integers(1, 3000))
        s = M.gen.planted(p, int(rng.integers(1, n // 3 + 2)), 9 + i, n) if i % 2 else M.gen.uniform(p, 9 + i, n)
        items.append((p, s))
    want = [O.linear_complexity(p, s) for p, s in items]
    dev, ptrs = _arena(torch, [s for _, s in items])
    out = torch.full((len(items),), -1, dtype=torch.int64, device="cuda")
    plan = M.fp.BatchPlan("lc", [p for p, _ in items], ptrs, [s.size for _, s in items], out.data_ptr())
    g = torch.cuda.CUDAGraph()
    st = torch.cuda.Stream()
    st.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(st):
        with torch.cuda.graph(g, stream=st):
            plan.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().wait_stream(st)
    for _ in range(2):
        out.fill_(-1)
        g.replay()
        torch.cuda.synchronize()
        assert out.cpu().tolist() == want
    plan.free()


def test_plan_rejects_bad_input(M):
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    with pytest.raises(M.ModlinError):
        M.fp.BatchPlan("rank", [1], [out.data_ptr()], [1], out.data_ptr())
    with pytest.raises(M.ModlinError):
        M.fp.BatchPlan("rank", [M61], [out.data_ptr()], [8193], out.data_ptr())
