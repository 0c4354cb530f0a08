"""Device entry points with stream NULL run on the legacy default stream, so a
copy queued there beforehand (PyTorch's default stream) is ordered before
them."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu


def test_null_stream_orders_after_default_stream_copy(M):
    import torch
    n = 2048
    src = torch.empty(n * n, dtype=torch.int64, device="cuda")
    M.gen.uniform_device(M61, 3, src.data_ptr(), n * n)
    r0 = M.fp.rank_device(M61, src.clone().data_ptr(), n)
    work = torch.zeros_like(src)
    for _ in range(3):
        work.zero_()
        torch.cuda.synchronize()
        work.copy_(src)  # queued on the default stream, not waited for
        assert M.fp.rank_device(M61, work.data_ptr(), n) == r0
    small = [torch.zeros(300 * 300, dtype=torch.int64, device="cuda") for _ in range(20)]
    srcs = []
    for i, t in enumerate(small):
        s = torch.empty_like(t)
        M.gen.uniform_device(M61, 50 + i, s.data_ptr(), t.numel())
        srcs.append(s)
    torch.cuda.synchronize()
    for t, s in zip(small, srcs):
        t.copy_(s)
    assert M.fp.rank_batch_device([M61] * 20, [t.data_ptr() for t in small], [300] * 20) == [300] * 20
