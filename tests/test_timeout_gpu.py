"""Failure detection on the device: a bounded wait that expires.

Every device-side wait of the library is bounded; when one gives up, the
kernel records an error and returns, and the call reports MODLIN_ETIMEOUT
(the reference has no device waits; it panics on errors, src/fp.rs:50-51).
The test makes a wait run out on purpose without faulting or hanging the GPU:
modlin_testing_grid_timeout_once gives the next grid Berlekamp-Massey launch
a short spin limit and has one CTA skip its arrival at the first step's grid
barrier. The call must return MODLIN_ETIMEOUT, and the next normal calls in
the same process must be exact (the context stays usable, the barrier state
is reset per launch).
"""
import pytest

pytestmark = pytest.mark.gpu

M61 = (1 << 61) - 1
ETIMEOUT = -6


@pytest.mark.parametrize("skip_cta", [0, 5])
def test_grid_barrier_timeout_then_exact(M, O, skip_cta):
    import numpy as np
    import torch

    s = O.gen_planted(M61, 900, 51, 6000)
    d = torch.from_numpy(np.ascontiguousarray(s).view(np.int64)).cuda()
    L = M.lib()
    # ~0.5 ms of spinning per wait at 2 GHz: the launch ends quickly.
    assert L.modlin_testing_grid_timeout_once(1_000_000, skip_cta) == 0
    with pytest.raises(M.ModlinError) as ei:
        M.fp.linear_complexity_device(M61, d.data_ptr(), s.size, kernel="grid", grid_ctas=8)
    assert ei.value.code == ETIMEOUT
    torch.cuda.synchronize()
    # The hook was consumed: the same call now runs normally and is exact.
    want = O.linear_complexity(M61, s)
    assert want == 900
    assert M.fp.linear_complexity_device(M61, d.data_ptr(), s.size, kernel="grid", grid_ctas=8) == want
    assert M.fp.linear_complexity_device(M61, d.data_ptr(), s.size, kernel="cluster") == want
