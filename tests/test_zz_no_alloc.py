"""The no-allocation Berlekamp-Massey entry point.

modlin_linear_complexity_device_noalloc exists for callers that cannot
allocate device memory when they call in (their pool allocator owns the
device memory, or their loop must not pay cudaMalloc's implicit
synchronisation); its scratch is shared memory or a fixed device array.

The tests call it through the C ABI: two calls in a row — a long uniform
sequence (scratch in the array), then a shorter planted one, so the second
call starts from the first call's leftovers — each checked against the
allocating entry point, modlin_linear_complexity_device, and against the
oracle, exactly (linear complexities are integers: tolerance zero); n = 0; a
call on a non-default stream; and that a call after the set-up call leaves
the device's free memory unchanged. This file is collected last and passes
alone in a fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M61 = (1 << 61) - 1


def _call(M, p, d_s, n, out, stream=None):
    rc = M.lib().modlin_linear_complexity_device_noalloc(p, d_s, n, out.data_ptr(), stream)
    assert rc == 0, M.lib().modlin_strerror(rc)


def test_no_alloc_matches_allocating_entry_point_and_oracle(M, O):
    import torch

    cases = [(M61, O.gen_uniform(M61, 41, 20000)), (65521, O.gen_planted(65521, 700, 42, 5000))]
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    for p, s in cases:
        d_s = torch.from_numpy(np.ascontiguousarray(s).view(np.int64)).cuda()
        _call(M, p, d_s.data_ptr(), s.size, out)
        torch.cuda.synchronize()
        got = int(out.item())
        want = M.fp.linear_complexity_device(p, d_s.data_ptr(), s.size)
        assert got == want == O.linear_complexity(p, s), (p, s.size, got, want)
    assert got == 700


def test_no_alloc_empty_sequence_and_stream(M, O):
    import torch

    out = torch.full((1,), 99, dtype=torch.int64, device="cuda")
    _call(M, M61, None, 0, out)
    torch.cuda.synchronize()
    assert int(out.item()) == 0
    s = O.gen_planted(M61, 1500, 43, 9000)
    d_s = torch.from_numpy(np.ascontiguousarray(s).view(np.int64)).cuda()
    out2 = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    st = torch.cuda.Stream()
    _call(M, M61, d_s.data_ptr(), s.size, out2, ctypes.c_void_p(st.cuda_stream))
    st.synchronize()
    assert int(out2.item()) == 1500


def test_no_alloc_call_leaves_free_memory_unchanged(M, O):
    import torch

    p = 2147483647
    s = O.gen_uniform(p, 44, 30000)
    d_s = torch.from_numpy(np.ascontiguousarray(s).view(np.int64)).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    _call(M, p, None, 0, out)  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _call(M, p, d_s.data_ptr(), s.size, out)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert int(out.item()) == O.linear_complexity(p, s)


def test_no_alloc_rejects_sizes_beyond_its_array(M):
    fn = M.lib().modlin_linear_complexity_device_noalloc
    rc = fn(M61, ctypes.c_void_p(16), (1 << 18) + 1, ctypes.c_void_p(16), None)
    assert rc == -2  # MODLIN_EINVAL_N, before any device access
