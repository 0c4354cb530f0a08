"""The no-allocation Berlekamp-Massey entry point.

modlin_linear_complexity_device_noalloc exists for callers that cannot
allocate device memory when they call in (their pool allocator owns the
device memory, or their loop must not pay cudaMalloc's implicit
synchronisation); its scratch is a fixed device array. This test calls it
through the C ABI twice in a row — a long uniform sequence, then a shorter
planted one, so the second call starts from the first call's leftovers in
the shared array — and checks each result against the allocating entry
point, modlin_linear_complexity_device, exactly (linear complexities are
integers: tolerance zero). It sits in its own file, collected last, and
passes alone in a fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M61 = (1 << 61) - 1


def test_no_alloc_matches_allocating_entry_point(M, O):
    import torch

    fn = M.lib().modlin_linear_complexity_device_noalloc
    cases = [(M61, O.gen_uniform(M61, 41, 20000)), (65521, O.gen_planted(65521, 700, 42, 5000))]
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    for p, s in cases:
        d_s = torch.from_numpy(np.ascontiguousarray(s).view(np.int64)).cuda()
        rc = fn(p, d_s.data_ptr(), s.size, out.data_ptr(), None)
        assert rc == 0, M.lib().modlin_strerror(rc)
        torch.cuda.synchronize()
        got = int(out.item())
        want = M.fp.linear_complexity_device(p, d_s.data_ptr(), s.size)
        assert got == want, (p, s.size, got, want)
    assert got == 700


def test_no_alloc_rejects_sizes_beyond_its_array(M):
    fn = M.lib().modlin_linear_complexity_device_noalloc
    rc = fn(M61, ctypes.c_void_p(16), (1 << 18) + 1, ctypes.c_void_p(16), None)
    assert rc == -2  # MODLIN_EINVAL_N, before any device access
