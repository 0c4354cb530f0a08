"""The column-sharded rank's device backend (modlin.shard.DeviceOps: block
inverse, multiplier and trailing-update entry points, the one-GPU engine for
the gathered rest) in one process on one GPU, against the oracle. The
exchanges between processes are covered on the CPU (tests/test_shard.py)."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu


def test_sharded_rank_device_one_gpu(M, O):
    import torch
    from modlin.shard import DeviceOps, rank_sharded, scatter_columns

    class Counting(DeviceOps):
        steps = 0

        def multipliers(self, *a):
            Counting.steps += 1
            return super().multipliers(*a)

    cases = [(M61, 1000, 0, 15), (M61, 700, 300, 4), (65521, 530, 0, None), ((1 << 62) - 57, 300, 0, 4),
             (2, 200, 0, None), (M61, 50, 0, 0)]
    for p, n, L, steps in cases:
        a = O.gen_planted(p, L, 4, n * n) if L else O.gen_uniform(p, 4, n * n)
        local = torch.from_numpy(scatter_columns(a, n, 0, 1).view(np.int64)).cuda()
        Counting.steps = 0
        got = rank_sharded(p, local, n, ops=Counting(p))
        assert got == O.rank(p, a, n), (p, n, L)
        if steps is not None:
            assert Counting.steps == steps, (p, n, L, Counting.steps)
