"""The column-sharded rank's device backend (modlin.shard.DeviceOps: block
inverse, panel pivots, multiplier and trailing-update entry points) in one
process on one GPU, against the oracle. The exchanges between processes are
covered on the CPU (tests/test_shard.py)."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu


def test_sharded_rank_device_one_gpu(M, O):
    import torch
    from modlin.shard import DeviceOps, rank_sharded, scatter_columns

    class Counting(DeviceOps):
        blocks = general = 0

        def block_inverse(self, *a):
            r = super().block_inverse(*a)
            Counting.blocks += r is not None
            return r

        def panel_pivots(self, *a):
            Counting.general += 1
            return super().panel_pivots(*a)

    # (block steps, general steps): full-rank matrices take block steps and a
    # general step on the ragged last panel; the planted rank-300 matrix takes
    # four block steps, a general step with 44 pivots and general steps on the
    # six zero panels after it.
    cases = [(M61, 1000, 0, (15, 1)), (M61, 700, 300, (4, 7)), (65521, 530, 0, None),
             ((1 << 62) - 57, 300, 0, (4, 1)), (2, 200, 0, None), (M61, 50, 0, (0, 1)), (97, 400, 150, None)]
    for p, n, L, steps in cases:
        a = O.gen_planted(p, L, 4, n * n) if L else O.gen_uniform(p, 4, n * n)
        local = torch.from_numpy(scatter_columns(a, n, 0, 1).view(np.int64)).cuda()
        Counting.blocks = Counting.general = 0
        got = rank_sharded(p, local, n, ops=Counting(p))
        assert got == O.rank(p, a, n), (p, n, L)
        if steps is not None:
            assert (Counting.blocks, Counting.general) == steps, (p, n, L, Counting.blocks, Counting.general)


def test_panel_pivots_match_host_elimination(M, O):
    """modlin_panel_pivots_device against the host elimination of the same
    panel: the same pivot columns (an invariant) and pivot rows whose block
    is invertible."""
    import torch
    from shard_host_ops import HostOps, inv_mod
    for p, rows, W, seed in [(M61, 300, 64, 1), (97, 200, 64, 2), (2, 150, 40, 3), (M61, 80, 17, 4)]:
        a = O.gen_planted(p, 20, seed, rows * W).reshape(rows, W) if seed == 1 else \
            O.gen_uniform(p, seed, rows * W).reshape(rows, W)
        t = torch.from_numpy(a.view(np.int64).copy())
        d = t.cuda()
        prow, pcol = M.fp.panel_pivots_device(p, d.data_ptr(), W, rows, W)
        hrow, hcol = HostOps(p, O).panel_pivots(t, 0, 0, W)
        assert sorted(pcol) == hcol, (p, rows, W)
        assert np.array_equal(d.cpu().numpy(), t.numpy())  # the panel is left unchanged
        P = [[int(a[r][c]) for c in pcol] for r in prow]
        assert len(set(prow)) == len(prow) and (not P or inv_mod(P, p) is not None)
