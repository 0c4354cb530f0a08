"""The autotuner: its choices are sane, and every AUTO path still gives the
oracle's results after it has run."""
import numpy as np
import pytest

from conftest import M61

pytestmark = pytest.mark.gpu


def test_autotune_then_auto_paths_exact(M, O):
    rep = M.autotune()
    ch = rep["choice"]
    assert len(ch["tc_crossover"]) == 4 and all(c >= 64 for c in ch["tc_crossover"])
    assert ch["bm_threads"] and all(t in (128, 256, 512, 1024) for t in ch["bm_threads"])
    assert all(t in (128, 256, 512) for t in ch["bm_batch_threads"])
    assert all(k in (200, 96, 48, 24) for k in ch["bm_batch_smem_kib"])
    assert ch["bm_cluster_min"] >= 4096
    assert ch["two_panel_min"] in (0, 2048, 4096, 6144, 8192, 12288, 1 << 30)
    assert len(rep["two_panel_ms"]) == 7
    assert rep["rank_ms"] and rep["bm_block_ms"] and rep["bm_batch_ms"]
    for p in [127, 65521, 2**31 - 1, M61]:
        for n in [100, 300, 700, 1100]:
            a = M.gen.uniform(p, n, n * n)
            r, pc = M.rank(p, a, n, pivot_cols=True)
            want, wpc = O.rank(p, a, n, with_pcols=True)
            assert (r, list(pc)) == (want, wpc), (p, n)
    for n in [500, 3000, 9000, 20000]:
        s = O.gen_uniform(M61, n, n)
        assert M.linear_complexity(M61, s) == O.linear_complexity(M61, s)
    items = [(65521, O.gen_uniform(65521, 7 + i, 200 + 37 * i)) for i in range(40)]
    assert M.lc_batch(items) == [O.linear_complexity(p, s) for p, s in items]
