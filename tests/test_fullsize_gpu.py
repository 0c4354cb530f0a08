"""Parity at the benchmark's full sizes, against the CPU oracle's answers.

"Full rank" alone says little about a 16384 x 16384 uniform matrix: almost
every matrix has it, including one whose elimination went wrong. These tests
pin the large workloads to the oracle (tests/golden/configs.json.gz, made by
tests/golden/make_config_golden.py):

* a 16384^2 matrix over 2^61-1 with 96 planted dependent columns and its last
  257 rows combinations of earlier rows: both trailing kernels must find rank
  16127 and the oracle's pivot-column profile, which skips the planted
  columns (a wrong residue anywhere makes a dependent row look independent);
  the same construction at 2048^2 is checked against the live oracle;
* the headline 16384^2 uniform matrix (SplitMix64(7)): the device
  generator's output has the oracle input's SHA-256, and both kernels give
  the oracle's rank and profile;
* the two long Berlekamp-Massey sequences (n = 200000): device inputs equal
  the oracle's (SHA-256) and the linear complexities equal the oracle's.
"""
import numpy as np
import pytest

import golden_configs as G

pytestmark = pytest.mark.gpu

M61 = (1 << 61) - 1


def _rank_both(M, torch, pristine, n, want_r, want_pcols_sha):
    work = torch.empty_like(pristine)
    for kern in ("tc", "plain"):
        work.copy_(pristine)
        r, pc = M.fp.rank_device(M61, work.data_ptr(), n, kernel=kern, pivot_cols=True)
        assert r == want_r, (kern, r, want_r)
        assert G.host_sha256(np.array(pc, dtype=np.uint64)) == want_pcols_sha, kern
    del work


def test_dependent_rank_2048_vs_live_oracle(M, O):
    import torch

    n = 2048
    m, dep = O.gen_dependent(M61, n, 19, 40, 70)
    want = O.rank(M61, m, n, with_pcols=True)
    assert want[0] == n - 70
    pristine = torch.from_numpy(m.view(np.int64)).cuda()
    _rank_both(M, torch, pristine, n, want[0], G.host_sha256(np.array(sorted(want[1]), dtype=np.uint64)))


def test_dependent_rank_16384_vs_oracle(M, O):
    import torch

    e = G.entry("rank_dependent_16384")
    n = e["n"]
    m, dep = O.gen_dependent(M61, n, e["seed"], len(e["dep_cols"]), e["dep_rows"])
    assert dep == e["dep_cols"]
    assert G.host_sha256(m) == e["input_sha256"]
    assert e["rank"] == n - e["dep_rows"] and e["pcols_are_first_free_columns"]
    pristine = torch.from_numpy(m.view(np.int64)).cuda()
    del m
    _rank_both(M, torch, pristine, n, e["rank"], e["pcols_sha256"])


def test_uniform_16384_vs_oracle(M):
    import torch

    e = G.entry("rank_uniform_16384")
    n = e["n"]
    pristine = torch.empty(n * n, dtype=torch.int64, device="cuda")
    M.gen.uniform_device(M61, e["seed"], pristine.data_ptr(), n * n)
    torch.cuda.synchronize()
    assert G.device_sha256(pristine) == e["input_sha256"]
    _rank_both(M, torch, pristine, n, e["rank"], e["pcols_sha256"])


@pytest.mark.parametrize("name", ["lc_planted_200000", "lc_iid_200000"])
def test_long_berlekamp_massey_vs_oracle(M, name):
    import torch

    e = G.entry(name)
    n = e["n"]
    t = torch.empty(n, dtype=torch.int64, device="cuda")
    if "order" in e:
        M.gen.planted_device(M61, e["order"], e["seed"], t.data_ptr(), n)
    else:
        M.gen.uniform_device(M61, e["seed"], t.data_ptr(), n)
    torch.cuda.synchronize()
    assert G.device_sha256(t) == e["input_sha256"]
    for kern in ("cluster", "grid"):
        assert M.fp.linear_complexity_device(M61, t.data_ptr(), n, kernel=kern) == e["lc"], kern
