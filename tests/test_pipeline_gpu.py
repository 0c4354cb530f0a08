"""The block pipeline's launch modes give the oracle's results.

Every kernel of the rank's block pipeline is launched with programmatic
dependent launch unless MODLIN_PDL=0 (read once per process), and the kernels
of a speculatively queued step are predicated on a device failure word. These
tests rank the same matrices in a child process without PDL and compare both
runs with the oracle: over 2^61 - 1 (limb planes written by the epilogues),
over a 16-bit prime (split kernels), and on a matrix whose planted dependent
columns make block steps fail mid-pipeline (the skipped step's panel takes the
general path and the pipeline restarts).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
M61 = (1 << 61) - 1

CHILD = r"""
import json, sys
import numpy as np
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/modlin-rs_b200"]
import modlin
out = []
for path, p, n in json.loads(sys.argv[2]):
    m = np.load(path)
    r, pc = modlin.rank(p, m, n, kernel="tc", pivot_cols=True)
    out.append([r, pc])
print(json.dumps(out))
"""


def _cases(O, tmp_path):
    cases = []
    m = O.gen_planted(M61, 600, 41, 1100 * 1100)
    cases.append((m, M61, 1100))
    m = O.gen_uniform(65521, 42, 700 * 700)
    cases.append((m, 65521, 700))
    m, _ = O.gen_dependent(M61, 1536, 43, 24, 40)
    cases.append((m, M61, 1536))
    paths = []
    for i, (m, p, n) in enumerate(cases):
        path = str(tmp_path / f"case{i}.npy")
        np.save(path, np.ascontiguousarray(m, dtype=np.uint64))
        paths.append([path, p, n])
    return cases, paths


def test_rank_with_and_without_pdl_vs_oracle(M, O, tmp_path):
    cases, paths = _cases(O, tmp_path)
    want = [O.rank(p, m, n, with_pcols=True) for m, p, n in cases]
    assert want[2][0] < 1536  # the planted dependencies make block steps fail
    got_pdl = [M.rank(p, m, n, kernel="tc", pivot_cols=True) for m, p, n in cases]
    for (r, pc), (er, epc) in zip(got_pdl, want):
        assert r == er and list(pc) == list(epc)
    env = dict(os.environ, MODLIN_PDL="0")
    res = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(paths)], env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    got = json.loads(res.stdout.strip().splitlines()[-1])
    for (r, pc), (er, epc) in zip(got, want):
        assert r == er and list(pc) == list(epc)
