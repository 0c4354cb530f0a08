"""Host build of the device field arithmetic (csrc/field.cuh) checked against
Python integers: the Fermat addition-chain inverse for 2^61 - 1 used by the
block inverse, the binary extended-Euclid inverse, and the lazy reductions
(src/fp.rs:34-114 defines the contract: canonical residues, exact results)."""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "modlin-rs_b200", "csrc")
M61 = (1 << 61) - 1

PROG = r"""
#include <cstdio>
#include <cstdlib>
#define MODLIN_HD inline
#include "field.cuh"
using namespace modlin;
int main(int argc, char** argv) {
  // stdin: lines "a b"; stdout: inv_m61(a) inv_binary(a) mul(a,b) reduce2(a*b + b*b)
  unsigned long long a, b;
  const FpM61 f;
  while (std::scanf("%llu %llu", &a, &b) == 2) {
    const unsigned long long i1 = fp_inv_m61(a), i2 = fp_inv_binary(a, kM61);
    const unsigned long long m = f.mul(a, b), r2 = f.reduce2(f.prod(a, b) + f.prod(b, b));
    std::printf("%llu %llu %llu %llu\n", i1, i2, m, r2);
  }
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_m61_inverses_and_reductions(tmp_path):
    src = tmp_path / "field_host.cpp"
    src.write_text(PROG)
    exe = tmp_path / "field_host"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    rng = random.Random(61)
    vals = [1, 2, 3, M61 - 1, M61 - 2, 1 << 60, (1 << 61) - 3] + [rng.randrange(1, M61) for _ in range(2000)]
    pairs = [(a, rng.randrange(0, M61)) for a in vals]
    out = subprocess.run([str(exe)], input="".join(f"{a} {b}\n" for a, b in pairs), capture_output=True, text=True,
                         check=True).stdout.split("\n")
    for (a, b), line in zip(pairs, out):
        i1, i2, m, r2 = map(int, line.split())
        want = pow(a, M61 - 2, M61)
        assert i1 == want and i2 == want, a
        assert m == a * b % M61
        assert r2 == (a * b + b * b) % M61
