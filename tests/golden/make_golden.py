"""Regenerates tests/golden/golden.json.

Two kinds of content:
* ``reference`` — known answers taken from the modlin crate's own tests and
  README (tests/test_prng.rs:23-34, :37-48, :51-62, :87-98,
  tests/test_stats.rs:11-71, README.md:61-158). They pin the oracle.
* ``oracle`` — outputs of the pinned CPU oracle on seeded inputs (p-values as
  exact float hex, ranks with column profiles, linear complexities with
  multiply-add counts), frozen so the product's host code and GPU kernels are
  checked against fixed vectors as well as against the live oracle.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

M61 = 2305843009213693951

REFERENCE = {
    # tests/test_prng.rs — first 10 raw 61-bit outputs (next_u64() >> 3) for
    # seed 1234567890123456789, printed by ROOT's mixmax.h/.icc.
    "mixmax_seed": 1234567890123456789,
    "mixmax17": [725153038902651861, 1378221679953707950, 1286954255613532202, 2183378240693018162,
                 480095223529858829, 1028486193651132422, 1683776858464191402, 752698145398996242,
                 1196878046144236647, 1221112387665998636],
    "mixmax240": [1894724080392768937, 2178403735632896525, 82974682673747095, 1362029167703491378,
                  175589691633294316, 1981764336260928646, 1644676922156291251, 463159379824582110,
                  73102843550620337, 783499878333038877],
    "mixmax256": [379984832372095102, 2262036764019001978, 952890261108261993, 1848869284066170746,
                  412703182074144958, 1796627384723021327, 1959941208714421405, 1149684300799040022,
                  525039624349349232, 110320404022327900],
    # tests/test_prng.rs:87-98 — xoroshiro128++ from SplitMix64(0).
    "xoroshiro_seed0": [8027914721839836897, 13805533416164201645, 5256508173613850168, 7973558954284022901,
                        8526501294691771125, 6116102375994396471, 16028966417245382669, 12808598746819302742,
                        15824426267781808726, 5829521525559713354],
    # README.md end-to-end runs: (generator, test, size, p, seed) -> (statistic, p-value string)
    "readme_runs": [
        ["mixmax17", "R", 500, M61, 1, 432, "1e-307"],
        ["mixmax17", "L", 1000, M61, 1, 272, "1e-307"],
        ["mixmax256", "L", 200000, M61, 1, 65280, "1e-307"],
        ["xoroshiro128pp", "R", 1000, 2, 0, 0, "1"],
        ["xoroshiro128pp", "L", 1000, 2, 0, 503, "0.9947916666666666"],
        ["xoroshiro128pp", "R", 1000, M61, 0, 0, "1"],
        ["xoroshiro128pp", "L", 10000, M61, 0, 5000, "1"],
    ],
    # README.md stdout lines of the 500x500 MIXMAX-17 run (src/main.rs:23-26, :74-78, :121-125).
    "readme_rank500_stdout": [
        "Generator: MIXMAX (TRandomMixMax17, N=17)",
        "Seed: 0x0000000000000001",
        "Running a modular rank test using 1.907 MiB of RAM: 1 500×500 matrix over the field of size "
        "2305843009213693951",
        "Matrix 1/1\tcorank=432\tp=1e-307",
    ],
    "readme_lc1000_stdout": [
        "Generator: MIXMAX (TRandomMixMax17, N=17)",
        "Seed: 0x0000000000000001",
        "Running a modular linear-complexity test using 0.031 MiB of RAM: 1 sequence of length 1000 over the "
        "field of size 2305843009213693951",
        "Sequence 1/1\tlinear complexity=272\tp=1e-307",
    ],
}

PRIMES = [2, 3, 97, 65537, 2147483647, M61, (1 << 62) + 135, (1 << 63) - 25]


def main():
    g = {"reference": REFERENCE, "oracle": {}}
    o = g["oracle"]
    # p-values on a grid spanning both CDF branches and the floor.
    pv = []
    for p in [2, 3, 5, 7, 127, 65521, 2147483647, M61]:
        for n in [1, 2, 5, 24, 64, 100, 305, 1000, 10000]:
            for c in sorted({0, 1, 2, 3, n // 3, n // 2, n - 1, n}):
                if 0 <= c <= n:
                    pv.append([p, n, c, O.corank_tail_pvalue(p, n, c).hex(), O.lc_left_tail_pvalue(p, n, c).hex()])
    o["pvalues"] = pv
    o["pretty"] = [[x.hex(), O.pretty_p_value(x)] for x in
                   [1e-307, 0.9947916666666666, 0.5, 0.75, 1e-4, 9.99e-5, 2.5e-5, 0.123456789, 1e16, 1.5e16,
                    123.0, 1234567.125, 3.0517578125e-05, 0.34375, 5e-324, 1.7976931348623157e308]]
    # Seeded rank cases with column profiles (uniform and planted, several primes).
    ranks = []
    for p in [2, 127, 65521, 2147483647, M61]:
        for n, L, seed in [(70, 0, 1), (130, 40, 2), (200, 0, 3), (129, 129, 4), (96, 13, 5)]:
            if L:
                m = O.gen_planted(p, L, seed, n * n)
            else:
                m = O.gen_uniform(p, seed, n * n)
            r, pcols = O.rank(p, m, n, with_pcols=True)
            ranks.append({"p": p, "n": n, "L": L, "seed": seed, "rank": r, "pcols": pcols})
    o["ranks"] = ranks
    lcs = []
    for p in [2, 3, 65521, 2147483647, M61]:
        for n, L, seed in [(1, 0, 1), (2, 0, 2), (300, 0, 3), (500, 17, 4), (1000, 0, 5), (777, 250, 6)]:
            s = O.gen_planted(p, L, seed, n) if L else O.gen_uniform(p, seed, n)
            lc, nd, na = O.linear_complexity(p, s, with_macs=True)
            lcs.append({"p": p, "n": n, "L": L, "seed": seed, "lc": lc, "dot_macs": nd, "axpy_macs": na})
    o["lcs"] = lcs
    o["uniform_heads"] = {str(p): [int(x) for x in O.gen_uniform(p, 7, 16)] for p in [2, 127, 65521, M61]}
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(g, fh, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
