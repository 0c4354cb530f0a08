"""Regenerates tests/golden/configs.json.gz: the CPU oracle's answers on the
benchmark's full-size workloads, so that the GPU tests and bench.py check
every large run against the oracle instead of against "full rank" alone.

Each entry records the workload's parameters, a SHA-256 of its input (the
residues as little-endian u64, in the order the benchmark lays them out) and
the oracle's results:

* rank_uniform_16384   16384^2 uniform residues over 2^61-1, SplitMix64(7):
                       rank and pivot columns
* rank_dependent_16384 the same size, SplitMix64(9), with 96 planted dependent
                       columns and the last 257 rows combinations of earlier
                       rows (oracle.gen_dependent): rank 16127, a pivot-column
                       profile that skips the planted columns
* rank_planted_16384   rows = successive windows of an order-4096 recurrence,
                       SplitMix64(8): rank and pivot columns
* lc_planted_200000 / lc_iid_200000   Berlekamp-Massey of the two long
                       sequences (order-65280 recurrence, seed 21; iid, seed 22):
                       linear complexity and multiply-add counts
* rank_batch_4096      the 4096-matrix batch (bench.rank_batch_jobs): every
                       rank and the batch's modMAC work
* lc_batch_65536       the 65536-sequence batch (bench.bm_batch_jobs): every
                       linear complexity

Pivot columns are stored as the SHA-256 of the increasing column list (u64).
Batch inputs are checked by a checksum of checksums: the SHA-256 of the
concatenated per-job SHA-256 digests, in job order.

Run from the repository root (about 50 minutes on 8 cores; --only NAME runs
one entry and keeps the others):
    python tests/golden/make_config_golden.py [--only NAME] [--procs N]
"""
import argparse
import gzip
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402

M61 = (1 << 61) - 1
OUT = os.path.join(HERE, "configs.json.gz")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()


def work_of(n, pcols):
    return sum((n - 1 - k) * (n - 1 - j) for k, j in enumerate(pcols))


def pcols_entry(n, r, pc):
    return {"rank": r, "pcols_sha256": sha(np.array(sorted(pc), dtype=np.uint64)),
            "pcols_is_prefix": sorted(pc) == list(range(r)), "work_modmac": work_of(n, pc)}


def rank_uniform(n=16384, seed=7):
    m = O.gen_uniform(M61, seed, n * n)
    e = {"n": n, "p": M61, "seed": seed, "input_sha256": sha(m)}
    r, pc = O.rank(M61, m, n, with_pcols=True)
    e.update(pcols_entry(n, r, pc))
    return e


def rank_dependent(n=16384, seed=9, ncols=96, nrows=257):
    m, dep = O.gen_dependent(M61, n, seed, ncols, nrows)
    e = {"n": n, "p": M61, "seed": seed, "dep_cols": dep, "dep_rows": nrows, "input_sha256": sha(m)}
    r, pc = O.rank(M61, m, n, with_pcols=True)
    e.update(pcols_entry(n, r, pc))
    ds = set(dep)
    e["pcols_are_first_free_columns"] = sorted(pc) == [c for c in range(n) if c not in ds][:r]
    return e


def rank_planted(n=16384, L=4096, seed=8):
    m = O.gen_planted(M61, L, seed, n * n)
    e = {"n": n, "p": M61, "order": L, "seed": seed, "input_sha256": sha(m)}
    r, pc = O.rank(M61, m, n, with_pcols=True)
    e.update(pcols_entry(n, r, pc))
    return e


def lc_long(planted, n=200000, L=65280):
    seed = 21 if planted else 22
    s = O.gen_planted(M61, L, seed, n) if planted else O.gen_uniform(M61, seed, n)
    lc, dot, axpy = O.linear_complexity(M61, s, with_macs=True)
    e = {"n": n, "p": M61, "seed": seed, "input_sha256": sha(s), "lc": lc, "dot_macs": dot, "axpy_macs": axpy}
    if planted:
        e["order"] = L
    return e


# ---- batches ---------------------------------------------------------------
# Worker processes are forked after the parent has generated the iid streams
# (no GPU is involved anywhere in this script), so they read them shared.
_STREAMS = {}


def _rank_job(arg):
    i, p, n, planted, L, seed, pi, off = arg
    a = O.gen_planted(p, L, seed, n * n) if planted else _STREAMS[pi][off:off + n * n]
    r, pc = O.rank(p, a, n, threads=1, with_pcols=True)
    return i, r, work_of(n, pc), hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def _lc_job(arg):
    i, p, n, planted, L, seed, pi, off = arg
    s = O.gen_planted(p, L, seed, n) if planted else _STREAMS[pi][off:off + n]
    lc, dot, axpy = O.linear_complexity(p, s, with_macs=True)
    return i, lc, dot + axpy, hashlib.sha256(np.ascontiguousarray(s).tobytes()).digest()


def _batch(kind, procs):
    import bench
    global _STREAMS
    if kind == "rank":
        jobs, iid_seeds = bench.rank_batch_jobs()
        primes, size = bench.RANK_PRIMES, (lambda n: n * n)
    else:
        jobs, iid_seeds = bench.bm_batch_jobs()
        primes, size = bench.BM_PRIMES, (lambda n: n)
    args, offs = [], [0] * len(primes)
    for i, (pi, n, planted, L, seed) in enumerate(jobs):
        off = 0
        if not planted:
            off = offs[pi]
            offs[pi] += size(n)
        args.append((i, primes[pi], n, planted, L, seed, pi, off))
    _STREAMS = {pi: O.gen_uniform(primes[pi], iid_seeds[pi], offs[pi]) for pi in range(len(primes)) if offs[pi]}
    args.sort(key=lambda a: -a[2])  # largest jobs first, so the pool ends together
    res = [None] * len(jobs)
    with mp.get_context("fork").Pool(procs) as pool:
        for out in pool.imap_unordered(_rank_job if kind == "rank" else _lc_job, args, chunksize=1):
            res[out[0]] = out[1:]
    _STREAMS = {}
    digest = hashlib.sha256(b"".join(r[2] for r in res)).hexdigest()
    if kind == "rank":
        return {"count": len(jobs), "input_sha256_of_job_sha256": digest, "ranks": [r[0] for r in res],
                "work_modmac": sum(r[1] for r in res)}
    return {"count": len(jobs), "input_sha256_of_job_sha256": digest, "lcs": [r[0] for r in res],
            "macs": sum(r[1] for r in res)}


ENTRIES = {
    "lc_planted_200000": lambda procs: lc_long(True),
    "lc_iid_200000": lambda procs: lc_long(False),
    "rank_uniform_16384": lambda procs: rank_uniform(),
    "rank_dependent_16384": lambda procs: rank_dependent(),
    "rank_batch_4096": lambda procs: _batch("rank", procs),
    "lc_batch_65536": lambda procs: _batch("lc", procs),
    "rank_planted_16384": lambda procs: rank_planted(),
}


def load():
    if os.path.exists(OUT):
        with gzip.open(OUT, "rt") as f:
            return json.load(f)
    return {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", action="append", choices=sorted(ENTRIES))
    ap.add_argument("--procs", type=int, default=os.cpu_count())
    args = ap.parse_args()
    O.build()
    for name in args.only or list(ENTRIES):
        t0 = time.time()
        e = ENTRIES[name](args.procs)
        e["oracle_seconds"] = round(time.time() - t0, 1)
        data = load()
        data[name] = e
        data["_generator"] = "tests/golden/make_config_golden.py"
        with gzip.GzipFile(OUT, "wb", mtime=0) as f:
            f.write(json.dumps(data, sort_keys=True).encode())
        print(name, "done in", round(time.time() - t0, 1), "s", flush=True)


if __name__ == "__main__":
    main()
