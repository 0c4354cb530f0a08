"""Benchmark: modular rank of a 16384 x 16384 matrix over p = 2^61 - 1.

Workload (the single large rank configuration): uniform residues in [0, p)
from SplitMix64(seed 7) with rejection sampling, row-major, generated on the
device; rank by blocked Gaussian elimination with the tensor-core (INT8-limb
tcgen05) trailing update when built, else the u64 Barrett one. One step = one
full rank of the matrix (a pristine device copy is restored into the work
buffer at the start of every step; the 2 GiB input is larger than L2).

metric value = algorithmic modular multiply-adds per second
    W = sum_k (n-1-k)(n-1-j_k) over the pivots (k-th pivot in column j_k),
i.e. the work of the reference's elimination (src/fp.rs:125-255), summed over
all ranks and divided by the max-over-ranks device time.

--impl reference times the reference algorithm's CPU restatement (the
oracle, OpenMP over all host threads) on a bounded sample of the same
workload; the reference itself is Rust and cannot be built here.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "modlin-rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

M61 = (1 << 61) - 1
N = 16384
METRIC = "Fp rank modmul/s (INT8-limb TC vs u64 Barrett); BM steps/s; bit-exact; 1 B200"
UNIT = "modMAC/s"


def algorithmic_work(n, pcols):
    return sum((n - 1 - k) * (n - 1 - j) for k, j in enumerate(pcols))


def trailing_work(n, pcols, panel=64):
    """modMACs of the trailing-update launches: per panel with pb pivots,
    (rows below the panel's pivots) x (columns right of the panel) x pb."""
    w, r0 = 0, 0
    pset = sorted(pcols)
    idx = 0
    for col in range(0, n, panel):
        jend = min(col + panel, n)
        pb = 0
        while idx < len(pset) and pset[idx] < jend:
            pb += 1
            idx += 1
        if pb and jend < n:
            w += (n - r0 - pb) * (n - jend) * pb
        r0 += pb
        if r0 >= n:
            break
    return w


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def golden_configs():
    """The CPU oracle's answers on these workloads at full size
    (tests/golden/configs.json.gz, written by tests/golden/make_config_golden.py);
    {} when the file is absent."""
    import gzip
    try:
        with gzip.open(os.path.join(ROOT, "tests", "golden", "configs.json.gz"), "rt") as f:
            return json.load(f)
    except Exception:
        return {}


def sha256_device(t, chunk=1 << 25):
    """SHA-256 of a device int64 tensor's little-endian bytes (host copies in chunks)."""
    import hashlib
    h = hashlib.sha256()
    flat = t.reshape(-1)
    for i in range(0, flat.numel(), chunk):
        h.update(flat[i:i + chunk].cpu().numpy().tobytes())
    return h.hexdigest()


def sha256_u64(values):
    import hashlib
    import numpy as np
    return hashlib.sha256(np.array(values, dtype=np.uint64).tobytes()).hexdigest()


def arena_digest(arena, ptrs, counts):
    """Checksum of checksums of a batch arena: SHA-256 of the concatenated
    per-job SHA-256 digests, jobs in order (the oracle's input checksum)."""
    import hashlib
    host = arena.cpu().numpy()
    base = ptrs[0]
    parts = [hashlib.sha256(host[(p - base) // 8:(p - base) // 8 + c].tobytes()).digest() for p, c in zip(ptrs, counts)]
    return hashlib.sha256(b"".join(parts)).hexdigest()


def int8_peak_tops(torch):
    """Dense INT8 tensor throughput on this GPU: cuBLASLt int8 GEMM via
    torch._int_mm (best of 5, 8192^3). None when unavailable."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda").t().contiguous().t()
        for _ in range(3):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            torch.cuda.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def int8_sustained_tops(torch, seconds=2.5):
    """INT8 tensor throughput under the power cap: cuBLASLt int8 GEMMs
    (8192^3, torch._int_mm) back to back for `seconds`, the last third timed
    with CUDA events. The peak for a kernel timed inside a long step (the
    burst figure above is for a kernel timed alone). None when unavailable."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda").t().contiguous().t()
        torch._int_mm(a, b)
        torch.cuda.synchronize()
        t0 = time.time()
        while time.time() - t0 < seconds * 2 / 3:
            for _ in range(8):
                torch._int_mm(a, b)
            torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 0
        s.record()
        t1 = time.time()
        while time.time() - t1 < seconds / 3:
            for _ in range(8):
                torch._int_mm(a, b)
            n += 8
            torch.cuda.synchronize()
        e.record()
        torch.cuda.synchronize()
        del a, b
        return 2 * 8192 ** 3 * n / (s.elapsed_time(e) * 1e-3) / 1e12
    except Exception:
        return None


def native_oracle():
    """The oracle built with -march=native for this host's CPU (the
    reference's release profile uses target-cpu=native), into a per-process
    file; the portable build when the native one cannot be built. Returns a
    label for the CPU-baseline description. Must run before the oracle's
    first use in this process."""
    import oracle
    if oracle._lib is not None:
        return "-O3" if oracle._SO.endswith("liboracle.so") else "-O3 -march=native"
    try:
        oracle.use_native(f"/tmp/modlin_oracle_native_{os.getpid()}.so")
        return "-O3 -march=native"
    except Exception:
        oracle.build()
        return "-O3 (native build failed)"


def cpu_rank_sample(threads=0, target_s=15.0):
    """The oracle's blocked rank (the reference algorithm, OpenMP over rows)
    on a uniform matrix over 2^61-1, sized from a 1024^2 probe so that the
    sample takes about target_s seconds of CPU time (10-30 s)."""
    import oracle
    n0 = 1024
    m = oracle.gen_uniform(M61, 7, n0 * n0)
    t0 = time.perf_counter()
    r, pc = oracle.rank(M61, m, n0, threads=threads, with_pcols=True)
    dt = time.perf_counter() - t0
    rate = algorithmic_work(n0, pc) / dt
    # W(n) ~ n^3 / 3: the side whose predicted time is target_s, in steps of 64.
    n = int((3 * rate * target_s) ** (1 / 3)) // 64 * 64
    n = max(n0, min(n, 8192))
    if n != n0:
        m = oracle.gen_uniform(M61, 7, n * n)
        t0 = time.perf_counter()
        r, pc = oracle.rank(M61, m, n, threads=threads, with_pcols=True)
        dt = time.perf_counter() - t0
    w = algorithmic_work(n, pc)
    return {"value": w / dt, "seconds": dt, "n": n, "rank": r, "work": w}


def splitmix64(seed):
    """SplitMix64 outputs (the workload generators' seeding convention)."""
    z = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        z = (z + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        w = z
        w = ((w ^ (w >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        w = ((w ^ (w >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield w ^ (w >> 31)


BM_PRIMES = [65521, (1 << 31) - 1, M61]


def bm_batch_jobs(count=65536, seed=31, nmin=256, nmax=8192):
    """The batched Berlekamp-Massey workload: `count` sequences, lengths
    uniform in [nmin, nmax], primes equally from BM_PRIMES, odd-indexed jobs
    planted order-L recurrences with L uniform in [16, n/4], even-indexed jobs
    iid uniform residues. Per job (prime index, n, L, seed) come from
    SplitMix64(seed); a planted job's stream is SplitMix64(its seed) through
    the planted generator, the iid jobs of one prime are consecutive slices of
    one uniform stream per prime."""
    g = splitmix64(seed)
    jobs = []
    for i in range(count):
        pi = next(g) % 3
        n = nmin + next(g) % (nmax - nmin + 1)
        planted = i % 2 == 1
        L = 16 + next(g) % (n // 4 - 16 + 1)
        jobs.append((pi, n, planted, L if planted else None, next(g)))
    iid_seeds = [next(g) for _ in range(3)]
    return jobs, iid_seeds


def bm_batch_build(torch, modlin, jobs, iid_seeds):
    """Device buffers of the batch: one arena, planted jobs by one launch of
    the planted generator, iid jobs by one uniform stream per prime."""
    total = sum(j[1] for j in jobs)
    arena = torch.empty(total, dtype=torch.int64, device="cuda")
    base = arena.data_ptr()
    ptrs, off = [], 0
    for j in jobs:
        ptrs.append(base + 8 * off)
        off += j[1]
    pl = [i for i, j in enumerate(jobs) if j[2]]
    modlin.gen.planted_batch_device([BM_PRIMES[jobs[i][0]] for i in pl], [jobs[i][3] for i in pl],
                                    [jobs[i][4] for i in pl], [ptrs[i] for i in pl], [jobs[i][1] for i in pl])
    for pi in range(3):
        ids = [i for i, j in enumerate(jobs) if not j[2] and j[0] == pi]
        cnt = sum(jobs[i][1] for i in ids)
        if not cnt:
            continue
        tmp = torch.empty(cnt, dtype=torch.int64, device="cuda")
        modlin.gen.uniform_device(BM_PRIMES[pi], iid_seeds[pi], tmp.data_ptr(), cnt)
        o = 0
        for i in ids:
            n = jobs[i][1]
            arena[(ptrs[i] - base) // 8:(ptrs[i] - base) // 8 + n].copy_(tmp[o:o + n])
            o += n
        del tmp
    torch.cuda.synchronize()
    return arena, ptrs


def bm_measure(torch, modlin, steps=2, warmup=1, long_n=200000, long_L=65280, batch_count=65536,
               plain_sample=512, cpu=True):
    """Berlekamp-Massey throughput (steps = sequence elements processed):
    the two long sequences on the cluster and grid kernels, the batch in one
    persistent launch, the plain one-sequence-per-launch form on a sample of
    the same batch and, with `cpu`, the oracle (the reference's single-
    threaded algorithm) on bounded samples of both."""
    from modlin import fp as mfp
    res = {}
    gold = golden_configs()
    for name, planted, seed in (("long_planted", True, 21), ("long_iid", False, 22)):
        t = torch.empty(long_n, dtype=torch.int64, device="cuda")
        if planted:
            modlin.gen.planted_device(M61, long_L, seed, t.data_ptr(), long_n)
        else:
            modlin.gen.uniform_device(M61, seed, t.data_ptr(), long_n)
        torch.cuda.synchronize()
        entry = {"n": long_n, "expected": long_L if planted else "about n/2"}
        g = gold.get(f"lc_{'planted' if planted else 'iid'}_{long_n}")
        if g:
            assert sha256_device(t) == g["input_sha256"], name
            entry["oracle"] = {"lc": g["lc"], "macs": g["dot_macs"] + g["axpy_macs"], "input_sha256_equal": True}
        # The default (one 16-CTA cluster) and the whole-grid kernel.
        for kern in ("cluster", "grid"):
            for _ in range(warmup):
                lc = mfp.linear_complexity_device(M61, t.data_ptr(), long_n, kernel=kern)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                lc = mfp.linear_complexity_device(M61, t.data_ptr(), long_n, kernel=kern)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            if planted:
                assert lc == long_L, (lc, long_L)
            if g:
                assert lc == g["lc"], (name, kern, lc, g["lc"])
            entry["lc"] = lc
            entry[kern] = {"ms": ms, "steps_per_s": long_n / (ms * 1e-3), "us_per_step": 1e3 * ms / long_n}
            if g:
                entry[kern]["mac_per_s"] = (g["dot_macs"] + g["axpy_macs"]) / (ms * 1e-3)
        entry["steps_per_s"] = entry["cluster"]["steps_per_s"]
        res[name] = entry
        del t
    jobs, iid_seeds = bm_batch_jobs(batch_count)
    arena, ptrs = bm_batch_build(torch, modlin, jobs, iid_seeds)
    ps = [BM_PRIMES[j[0]] for j in jobs]
    ns = [j[1] for j in jobs]
    total = sum(ns)
    for _ in range(warmup):
        lcs = mfp.lc_batch_device(ps, ptrs, ns)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        lcs = mfp.lc_batch_device(ps, ptrs, ns)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    bad = [i for i, j in enumerate(jobs) if j[2] and lcs[i] != j[3]]
    assert not bad, bad[:5]
    iid_dev = max(abs(lcs[i] - (j[1] + 1) // 2) for i, j in enumerate(jobs) if not j[2])
    batch = {"sequences": len(jobs), "total_steps": total, "ms": ms, "steps_per_s": total / (ms * 1e-3),
             "planted_exact": True, "iid_max_dev_from_half": iid_dev}
    g = gold.get(f"lc_batch_{len(jobs)}")
    cached = bool(g)
    if not g and len(jobs) <= 8192:  # no cached answers for this size: the live oracle
        import oracle
        host = arena.cpu().numpy().view("uint64")
        g = {"lcs": [], "macs": 0}
        for i in range(len(jobs)):
            o = (ptrs[i] - ptrs[0]) // 8
            lc_, d_, x_ = oracle.linear_complexity(ps[i], host[o:o + ns[i]], with_macs=True)
            g["lcs"].append(lc_)
            g["macs"] += d_ + x_
    elif g:
        assert arena_digest(arena, ptrs, ns) == g["input_sha256_of_job_sha256"]
    if g:
        wrong = [i for i in range(len(jobs)) if lcs[i] != g["lcs"][i]]
        assert not wrong, wrong[:5]
        batch["oracle"] = {"all_lcs_equal": True, "sequences_compared": len(jobs),
                           "answers": "cached, input digest equal" if cached else "live oracle", "macs": g["macs"]}
        batch["mac_per_s"] = g["macs"] / (ms * 1e-3)
    # Plain form: one sequence per launch, each call waits for its result.
    idx = list(range(0, len(jobs), max(1, len(jobs) // plain_sample)))[:plain_sample]
    sub = sum(ns[i] for i in idx)
    mfp.linear_complexity_device(ps[idx[0]], ptrs[idx[0]], ns[idx[0]], kernel="block")
    torch.cuda.synchronize()
    e0.record()
    for i in idx:
        assert mfp.linear_complexity_device(ps[i], ptrs[i], ns[i], kernel="block") == lcs[i]
    e1.record()
    torch.cuda.synchronize()
    pms = e0.elapsed_time(e1)
    batch["plain_one_per_launch"] = {"sequences": len(idx), "steps": sub, "ms": pms,
                                     "steps_per_s": sub / (pms * 1e-3)}
    batch["speedup_vs_plain"] = batch["steps_per_s"] / batch["plain_one_per_launch"]["steps_per_s"]
    # The batch as a plan captured in a CUDA graph (one counter reset and one
    # persistent launch per replay).
    out = torch.empty(len(jobs), dtype=torch.int64, device="cuda")
    plan = mfp.BatchPlan("lc", ps, ptrs, ns, out.data_ptr())
    g = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(cs):
        with torch.cuda.graph(g, stream=cs):
            plan.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().wait_stream(cs)
    g.replay()
    torch.cuda.synchronize()
    assert out.cpu().tolist() == lcs
    e0.record()
    for _ in range(steps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    gms = e0.elapsed_time(e1) / steps
    batch["cuda_graph"] = {"ms": gms, "steps_per_s": total / (gms * 1e-3)}
    del g
    plan.free()
    if cpu:
        # The reference runs BM single-threaded, one sequence after another.
        import oracle
        oracle.build()
        sample = idx[:48]
        base = ptrs[0]
        host = arena.cpu().numpy().view("uint64")
        t0 = time.perf_counter()
        for i in sample:
            o = (ptrs[i] - base) // 8
            assert oracle.linear_complexity(ps[i], host[o:o + ns[i]]) == lcs[i]
        dt = time.perf_counter() - t0
        steps_cpu = sum(ns[i] for i in sample)
        batch["cpu_oracle_one_thread"] = {"sequences": len(sample), "steps": steps_cpu, "s": dt,
                                          "steps_per_s": steps_cpu / dt}
        # The whole n = 200000 iid sequence (about a minute on one core).
        t = modlin.gen.uniform(M61, 22, long_n)
        t0 = time.perf_counter()
        lc_cpu = oracle.linear_complexity(M61, t)
        dt = time.perf_counter() - t0
        assert lc_cpu == res["long_iid"]["lc"]
        res["long_iid"]["cpu_oracle_one_thread"] = {"n": long_n, "s": dt, "steps_per_s": long_n / dt,
                                                    "note": "the whole sequence, one thread (as the reference)"}
    res["batch"] = batch
    del arena
    return res


RANK_PRIMES = [127, 65521, (1 << 31) - 1, M61]


def rank_batch_jobs(count=4096, seed=11, nmin=64, nmax=1024):
    """The batched rank workload: `count` matrices, sides uniform in
    [nmin, nmax], primes equally from RANK_PRIMES; even-indexed jobs iid
    uniform residues, odd-indexed jobs rows = successive length-n windows of
    an order-L recurrence, L uniform in [n/4, n]. Per job (prime index, n, L,
    seed) come from SplitMix64(seed); iid jobs of one prime are consecutive
    slices of one uniform stream per prime."""
    g = splitmix64(seed)
    jobs = []
    for i in range(count):
        pi = next(g) % len(RANK_PRIMES)
        n = nmin + next(g) % (nmax - nmin + 1)
        planted = i % 2 == 1
        L = n // 4 + next(g) % (n - n // 4 + 1)
        jobs.append((pi, n, planted, L if planted else None, next(g)))
    iid_seeds = [next(g) for _ in RANK_PRIMES]
    return jobs, iid_seeds


def rank_batch_build(torch, modlin, jobs, iid_seeds):
    total = sum(j[1] * j[1] for j in jobs)
    arena = torch.empty(total, dtype=torch.int64, device="cuda")
    base = arena.data_ptr()
    ptrs, offs, off = [], [], 0
    for j in jobs:
        ptrs.append(base + 8 * off)
        offs.append(off)
        off += j[1] * j[1]
    pl = [i for i, j in enumerate(jobs) if j[2]]
    modlin.gen.planted_batch_device([RANK_PRIMES[jobs[i][0]] for i in pl], [jobs[i][3] for i in pl],
                                    [jobs[i][4] for i in pl], [ptrs[i] for i in pl], [jobs[i][1] ** 2 for i in pl])
    for pi in range(len(RANK_PRIMES)):
        ids = [i for i, j in enumerate(jobs) if not j[2] and j[0] == pi]
        cnt = sum(jobs[i][1] ** 2 for i in ids)
        if not cnt:
            continue
        tmp = torch.empty(cnt, dtype=torch.int64, device="cuda")
        modlin.gen.uniform_device(RANK_PRIMES[pi], iid_seeds[pi], tmp.data_ptr(), cnt)
        o = 0
        for i in ids:
            nn = jobs[i][1] ** 2
            arena[offs[i]:offs[i] + nn].copy_(tmp[o:o + nn])
            o += nn
        del tmp
    torch.cuda.synchronize()
    return arena, ptrs


def rank_batch_measure(torch, modlin, steps=2, warmup=1, count=4096, single_sample=32):
    """Batched rank: every matrix in one persistent launch, inputs resident in
    HBM (a pristine arena restored into the work arena at each step). Work is
    the reference's modMAC count: sum over pivots of (n-1-k)(n-1-j_k), with
    pivot columns 0..r-1 (iid: full rank; planted: the first L columns span,
    the others are recurrence combinations)."""
    from modlin import fp as mfp
    jobs, iid_seeds = rank_batch_jobs(count)
    pristine, pptrs = rank_batch_build(torch, modlin, jobs, iid_seeds)
    work = torch.empty_like(pristine)
    off = work.data_ptr() - pristine.data_ptr()
    ptrs = [x + off for x in pptrs]
    ps = [RANK_PRIMES[j[0]] for j in jobs]
    ns = [j[1] for j in jobs]

    def step():
        work.copy_(pristine)
        return mfp.rank_batch_device(ps, ptrs, ns)

    for _ in range(warmup):
        ranks = step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ranks = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # Every rank against the oracle's (tests/golden/configs.json.gz, or the
    # live oracle for a batch size with no cached answers), whose column
    # profiles also give the batch's exact modMAC work.
    g = golden_configs().get(f"rank_batch_{len(jobs)}")
    cached = bool(g)
    if g:
        assert arena_digest(pristine, pptrs, [n * n for n in ns]) == g["input_sha256_of_job_sha256"]
    else:
        import oracle
        host = pristine.cpu().numpy().view("uint64")
        g = {"ranks": [], "work_modmac": 0}
        for i in range(len(jobs)):
            o = (pptrs[i] - pptrs[0]) // 8
            r_, pc = oracle.rank(ps[i], host[o:o + ns[i] * ns[i]], ns[i], with_pcols=True)
            g["ranks"].append(r_)
            g["work_modmac"] += algorithmic_work(ns[i], pc)
    wrong = [i for i in range(len(jobs)) if ranks[i] != g["ranks"][i]]
    assert not wrong, wrong[:5]
    work_mac = g["work_modmac"]
    want = [j[3] if j[2] else j[1] for j in jobs]
    res = {"matrices": len(jobs), "ms": ms, "matrices_per_s": len(jobs) / (ms * 1e-3), "work_modmac": work_mac,
           "modmac_per_s": work_mac / (ms * 1e-3),
           "oracle": {"all_ranks_equal": True, "matrices_compared": len(jobs),
                      "answers": "cached, input digest equal" if cached else "live oracle",
                      "non_generic_ranks": sum(1 for i in range(len(jobs)) if ranks[i] != want[i])},
           "step": "restore the 4096 matrices from a pristine copy + one batched call"}
    # The same batch as a plan captured in a CUDA graph: each replay restores
    # the matrices and ranks them all (one copy, one counter reset, one
    # persistent launch; no host synchronisation inside).
    out = torch.empty(len(jobs), dtype=torch.int64, device="cuda")
    plan = mfp.BatchPlan("rank", ps, ptrs, ns, out.data_ptr())
    g = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(cs):
        with torch.cuda.graph(g, stream=cs):
            work.copy_(pristine)
            plan.launch(torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().wait_stream(cs)
    g.replay()
    torch.cuda.synchronize()
    assert out.cpu().tolist() == ranks
    e0.record()
    for _ in range(steps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    gms = e0.elapsed_time(e1) / steps
    res["cuda_graph"] = {"ms": gms, "modmac_per_s": work_mac / (gms * 1e-3), "matrices_per_s": len(jobs) / (gms * 1e-3)}
    del g
    plan.free()
    # The same matrices through the single-matrix engine, one call each.
    idx = list(range(0, len(jobs), max(1, len(jobs) // single_sample)))[:single_sample]
    work.copy_(pristine)
    torch.cuda.synchronize()
    e0.record()
    for i in idx:
        assert mfp.rank_device(ps[i], ptrs[i], ns[i]) == ranks[i]
    e1.record()
    torch.cuda.synchronize()
    sms = e0.elapsed_time(e1)
    sw = sum(sum((ns[i] - 1 - k) ** 2 for k in range(ranks[i])) for i in idx)
    res["single_engine_one_per_call"] = {"matrices": len(idx), "ms": sms, "modmac_per_s": sw / (sms * 1e-3)}
    del work, pristine
    return res


def rank_planted_measure(torch, modlin, n=16384, L=4096, seed=8, steps=1):
    """The planted large rank: rows are successive length-n windows of an
    order-L recurrence from SplitMix64(seed), so the rank is L (pivot columns
    0..L-1) and everything after the first L columns is eliminated to zero.
    Both trailing kernels, one rank each per step, ranks and column profiles
    checked."""
    from modlin import fp as mfp
    pristine = torch.empty(n * n, dtype=torch.int64, device="cuda")
    t0 = time.perf_counter()
    modlin.gen.planted_device(M61, L, seed, pristine.data_ptr(), n * n)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    work = torch.empty_like(pristine)
    W = sum((n - 1 - k) ** 2 for k in range(L))
    res = {"n": n, "order": L, "work_modmac": W, "generation_s": gen_s}
    g = golden_configs().get(f"rank_planted_{n}")
    if g:
        assert sha256_device(pristine) == g["input_sha256"]
        assert g["rank"] == L and g["work_modmac"] == W
    for kern in ("tc", "plain"):
        work.copy_(pristine)
        r, pc = mfp.rank_device(M61, work.data_ptr(), n, kernel=kern, pivot_cols=True)
        assert r == L and list(pc) == list(range(L)), (kern, r)
        if g:
            assert sha256_u64(pc) == g["pcols_sha256"]
            res["oracle"] = {"rank": g["rank"], "pcols_equal": True, "input_sha256_equal": True}
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = 0.0
        for _ in range(steps):
            work.copy_(pristine)
            e0.record()
            assert mfp.rank_device(M61, work.data_ptr(), n, kernel=kern) == L
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        ms /= steps
        res[kern] = {"rank": r, "corank": n - r, "ms": ms, "modmac_per_s": W / (ms * 1e-3)}
    res["tc_speedup_vs_plain"] = res["tc"]["modmac_per_s"] / res["plain"]["modmac_per_s"]
    del work, pristine
    return res


def trailing_measure(torch, modlin, n=N, reps=3):
    """The trailing update alone, both kernels on the same shape: the first
    update of an n x n rank, C[(n-128) x (n-128)] -= L * U over 2^61-1
    (src/fp.rs:202-248), uniform residues. K = 64 (one panel: the plain
    kernel's depth) for both, and K = 128 (the two-panel depth the
    tensor-core rank uses) on the tensor cores, against two K = 64 plain
    updates. Each figure is the best of `reps` CUDA-event timings of
    modlin_trailing_update_device (the tensor-core time includes its limb
    splits). Also the plain kernel's roofline (modlin_plain_mac_peak: its
    inner loop with no global traffic) and the plain kernel's fraction of it."""
    from modlin import fp as mfp
    M = n - 128
    C = torch.empty(M * M, dtype=torch.int64, device="cuda")
    L128 = torch.empty(M * 128, dtype=torch.int64, device="cuda")
    U = torch.empty(128 * M, dtype=torch.int64, device="cuda")
    modlin.gen.uniform_device(M61, 71, C.data_ptr(), M * M)
    modlin.gen.uniform_device(M61, 72, L128.data_ptr(), M * 128)
    modlin.gen.uniform_device(M61, 73, U.data_ptr(), 128 * M)
    L64 = L128.view(M, 128)[:, :64].contiguous()
    torch.cuda.synchronize()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    def upd(L, K, kern):
        return lambda: mfp.trailing_update_device(M61, C.data_ptr(), M, M, M, L.data_ptr(), U.data_ptr(), M, K,
                                                  kernel=kern)
    res = {"shape": f"C {M}x{M} -= L {M}xK * U Kx{M} over 2^61-1", "ms": {}}
    res["ms"]["plain_k64"] = timed(upd(L64, 64, "plain"))
    res["ms"]["tc_k64"] = timed(upd(L64, 64, "tc"))
    res["ms"]["tc_k128"] = timed(upd(L128, 128, "tc"))
    macs64 = M * M * 64
    rate = {k: (macs64 * (2 if k.endswith("128") else 1)) / (v * 1e-3) for k, v in res["ms"].items()}
    res["modmac_per_s"] = rate
    res["plain_trailing_modmac_per_s"] = rate["plain_k64"]
    res["tc_trailing_modmac_per_s"] = rate["tc_k128"]
    res["tc_vs_plain_same_shape_k64"] = rate["tc_k64"] / rate["plain_k64"]
    res["tc_vs_plain"] = rate["tc_k128"] / rate["plain_k64"]
    peak = mfp.plain_mac_peak(M61)
    res["plain_mac_peak_modmac_per_s"] = peak
    res["int_pipe_frac"] = rate["plain_k64"] / peak
    res["roofline_plain"] = {"bound": "integer pipes", "achieved": rate["plain_k64"], "peak": peak,
                             "unit": "modMAC/s", "frac": rate["plain_k64"] / peak,
                             "peak_source": "measured: the plain kernel's inner loop alone (modlin_plain_mac_peak)"}
    del C, L128, L64, U
    torch.cuda.empty_cache()
    return res


def block_inverse_measure(torch, modlin, calls=4, seed=5):
    """The 64 x 64 block inverse of the rank's block steps
    (modlin_block_inverse_device) on a seeded uniform block over 2^61-1:
    `calls` calls timed with CUDA events, the result checked as P (-P^-1) = -I
    with exact integers."""
    from modlin import fp as mfp
    P = torch.empty(64 * 64, dtype=torch.int64, device="cuda")
    out = torch.empty(64 * 64, dtype=torch.int64, device="cuda")
    modlin.gen.uniform_device(M61, seed, P.data_ptr(), 64 * 64)
    assert mfp.block_inverse_device(M61, P.data_ptr(), 64, out.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(calls):
        mfp.block_inverse_device(M61, P.data_ptr(), 64, out.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    a = [[int(x) for x in row] for row in P.cpu().numpy().view("uint64").reshape(64, 64)]
    b = [[int(x) for x in row] for row in out.cpu().numpy().view("uint64").reshape(64, 64)]
    for i in range(64):
        for j in range(64):
            v = sum(a[i][k] * b[k][j] for k in range(64)) % M61
            assert v == ((M61 - 1) if i == j else 0), (i, j)
    return {"us_per_call": 1e3 * e0.elapsed_time(e1) / calls, "calls": calls, "check": "P (-P^-1) = -I exactly"}


def prng_fill_measure(torch, modlin, count=1 << 32, host_sample=1 << 23, readme_side=65536):
    """The generators' device fill (modlin_prng_fill_device) of the README's
    largest job, 2^32 outputs reduced mod 2^61-1 (a 65536^2 matrix), for
    MIXMAX-256 and xoroshiro128++, against the host stream's rate; then that
    whole job (generate + rank, modlin_rank_prng): MIXMAX-256 seed 1 has
    corank 65536 - 65280 = 256 (README.md:98-113)."""
    from modlin import fp as mfp
    out = torch.empty(count, dtype=torch.int64, device="cuda")
    peak = measured_peaks().get("hbm_gbs", 6650.0)
    res = {"outputs": count}
    for kind in ("mixmax256", "xoroshiro128pp"):
        g = modlin.prng.Prng(kind, 1)
        g.fill_device(out.data_ptr(), 1 << 20, M61)  # warm-up: jump matrices, workspace
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        g.fill_device(out.data_ptr(), count, M61)
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1)
        h = modlin.prng.Prng(kind, 1)
        h.fill(1 << 20)
        t0 = time.perf_counter()
        h.fill(host_sample)
        hs = time.perf_counter() - t0
        gbs = 8 * count / (ms * 1e-3) / 1e9
        res[kind] = {"ms": ms, "wall_ms": wall * 1e3, "outputs_per_s": count / (ms * 1e-3), "write_gbs": gbs,
                     "hbm_frac_of_measured": gbs / peak,
                     "host_outputs_per_s": host_sample / hs,
                     "speedup_vs_host_fill": (count / (ms * 1e-3)) / (host_sample / hs)}
    del out
    torch.cuda.empty_cache()
    g = modlin.prng.Prng("mixmax256", 1)
    t0 = time.perf_counter()
    r = mfp.rank_prng(M61, g, readme_side)
    job_s = time.perf_counter() - t0
    assert readme_side - r == 256, r
    res["readme_rank_job"] = {"side": readme_side, "generator": "MIXMAX-256 seed 1", "corank": readme_side - r,
                              "seconds": job_s,
                              "note": "README.md:110-113: 'a couple of hours' for the reference on a CPU"}
    torch.cuda.empty_cache()
    return res


def tc_update_schedule(n, two_panel_min):
    """Timed (wide) trailing updates of a full-rank n x n rank on the
    tensor-core block pipeline: steps of w = 128 columns (K = 128) while at
    least two_panel_min rows remain, then w = 64 (K = 64); each step's wide
    update covers the rows below its block and the columns after the next
    step's (the narrow update takes those). Returns (K = 128 updates, K = 64
    updates, total C outputs of the wide updates)."""
    def width(c):
        if n - c >= two_panel_min and n - c >= 128:
            return 128
        return 64 if n - c >= 64 else 0
    col, k128, k64, outs = 0, 0, 0, 0
    while col < n:
        w = width(col)
        if w == 0:
            break
        wn = width(col + w) if col + w < n else 0
        cw = col + w + wn
        if col + w < n and cw < n:
            if w == 128:
                k128 += 1
            else:
                k64 += 1
            outs += (n - col - w) * (n - cw)
        col += w
    return k128, k64, outs


def host_cores():
    try:
        import oracle
        import ctypes
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count()


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args, rank, world):
    if rank != 0:
        return
    flags = native_oracle()
    cores = host_cores()
    samples = []
    for i in range(args.warmup + args.steps):
        s = cpu_rank_sample(threads=0, target_s=12.0)
        if i >= args.warmup:
            samples.append(s)
    v = statistics.median([s["value"] for s in samples])
    n = samples[0]["n"]
    sample = (f"rank of one uniform {n}x{n} matrix over 2^61-1 per step (W={samples[0]['work']:.4g} modMAC), "
              f"oracle restatement of src/fp.rs:125-255 ({flags}) with OpenMP over {cores} threads on {cpu_model()}")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median([s["seconds"] for s in samples]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"rank {N}x{N} over 2^61-1, uniform SplitMix64(7) residues (bounded CPU sample)",
                   "n": N, "p": M61},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Rust (no rustc here); the oracle is its C restatement",
    }
    print(json.dumps(line), flush=True)


def run_sharded_rank(args, torch, dist, modlin, rank, world, local):
    """One n x n rank over 2^61-1 with its 64-column panels dealt
    block-cyclically over the `world` processes (modlin.shard.rank_sharded):
    strong scaling, total work fixed. Each step regenerates this process's
    columns of the SplitMix64(7) matrix from a device copy; the time is the
    max over ranks of CUDA-event time around the rank."""
    import numpy as np
    from modlin import shard
    n = args.n
    full = torch.empty(n * n, dtype=torch.int64, device="cuda")
    modlin.gen.uniform_device(M61, 7, full.data_ptr(), n * n)
    cols = torch.tensor(shard.local_columns(n, rank, world), device="cuda")
    pristine = full.view(n, n).index_select(1, cols).contiguous()
    del full
    torch.cuda.empty_cache()
    work = torch.empty_like(pristine)
    ops = shard.DeviceOps(M61)

    def step():
        work.copy_(pristine)
        return shard.rank_sharded(M61, work, n, ops=ops)

    for _ in range(args.warmup):
        r = step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    W = algorithmic_work(n, range(r))
    g = golden_configs().get(f"rank_uniform_{n}")
    if g:
        assert r == g["rank"], (r, g["rank"])
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": W / (ms_per_step * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u64 (INT8 limbs on the tensor cores)", "data": "synthetic",
            "config": {"workload": f"one rank {n}x{n} over p=2^61-1, uniform SplitMix64(7) residues, column panels "
                                   f"dealt over {world} GPU(s)", "n": n, "p": M61, "rank": r, "work_modmac": W,
                       "parallelism": f"column-sharded x{world}", "l2": "inputs larger than L2"},
            "parity": {"oracle_rank": g["rank"] if g else None}}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--kernel", default="auto", choices=["auto", "plain", "tc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default AUTO choices")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "sharded"],
                    help="N > 1 GPUs: independent replicas of the rank (weak scaling, default) or one rank "
                         "with its column panels dealt over the GPUs (strong scaling, modlin.shard.rank_sharded)")
    ap.add_argument("--tc-pairs", type=int, default=-1, choices=[-1, 0, 1],
                    help="tensor-core updates over 2^61-1 on CTA pairs (1) or single CTAs (0); -1: library default")
    ap.add_argument("--batch-count", type=int, default=0,
                    help="bm / rank-batch workloads: jobs in the batch (default: the full 65536 / 4096)")
    ap.add_argument("--workload", default="rank",
                    choices=["rank", "bm", "rank-batch", "rank-planted", "trailing", "block-inverse", "fill"],
                    help="rank: the 16384^2 rank (default line); bm / rank-batch: only those measurements")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    oracle_flags = native_oracle() if not args.no_cpu_baseline and rank == 0 else None

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import modlin
    from modlin import fp as mfp

    if args.tc_pairs >= 0:
        modlin.lib().modlin_set_tc_pairs(args.tc_pairs)
    # The AUTO choices measured on this GPU (a few seconds, before any timing).
    tune = (modlin.autotune()["choice"]
            if not args.no_autotune and args.workload not in ("trailing", "block-inverse", "fill") else None)

    if args.workload == "bm":
        res = bm_measure(torch, modlin, steps=args.steps, warmup=args.warmup,
                         batch_count=args.batch_count or 65536, cpu=not args.no_cpu_baseline)
        if rank == 0:
            print(json.dumps({"workload": "berlekamp-massey", **res}), flush=True)
        return
    if args.workload == "rank-planted":
        res = rank_planted_measure(torch, modlin, steps=args.steps)
        if rank == 0:
            print(json.dumps({"workload": "planted large rank", **res}), flush=True)
        return
    if args.workload == "block-inverse":
        res = block_inverse_measure(torch, modlin, calls=max(args.steps, 1))
        print(json.dumps({"workload": "block inverse 64x64 over 2^61-1", **res}), flush=True)
        return
    if args.workload == "fill":
        # MIXMAX-256 device fill of 2^26 outputs mod 2^61-1, `steps` times.
        g = modlin.prng.Prng("mixmax256", 1)
        t = torch.empty(1 << 26, dtype=torch.int64, device="cuda")
        times = []
        for _ in range(max(args.steps, 1)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            g.fill_device(t.data_ptr(), 1 << 26, M61)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        print(json.dumps({"workload": "MIXMAX-256 device fill, 2^26 outputs mod 2^61-1", "ms": times}), flush=True)
        return
    if args.workload == "trailing":
        res = trailing_measure(torch, modlin, n=args.n, reps=args.steps)
        if rank == 0:
            print(json.dumps({"workload": "trailing update", **res}), flush=True)
        return
    if args.workload == "rank-batch":
        res = rank_batch_measure(torch, modlin, steps=args.steps, warmup=args.warmup, count=args.batch_count or 4096)
        if rank == 0:
            print(json.dumps({"workload": "batched rank", **res}), flush=True)
        return

    if args.mode == "sharded":
        return run_sharded_rank(args, torch, dist, modlin, rank, world, local)

    n = args.n
    kernel = args.kernel
    if kernel == "auto":
        try:
            modlin.rank(M61, np.eye(130, dtype=np.uint64), 130, kernel="tc")
            kernel = "tc"
        except modlin.ModlinError:
            kernel = "plain"

    def barrier():
        if world > 1:
            dist.barrier()

    # Inputs resident in HBM: a pristine copy and a work buffer (2 x 2 GiB).
    pristine = torch.empty(n * n, dtype=torch.int64, device="cuda")
    work = torch.empty_like(pristine)
    modlin.gen.uniform_device(M61, 7 + rank, pristine.data_ptr(), n * n)
    torch.cuda.synchronize()

    def step(kern, want_pcols=False):
        work.copy_(pristine)
        return mfp.rank_device(M61, work.data_ptr(), n, kernel=kern, pivot_cols=want_pcols)

    r, pcols = step(kernel, True)
    W = algorithmic_work(n, pcols)
    # The oracle's answer for this matrix (computed once on the CPU, cached
    # with the input's SHA-256): same input, same rank, same pivot columns.
    parity = {"oracle": "no cached answer for this size"}
    g = golden_configs().get(f"rank_uniform_{n}")
    if g and rank == 0:
        assert sha256_device(pristine) == g["input_sha256"], "input differs from the oracle's"
        assert r == g["rank"], (r, g["rank"])
        assert sha256_u64(pcols) == g["pcols_sha256"]
        parity = {"oracle": "rank and pivot columns equal the CPU oracle's on the same input (SHA-256 checked)",
                  "oracle_rank": g["rank"], "oracle_work_modmac": g["work_modmac"]}
    Wtr = trailing_work(n, pcols)
    for _ in range(args.warmup):
        step(kernel)
    torch.cuda.synchronize()
    barrier()
    launches0 = modlin.kernel_launches()
    trailing_ms = []
    trailing_macs = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        ranks = []
        for _ in range(args.steps):
            ranks.append(step(kernel))
            trailing_ms.append(modlin.last_trailing_ms())
            trailing_macs.append(modlin.last_trailing_macs())
        ev1.record()
        torch.cuda.synchronize()
        barrier()
    launches = modlin.kernel_launches() - launches0
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = W * world / (ms_per_step * 1e-3)
    assert all(x == r for x in ranks)

    extras = {}
    if rank == 0 and not args.no_extras:
        # The other kernel at the same size (the TC speed-up claim).
        other = "plain" if kernel == "tc" else None
        if other:
            step(other)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step(other)
            e1.record()
            torch.cuda.synchronize()
            extras["plain_modmac_per_s"] = W / (e0.elapsed_time(e1) * 1e-3)
            extras["tc_speedup_vs_plain"] = value / world / extras["plain_modmac_per_s"]
        # The trailing update alone: both kernels on the same shape.
        extras["trailing_update"] = trailing_measure(torch, modlin)
        extras["plain_trailing_modmac_per_s"] = extras["trailing_update"]["plain_trailing_modmac_per_s"]
        extras["tc_trailing_modmac_per_s"] = extras["trailing_update"]["tc_trailing_modmac_per_s"]
        extras["tc_vs_plain_trailing"] = extras["trailing_update"]["tc_vs_plain"]
        # Berlekamp-Massey: the long sequences and the 65536-sequence batch.
        extras["berlekamp_massey"] = bm_measure(torch, modlin, steps=1, warmup=1, plain_sample=128,
                                                cpu=not args.no_cpu_baseline)
        # The planted large rank (order-4096 recurrence windows, rank 4096).
        extras["rank_planted"] = rank_planted_measure(torch, modlin)
        # Batched rank: 4096 matrices of sides 64..1024 in one launch.
        extras["rank_batch"] = rank_batch_measure(torch, modlin, steps=1, warmup=1, single_sample=16)
        # The generators' device fill and the README's largest rank job.
        extras["prng_fill"] = prng_fill_measure(torch, modlin)
        # Rooflines of the other workloads. Integer-pipe work against the
        # measured u64 multiply-accumulate peak (the plain trailing update's
        # inner loop alone, all SMs); tensor-core work against the int8 GEMM.
        peak_int = extras["trailing_update"]["plain_mac_peak_modmac_per_s"]
        int8 = int8_sustained_tops(torch) or int8_peak_tops(torch)
        int_src = "measured: u64 x u64 -> u128 multiply-accumulate loop on operands in shared memory, all SMs " \
                  "(modlin_plain_mac_peak)"
        bm = extras["berlekamp_massey"]
        if "mac_per_s" in bm["batch"]:
            a = bm["batch"]["mac_per_s"]
            bm["batch"]["roofline"] = {"bound": "latency: one block barrier per sequence step", "achieved": a,
                                       "peak": peak_int, "unit": "modMAC/s", "frac": a / peak_int,
                                       "peak_source": int_src}
        for key in ("long_planted", "long_iid"):
            e = bm[key]
            if "mac_per_s" in e.get("cluster", {}):
                a, pk = e["cluster"]["mac_per_s"], peak_int * 16 / 148
                e["roofline"] = {"bound": "latency: one 16-CTA cluster barrier per step", "achieved": a, "peak": pk,
                                 "unit": "modMAC/s", "frac": a / pk,
                                 "peak_source": int_src + ", scaled to the cluster's 16 SMs"}
        rb = extras["rank_batch"]
        rb["roofline"] = {"bound": "integer pipes (panel method per CTA)", "achieved": rb["modmac_per_s"],
                          "peak": peak_int, "unit": "modMAC/s", "frac": rb["modmac_per_s"] / peak_int,
                          "peak_source": int_src}
        rp = extras["rank_planted"]
        if int8:
            a = rp["tc"]["modmac_per_s"] * 128 / 1e12
            rp["roofline"] = {"bound": "tensor", "achieved": a, "peak": int8, "unit": "TFLOP/s", "frac": a / int8,
                              "peak_source": "measured, sustained: cuBLASLt int8 GEMM 8192^3 (torch._int_mm) back to "
                                             "back for 2.5 s on this GPU",
                              "note": "whole planted rank: all its modMACs x 64 limb products x 2 ops / rank time"}

    # End to end through the public C ABI with host buffers: pinned host
    # matrix -> modlin_rank (H2D copy + rank + D2H of the result) each step.
    host = torch.empty(n * n, dtype=torch.int64, pin_memory=True)
    host.copy_(pristine)
    hnp = host.numpy().view(np.uint64)
    import ctypes
    from modlin._lib import RankOpts, lib, szt, u64p
    opts = RankOpts(mfp.KERNELS[kernel], 0)
    out = szt(0)
    hp = hnp.ctypes.data_as(u64p)

    def e2e_step():
        rc = lib().modlin_rank_ex(M61, hp, n, ctypes.byref(opts), ctypes.byref(out), None,
                                  ctypes.cast(None, modlin._lib.PROGRESS), None)
        assert rc == 0 and out.value == r
    e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": W * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": 8,
           "ms_per_step": e2e_s * 1e3, "host_memory": "pinned"}
    # The same call on pageable host memory (a Rust Vec<u64> or a numpy array
    # is pageable): the driver stages the copy through its own pinned buffers.
    hpage = np.array(hnp, copy=True)
    hpp = hpage.ctypes.data_as(u64p)

    def e2e_page_step():
        rc = lib().modlin_rank_ex(M61, hpp, n, ctypes.byref(opts), ctypes.byref(out), None,
                                  ctypes.cast(None, modlin._lib.PROGRESS), None)
        assert rc == 0 and out.value == r
    e2e_page_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_page_step()
    e2e_p = (time.perf_counter() - t0) / args.steps
    if world > 1:
        t = torch.tensor([e2e_p], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_p = float(t.item())
    e2e_pageable = {"value": W * world / e2e_p, "unit": UNIT, "h2d_bytes_per_step": n * n * 8,
                    "d2h_bytes_per_step": 8, "ms_per_step": e2e_p * 1e3, "host_memory": "pageable"}
    del hpage

    if rank == 0:
        peaks = measured_peaks()
        tr_ms = statistics.median(trailing_ms)
        Wtr = statistics.median(trailing_macs)
        # Timed trailing updates per rank: one per block step on the
        # tensor-core path (K = 128 while at least the tuned two_panel_min
        # rows remain, the library default 256 without tuning; K = 64 after),
        # one per panel on the plain path.
        tpm = tune["two_panel_min"] if tune else 256
        k128, k64, outs = tc_update_schedule(n, tpm)
        n_tr = k128 + k64 if kernel == "tc" else sum(1 for _ in range(0, n, 64)) - 1
        per_launch_ms = tr_ms / max(n_tr, 1)
        if kernel == "tc":
            int8 = int8_peak_tops(torch)
            int8_s = int8_sustained_tops(torch)
            if int8_s:
                peak = int8_s
                peak_note = ("measured, sustained: cuBLASLt int8 GEMM 8192^3 (torch._int_mm) back to back for 2.5 s "
                             "on this GPU (the wide updates run inside a long step under the power cap); burst "
                             f"(best single GEMM): {int8:.0f} TOPS" if int8 else "")
            elif int8:
                peak, peak_note = int8, "measured: cuBLASLt int8 GEMM 8192^3 (torch._int_mm) on this GPU"
            else:
                peak = 2 * peaks.get("bf16_tflops", 1590.0)
                peak_note = "2 x measured bf16 dense (MEASURED_PEAKS.json); int8 GEMM unavailable"
            achieved = Wtr * 64 * 2 / (tr_ms * 1e-3) / 1e12
            # DRAM traffic per launch: ncu (dram__bytes_read + dram__bytes_write) of
            # the first wide K = 128 update of the 8192^2 rank was 550.0 + 454.4 MB
            # for 8064 x 7936 outputs (15.69 B per output against 16 algorithmic:
            # C read + write); scaled to this run's average launch by its outputs.
            outputs_per_launch = outs / max(n_tr, 1)
            traffic = 15.69 * outputs_per_launch
            roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "traffic_note": "bytes per launch: ncu DRAM bytes per output of an 8192^2 wide update "
                                    "x outputs per launch here (algorithmic: 16 B per output)",
                    "hbm_gbs_of_c": 16 * outputs_per_launch / (per_launch_ms * 1e-3) / 1e9,
                    "kernel": "trailing_tc (tcgen05 kind::i8)",
                    "peak_source": peak_note,
                    "algorithmic_per_launch": f"{Wtr / max(n_tr, 1):.4g} modMAC x 64 limb products x 2 ops "
                                              f"({k128} updates at K = 128, {k64} at K = 64 per rank)",
                    "avg_launch_ms": per_launch_ms,
                    "peak_burst": int8, "frac_of_burst": achieved / int8 if int8 else None}
        else:
            peak = peaks.get("hbm_gbs", 6650.0)
            # Algorithmic bytes of the plain trailing update: C read + write.
            bytes_tr = 0
            for k in range(n_tr):
                rows = n - 64 * (k + 1)
                bytes_tr += 16 * rows * rows
            achieved = bytes_tr / (tr_ms * 1e-3) / 1e9
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "kernel": "trailing_plain (u64 Barrett, integer pipes)",
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "avg_launch_ms": per_launch_ms,
                    "int_pipe_modmac_per_s": Wtr / (tr_ms * 1e-3)}
        cpu = None
        if not args.no_cpu_baseline:
            s = cpu_rank_sample(threads=0, target_s=15.0)
            cpu = {"value": s["value"], "unit": UNIT, "cores": host_cores(), "kind": "port",
                   "sample": f"oracle rank (src/fp.rs:125-255 restated, {oracle_flags}, OpenMP) of one uniform "
                             f"{s['n']}x{s['n']} matrix over 2^61-1, {s['seconds']:.1f} s, on {cpu_model()}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 (INT8 limbs on the tensor cores)" if kernel == "tc"
            else "u64", "data": "synthetic",
            "config": {"workload": f"single large rank {n}x{n} over p=2^61-1, uniform SplitMix64({7}+rank) "
                                   "residues, resident in HBM", "n": n, "p": M61, "kernel": kernel,
                       "parallelism": f"replicas{world}" if world > 1 else "1 GPU",
                       "l2": "inputs (2 GiB) larger than L2", "rank": r, "work_modmac": W,
                       "autotuned": tune},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_pageable": e2e_pageable,
            "gpu_launches": int(launches), "parity": parity,
            "clocks": clk.summary(), **extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
