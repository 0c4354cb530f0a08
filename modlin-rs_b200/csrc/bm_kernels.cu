// Berlekamp-Massey over F_p on the GPU (src/fp.rs:257-308).
//
// The reference keeps c (connection polynomial), b (the polynomial before the
// last length change) and a scratch t, computes the discrepancy
// d = s[i] + sum_{j=1..l} c[j] s[i-j] and updates c[m..m+bl) -= (d/bb) b
// (src/fp.rs:272-306). The GPU kernels run the same steps fraction-free:
//     c <- bb * c - d * x^m * b,      b <- old c,  bb <- d   (length change)
// which keeps every c a nonzero scalar multiple of the reference's c, so every
// discrepancy is zero exactly when the reference's is and l, m, bl evolve
// identically — the linear complexity is bit-exact — while no modular inverse
// (a ~120-multiplication Fermat chain) sits on the sequential path.
//
// Kernels:
//  * bm_block_kernel   — one CTA per sequence; the dot product is a warp-
//                        shuffle tree reduction mod p, the update a strided
//                        axpy mod p. Plain form: one sequence per launch.
//  * bm_batch_kernel   — persistent CTAs pulling sequences (longest first)
//                        from a device queue: thousands of uneven sequences
//                        and primes in one launch.
//  * bm_grid_kernel    — one long sequence on a cooperative grid: every CTA
//                        owns a slice of c in shared memory; per step one
//                        bounded-spin grid all-reduce of the partial dots.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "bm_kernels.cuh"
#include "field.cuh"

namespace modlin {

// Per-thread partial dot sum_{j in my indices, j <= l} c[j] * s[i - j].
template <class F>
__device__ __forceinline__ uint64_t partial_dot(const F& f, const uint64_t* c, const uint64_t* __restrict__ s, int64_t i,
                                                int64_t jbeg, int64_t jend_incl, int stride) {
  const uint64_t sb = f.safe_batch();
  u128 acc = 0;
  uint64_t tot = 0, cnt = 0;
  for (int64_t j = jbeg; j <= jend_incl; j += stride) {
    acc += f.prod(c[j], s[i - j]);
    if (++cnt == sb) {
      tot = f.add(tot, f.reduce(acc));
      acc = 0;
      cnt = 0;
    }
  }
  return f.add(tot, f.reduce(acc));
}

template <class F>
__device__ __forceinline__ uint64_t warp_sum_mod(const F& f, uint64_t v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = f.add(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

// One sequence with the whole CTA. c, b, t: n-entry buffers (shared or global
// memory) owned by this CTA; ws: 2 x 32 partial slots in shared memory.
template <class F>
__device__ int64_t bm_block_run(const F& f, const uint64_t* __restrict__ s, int64_t n, uint64_t* c, uint64_t* b,
                                uint64_t* t, uint64_t (*ws)[32]) {
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = T >> 5;
  for (int64_t j = tid; j < n; j += T) {
    c[j] = j == 0;
    b[j] = j == 0;
  }
  __syncthreads();
  int64_t l = 0, m = 1, bl = 1;
  uint64_t bb = 1;
  for (int64_t i = 0; i < n; ++i) {
    uint64_t part = partial_dot(f, c, s, i, tid, l, T);
    part = warp_sum_mod(f, part);
    if (lane == 0) ws[i & 1][warp] = part;
    __syncthreads();
    uint64_t d = 0;
    for (int w = 0; w < nw; ++w) d = f.add(d, ws[i & 1][w]);
    if (d == 0) {
      ++m;
      continue;
    }
    const bool lenchg = 2 * l <= i;
    const uint64_t nd = f.modulus() - d;  // c <- bb c + (p - d) x^m b: one reduction per entry
    int64_t hi = l + 1 > m + bl ? l + 1 : m + bl;
    if (hi > n) hi = n;
    for (int64_t j = tid; j < hi; j += T) {
      const uint64_t old = c[j];
      const int64_t jb = j - m;
      const uint64_t bj = (jb >= 0 && jb < bl) ? b[jb] : 0;
      c[j] = f.reduce2(f.prod(bb, old) + f.prod(nd, bj));
      if (lenchg && j <= l) t[j] = old;
    }
    if (lenchg) {
      uint64_t* tmp = b;
      b = t;
      t = tmp;
      bl = l + 1;
      bb = d;
      l = i + 1 - l;
      m = 1;
    } else {
      ++m;
    }
    // No barrier here: every thread reads and writes only its own entries of
    // c (j = tid mod T), ws is double-buffered, and the b entries written at
    // a length change are first read after the next step's barrier, which
    // every thread reaches only after finishing this step.
  }
  return l;
}

template <class F>
__device__ __forceinline__ int64_t bm_block_dispatch(const BmJob& job, uint64_t* c, uint64_t* b, uint64_t* t,
                                                     uint64_t (*ws)[32]) {
  FieldParams fp{job.p, job.mu_lo, job.mu_hi, job.safe_batch};
  return bm_block_run(F(fp), job.s, job.n, c, b, t, ws);
}

// Plain form: one CTA runs one sequence. Buffers in dynamic shared memory
// when 3n words fit (smem_words >= 3n), else in the global workspace.
__global__ void __launch_bounds__(1024) bm_block_kernel(BmJob job, uint64_t* gws, int64_t smem_words, int64_t* out) {
  extern __shared__ __align__(16) uint64_t bm_smem[];
  __shared__ uint64_t ws[2][32];
  uint64_t* base = (3 * job.n <= smem_words) ? bm_smem : gws;
  uint64_t *c = base, *b = base + job.n, *t = base + 2 * job.n;
  const int64_t l = job.p == kM61              ? bm_block_dispatch<FpM61>(job, c, b, t, ws)
                    : job.p < (1ULL << 32) ? bm_block_dispatch<FpSmall>(job, c, b, t, ws)
                                           : bm_block_dispatch<FpBarrett>(job, c, b, t, ws);
  if (threadIdx.x == 0) *out = l;
}

// Batched form: persistent CTAs take jobs from a device counter; the host
// orders jobs longest first (LPT). Each CTA has smem_words of dynamic shared
// memory and a private global slice of gws_words for jobs that do not fit.
__global__ void bm_batch_kernel(const BmJob* __restrict__ jobs, int64_t count, unsigned long long* next,
                                uint64_t* gws, int64_t gws_words, int64_t smem_words, int64_t* out) {
  extern __shared__ __align__(16) uint64_t bm_smem[];
  __shared__ uint64_t ws[2][32];
  __shared__ long long sh_job;
  for (;;) {
    if (threadIdx.x == 0) sh_job = (long long)atomicAdd(next, 1ULL);
    __syncthreads();
    const long long q = sh_job;
    __syncthreads();
    if (q >= count) break;
    const BmJob job = jobs[q];
    uint64_t* base = (3 * job.n <= smem_words) ? bm_smem : gws + (int64_t)blockIdx.x * gws_words;
    uint64_t *c = base, *b = base + job.n, *t = base + 2 * job.n;
    const int64_t l = job.p == kM61              ? bm_block_dispatch<FpM61>(job, c, b, t, ws)
                      : job.p < (1ULL << 32) ? bm_block_dispatch<FpSmall>(job, c, b, t, ws)
                                             : bm_block_dispatch<FpBarrett>(job, c, b, t, ws);
    if (threadIdx.x == 0) out[job.slot] = l;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Cooperative grid kernel for one long sequence.
// ---------------------------------------------------------------------------
struct GridSync {
  unsigned long long lo[3], hi[3];
  unsigned int count;
  int err;
};

__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int* p) {
  return *(const volatile unsigned int*)p;
}

template <class F>
// skip_cta >= 0 is a failure-detection test: that CTA does not arrive at the
// barrier of step 0, so every CTA's bounded wait expires, the error word is
// set and the host reports MODLIN_ETIMEOUT.
__global__ void bm_grid_kernel(F f, const uint64_t* __restrict__ s, int64_t n, int64_t chunk, uint64_t* bbuf0,
                               uint64_t* bbuf1, GridSync* gs, long long spin_limit_cycles, int skip_cta,
                               int64_t* out) {
  extern __shared__ __align__(16) uint64_t cs[];  // my slice of c: [lo, lo + chunk)
  __shared__ uint64_t ws[2][32];
  __shared__ uint64_t sh_d;
  __shared__ int sh_err;
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = T >> 5;
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi_own = lo + chunk < n ? lo + chunk : n;
  const unsigned G = gridDim.x;
  for (int64_t j = lo + tid; j < hi_own; j += T) {
    cs[j - lo] = j == 0;
    bbuf0[j] = j == 0;
  }
  if (tid == 0) sh_err = 0;
  // All b initialisations must be visible grid-wide before step 0 reads them.
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    atomicAdd(&gs->count, 1u);
    const long long t0 = clock64();
    while (ld_volatile_u32(&gs->count) < G) {
      if (clock64() - t0 > spin_limit_cycles || *(volatile int*)&gs->err) {
        atomicExch(&gs->err, 1);
        sh_err = 1;
        break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  if (sh_err) return;

  uint64_t* bcur = bbuf0;
  uint64_t* bnext = bbuf1;
  int64_t l = 0, m = 1, bl = 1;
  uint64_t bb = 1;
  for (int64_t i = 0; i < n; ++i) {
    // Partial dot over my slice j in [lo, hi_own) with j <= l.
    const int64_t jl = l < hi_own - 1 ? l : hi_own - 1;
    uint64_t part = 0;
    if (lo <= jl) {
      const uint64_t sb = f.safe_batch();
      u128 acc = 0;
      uint64_t cnt = 0;
      for (int64_t j = lo + tid; j <= jl; j += T) {
        acc += (u128)cs[j - lo] * s[i - j];
        if (++cnt == sb) {
          part = f.add(part, f.reduce(acc));
          acc = 0;
          cnt = 0;
        }
      }
      part = f.add(part, f.reduce(acc));
    }
    part = warp_sum_mod(f, part);
    if (lane == 0) ws[i & 1][warp] = part;
    __syncthreads();
    if (tid == 0) {
      uint64_t bp = 0;
      for (int w = 0; w < nw; ++w) bp = f.add(bp, ws[i & 1][w]);
      const int slot = (int)(i % 3);
      atomicAdd(&gs->lo[slot], (unsigned long long)(bp & 0xffffffffULL));
      atomicAdd(&gs->hi[slot], (unsigned long long)(bp >> 32));
      __threadfence();
      if (i != 0 || (int)blockIdx.x != skip_cta) atomicAdd(&gs->count, 1u);
      const unsigned target = (unsigned)(i + 2) * G;
      const long long t0 = clock64();
      while (ld_volatile_u32(&gs->count) < target) {
        if (clock64() - t0 > spin_limit_cycles || *(volatile int*)&gs->err) {
          atomicExch(&gs->err, 1);
          sh_err = 1;
          break;
        }
      }
      __threadfence();
      const unsigned long long slo = *(volatile unsigned long long*)&gs->lo[slot];
      const unsigned long long shi = *(volatile unsigned long long*)&gs->hi[slot];
      sh_d = f.reduce(((u128)shi << 32) + slo);
      if (blockIdx.x == 0) {
        const int rs = (int)((i + 2) % 3);
        gs->lo[rs] = 0;
        gs->hi[rs] = 0;
      }
    }
    __syncthreads();
    if (sh_err) return;
    const uint64_t d = sh_d;
    if (d == 0) {
      ++m;
      continue;
    }
    const bool lenchg = 2 * l <= i;
    const uint64_t nd = f.modulus() - d;  // c <- bb c + (p - d) x^m b: one reduction per entry
    int64_t uhi = l + 1 > m + bl ? l + 1 : m + bl;
    if (uhi > n) uhi = n;
    const int64_t jhi = uhi < hi_own ? uhi : hi_own;
    for (int64_t j = lo + tid; j < jhi; j += T) {
      const uint64_t old = cs[j - lo];
      const int64_t jb = j - m;
      const uint64_t bj = (jb >= 0 && jb < bl) ? __ldcg(bcur + jb) : 0;
      cs[j - lo] = f.reduce2(f.prod(bb, old) + f.prod(nd, bj));
      if (lenchg && j <= l) __stcg(bnext + j, old);
    }
    if (lenchg) {
      uint64_t* tmp = bcur;
      bcur = bnext;
      bnext = tmp;
      bl = l + 1;
      bb = d;
      l = i + 1 - l;
      m = 1;
    } else {
      ++m;
    }
    // Own-slice writes are re-read by the same thread next step; the next
    // grid barrier orders the b writes for the other CTAs.
    __syncthreads();
  }
  if (blockIdx.x == 0 && tid == 0) *out = l;
}

// ---------------------------------------------------------------------------
// Cluster kernel for one long sequence: one thread-block cluster (up to 16
// CTAs of 512 threads on 16 SMs), each CTA owning a slice of c in shared
// memory. The per-step all-reduce of the partial discrepancies is one
// hardware cluster barrier: every CTA posts its partial in its own shared
// memory, and after the barrier every warp reads the cluster's partials
// through distributed shared memory. b lives in global memory (L2); its
// writes before a barrier are visible to the whole cluster after it.
// ---------------------------------------------------------------------------
constexpr int kClusterMax = 16;  // CTAs per cluster (non-portable size)
constexpr int kTileBatch = 8;    // tiles whose global loads are issued together
constexpr int kClusterThreads = 512;  // threads per CTA = indices per tile

template <class F>
__global__ void __launch_bounds__(kClusterThreads, 1) bm_cluster_kernel(F f, const uint64_t* __restrict__ s, int64_t n,
                                                             int64_t chunk, uint64_t* bbuf0, uint64_t* bbuf1,
                                                             int64_t* out) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  // c is dealt out in tiles of TH = 512 consecutive indices, tile t to CTA
  // t mod R (so the active prefix j <= l is spread over the whole cluster);
  // thread tid owns index j = TH t + tid of each of its tiles.
  constexpr int TH = kClusterThreads;
  extern __shared__ __align__(16) uint64_t cs[];  // my tiles, TH words each
  __shared__ uint64_t ws[TH / 32];
  __shared__ uint64_t part[2][kClusterMax];  // [step parity][CTA]: partials pushed by every CTA
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int R = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  // Indices fit in 32 bits here (n <= 409600).
  const int nn = (int)n;
  const int ntiles = (nn + TH - 1) / TH;
  const int my_tiles = ntiles > rank ? (ntiles - rank + R - 1) / R : 0;
  const int j0 = rank * TH + tid, jstride = R * TH;  // my index in tile k: j0 + k * jstride
  for (int k = 0; k < my_tiles; ++k) {
    const int j = j0 + k * jstride;
    cs[k * TH + tid] = j == 0;
    if (j < nn) bbuf0[j] = j == 0;
  }
  uint64_t* part_dst = lane < R ? cl.map_shared_rank(&part[0][rank], lane) : nullptr;
  cl.sync();
  uint64_t* bcur = bbuf0;
  uint64_t* bnext = bbuf1;
  int l = 0, m = 1, bl = 1;
  uint64_t bb = 1;
  for (int i = 0; i < nn; ++i) {
    // Partial discrepancy over my indices j <= l; the loads of a batch of
    // tiles are issued together so that one L2 latency covers them.
    uint64_t tot = 0;
    const int kend = (l / TH - rank + R) / R;  // tiles that may hold j <= l
    const int kn = kend < my_tiles ? kend : my_tiles;
    for (int k0 = 0; k0 < kn; k0 += kTileBatch) {
      uint64_t sv[kTileBatch], cv[kTileBatch];
#pragma unroll
      for (int q = 0; q < kTileBatch; ++q) {
        const int k = k0 + q;
        const int j = j0 + k * jstride;
        const bool on = k < kn && j <= l;
        sv[q] = on ? s[i - j] : 0;
        cv[q] = on ? cs[k * TH + tid] : 0;
      }
      // Two independent chains of kTileBatch / 2 <= 4 <= safe_batch
      // products each (p < 2^63), reduced at the end of the batch.
      u128 a0 = 0, a1 = 0;
#pragma unroll
      for (int q = 0; q < kTileBatch; q += 2) {
        a0 += f.prod(cv[q], sv[q]);
        a1 += f.prod(cv[q + 1], sv[q + 1]);
      }
      tot = f.add(tot, f.add(f.reduce(a0), f.reduce(a1)));
    }
    uint64_t v = warp_sum_mod(f, tot);
    if (lane == 0) ws[warp] = v;
    __syncthreads();
    if (warp == 0) {
      v = warp_sum_mod(f, lane < TH / 32 ? ws[lane] : 0);
      v = __shfl_sync(0xffffffffu, v, 0);
      // Push this CTA's partial into every CTA's shared memory.
      if (lane < R) part_dst[(i & 1) * kClusterMax] = v;
    }
    cl.sync();
    // Every warp sums the cluster's partials from its own shared memory
    // (exact, so every thread gets the same discrepancy).
    uint64_t dv = lane < R ? part[i & 1][lane] : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dv = f.add(dv, __shfl_xor_sync(0xffffffffu, dv, off));
    const uint64_t d = dv;
    if (d == 0) {
      ++m;
      continue;
    }
    const bool lenchg = 2 * l <= i;
    const uint64_t nd = f.modulus() - d;  // c <- bb c + (p - d) x^m b: one reduction per entry
    int uhi = l + 1 > m + bl ? l + 1 : m + bl;
    if (uhi > nn) uhi = nn;
    const int kuend = ((uhi - 1) / TH - rank + R) / R;  // tiles that may hold j < uhi
    const int ku = kuend < my_tiles ? kuend : my_tiles;
    for (int k0 = 0; k0 < ku; k0 += kTileBatch) {
      uint64_t bv[kTileBatch];
#pragma unroll
      for (int q = 0; q < kTileBatch; ++q) {
        const int k = k0 + q;
        const int j = j0 + k * jstride;
        const int jb = j - m;
        bv[q] = (k < ku && j < uhi && jb >= 0 && jb < bl) ? __ldcg(bcur + jb) : 0;
      }
#pragma unroll
      for (int q = 0; q < kTileBatch; ++q) {
        const int k = k0 + q;
        const int j = j0 + k * jstride;
        if (k < ku && j < uhi) {
          uint64_t* cp = cs + k * TH + tid;
          const uint64_t old = *cp;
          *cp = f.reduce2(f.prod(bb, old) + f.prod(nd, bv[q]));
          if (lenchg && j <= l) __stcg(bnext + j, old);
        }
      }
    }
    if (lenchg) {
      uint64_t* tmp = bcur;
      bcur = bnext;
      bnext = tmp;
      bl = l + 1;
      bb = d;
      l = i + 1 - l;
      m = 1;
    } else {
      ++m;
    }
  }
  if (rank == 0 && tid == 0) *out = l;
  cl.sync();  // no CTA leaves while others may still write into its shared memory
}

// ---------------------------------------------------------------------------
// Host launchers.
// ---------------------------------------------------------------------------
cudaError_t launch_bm_block(const BmJob& job, uint64_t* gws, int64_t smem_words, int threads, int64_t* d_out,
                            cudaStream_t st) {
  const size_t smem = (3 * job.n <= smem_words) ? (size_t)(3 * job.n) * 8 : 0;
  if (smem > 0)  // dynamic + static shared memory may pass 48 KiB even when smem alone does not
    cudaFuncSetAttribute(bm_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  bm_block_kernel<<<1, threads, smem, st>>>(job, gws, smem_words, d_out);
  return cudaGetLastError();
}

cudaError_t bm_block_prepare() {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, bm_block_kernel);
}

// The batch kernel's dynamic shared memory cap is set once to the largest
// size any batch asks for (200 KiB), so launches of any batch, graph-captured
// ones included, need no attribute call.
static cudaError_t bm_batch_attr() {
  static cudaError_t e =
      cudaFuncSetAttribute(bm_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e;
}

cudaError_t launch_bm_batch(const BmJob* d_jobs, int64_t count, unsigned long long* d_next, uint64_t* gws,
                            int64_t gws_words, int64_t smem_words, int blocks, int threads, int64_t* d_out,
                            cudaStream_t st) {
  const size_t smem = (size_t)smem_words * 8;
  cudaError_t e = bm_batch_attr();
  if (e != cudaSuccess) return e;
  bm_batch_kernel<<<blocks, threads, smem, st>>>(d_jobs, count, d_next, gws, gws_words, smem_words, d_out);
  return cudaGetLastError();
}

int bm_batch_max_blocks_per_sm(int threads, int64_t smem_words) {
  const size_t smem = (size_t)smem_words * 8;
  if (bm_batch_attr() != cudaSuccess) return 0;
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bm_batch_kernel, threads, smem);
  return nb;
}

template <class F>
static cudaError_t launch_grid_t(const F& f, const uint64_t* s, int64_t n, int ctas, int threads, uint64_t* b0,
                                 uint64_t* b1, void* gs, long long spin, int skip_cta, int64_t* d_out,
                                 cudaStream_t st, int* ctas_used) {
  const int64_t chunk = (n + ctas - 1) / ctas;
  const size_t smem = (size_t)chunk * 8;
  if (smem > 0)  // dynamic + static shared memory may pass 48 KiB even when smem alone does not
    cudaFuncSetAttribute(bm_grid_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bm_grid_kernel<F>, threads, smem);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (per_sm < 1 || ctas > per_sm * sms) return cudaErrorCooperativeLaunchTooLarge;
  *ctas_used = ctas;
  GridSync* g = (GridSync*)gs;
  F fc = f;
  const uint64_t* sp = s;
  int64_t nn = n, ch = chunk;
  void* args[] = {(void*)&fc, (void*)&sp, (void*)&nn,   (void*)&ch,       (void*)&b0,
                  (void*)&b1, (void*)&g,  (void*)&spin, (void*)&skip_cta, (void*)&d_out};
  return cudaLaunchCooperativeKernel((void*)bm_grid_kernel<F>, dim3(ctas), dim3(threads), args, smem, st);
}

cudaError_t launch_bm_grid(const FieldParams& fp, const uint64_t* s, int64_t n, int ctas, int threads, uint64_t* b0,
                           uint64_t* b1, void* gs, long long spin, int skip_cta, int64_t* d_out, cudaStream_t st,
                           int* ctas_used) {
  if (fp.p == kM61)
    return launch_grid_t(FpM61(fp), s, n, ctas, threads, b0, b1, gs, spin, skip_cta, d_out, st, ctas_used);
  return launch_grid_t(FpBarrett(fp), s, n, ctas, threads, b0, b1, gs, spin, skip_cta, d_out, st, ctas_used);
}

template <class F>
static cudaError_t launch_cluster_t(const F& f, const uint64_t* s, int64_t n, int R, uint64_t* b0, uint64_t* b1,
                                   int64_t* d_out, cudaStream_t st) {
  const int64_t ntiles = (n + kClusterThreads - 1) / kClusterThreads;
  const int64_t chunk = (ntiles + R - 1) / R * kClusterThreads;  // words of c per CTA
  const size_t smem = (size_t)chunk * 8;
  cudaError_t e = cudaFuncSetAttribute(bm_cluster_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (R > 8) {
    e = cudaFuncSetAttribute(bm_cluster_kernel<F>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(R);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = R;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  e = cudaOccupancyMaxActiveClusters(&nclusters, bm_cluster_kernel<F>, &cfg);
  if (e != cudaSuccess) return e;
  if (nclusters < 1) return cudaErrorInvalidConfiguration;
  return cudaLaunchKernelEx(&cfg, bm_cluster_kernel<F>, f, s, n, chunk, b0, b1, d_out);
}

int bm_cluster_size(int64_t n) {
  return ((n + kClusterThreads - 1) / kClusterThreads + 15) / 16 * kClusterThreads * 8 <= kBmClusterSliceBytes ? 16 : 0;
}

template <class F>
static cudaError_t launch_cluster_any(const F& f, const uint64_t* s, int64_t n, int R, uint64_t* b0, uint64_t* b1,
                                     int64_t* d_out, cudaStream_t st) {
  cudaError_t e = launch_cluster_t(f, s, n, R, b0, b1, d_out, st);
  // A device without 16-CTA clusters: 8 CTAs when the slices still fit.
  if (e != cudaSuccess && R > 8 &&
      ((n + kClusterThreads - 1) / kClusterThreads + 7) / 8 * kClusterThreads * 8 <= kBmClusterSliceBytes) {
    cudaGetLastError();
    e = launch_cluster_t(f, s, n, 8, b0, b1, d_out, st);
  }
  return e;
}

cudaError_t launch_bm_cluster(const FieldParams& fp, const uint64_t* s, int64_t n, int R, uint64_t* b0, uint64_t* b1,
                              int64_t* d_out, cudaStream_t st) {
  if (fp.p == kM61) return launch_cluster_any(FpM61(fp), s, n, R, b0, b1, d_out, st);
  if (fp.p < (1ULL << 32)) return launch_cluster_any(FpSmall(fp), s, n, R, b0, b1, d_out, st);
  return launch_cluster_any(FpBarrett(fp), s, n, R, b0, b1, d_out, st);
}

size_t grid_sync_bytes() { return sizeof(GridSync); }

int grid_sync_err_offset() { return (int)offsetof(GridSync, err); }

}  // namespace modlin
