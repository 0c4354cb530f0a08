// Batched rank: thousands of matrices of uneven sides and primes in one
// persistent launch (the CLI's `reps` loop, src/main.rs:82, with every job
// in flight at once).
//
// One CTA eliminates one matrix at a time, pulling jobs (largest first) from a
// device counter. The method is the reference's blocked elimination
// (src/fp.rs:125-255) with PANEL = 64:
//   A. in-panel elimination: per column, the first nonzero row at or below
//      the current rank is the pivot (src/fp.rs:151-156); the row order is a
//      logical permutation in shared memory instead of physical swaps
//      (src/fp.rs:158-162); each row below stores its multiplier in place of
//      the eliminated entry (src/fp.rs:169-170) and updates the rest of the
//      panel (src/fp.rs:171-173);
//   B. U block: forward substitution among the panel's pivot rows
//      (src/fp.rs:181-200), done per 64-column tile in shared memory;
//   C. trailing update: rows below the pivots -= multipliers x U
//      (src/fp.rs:202-248), 64x64 tiles, u128 accumulators reduced once per
//      safe_batch products.
// The rank is the number of pivots; every residue is exact, so the result is
// the reference's bit for bit.
#include <cuda_runtime.h>

#include <climits>

#include "field.cuh"
#include "rank_batch.cuh"

namespace modlin {

namespace {

constexpr int kT = kRankBatchThreads;  // 256
constexpr int kNW = kT / 32;
constexpr int kP = 64;  // panel width
constexpr int kG = 8;   // rows per warp in flight during the in-panel elimination

// Lazy accumulation of products of residues: u128 sums reduced once per
// safe_batch products in general; for p < 2^32 a product fits in 32 x 32 ->
// 64 bits, so the sums stay in a u64 and are reduced once per
// floor((2^64 - 1) / (p - 1)^2) products (at least 1; p < 2^31 gives >= 4).
// A reduced sum (< p) counts as one product.
template <class F>
struct Acc {
  using T = u128;
  __device__ static T prod(const F& f, uint64_t a, uint64_t b) { return f.prod(a, b); }
  __device__ static uint64_t reduce(const F& f, T x) { return f.reduce(x); }
  __device__ static uint64_t batch(const F& f) { return f.safe_batch(); }
};
template <>
struct Acc<FpSmall> {
  using T = uint64_t;
  __device__ static T prod(const FpSmall&, uint64_t a, uint64_t b) { return (uint64_t)(uint32_t)a * (uint32_t)b; }
  __device__ static uint64_t reduce(const FpSmall& f, T x) { return f.reduce64(x); }
  __device__ static uint64_t batch(const FpSmall& f) {
    const uint64_t q = f.modulus() - 1;
    return q <= 1 ? UINT64_MAX : UINT64_MAX / (q * q);
  }
};

struct BatchSmem {
  uint64_t LF[kP][kP + 1];  // multipliers of a row tile, or the pivot rows' multipliers F[k][k2]
  uint64_t Us[kP][kP];      // U block of one 64-column tile
  uint64_t prow[kP];        // pivot row's panel segment
  int pcol[kP];
  int red[kNW];
  uint64_t inv;
  int found;
  long long job;
};

template <class F>
__device__ __noinline__ int rank_one(const F& f, uint64_t* __restrict__ m, const int n, int* perm, BatchSmem& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  using A = Acc<F>;
  using AT = typename A::T;
  const uint64_t p = f.modulus();
  const uint64_t sb = A::batch(f);
  for (int i = tid; i < n; i += kT) perm[i] = i;
  __syncthreads();
  int r0 = 0;
  for (int c0 = 0; c0 < n && r0 < n; c0 += kP) {
    const int W = min(kP, n - c0);
    int pb = 0;
    // ---- A. in-panel elimination ------------------------------------------
    for (int kk = 0; kk < W && r0 + pb < n; ++kk) {
      const int c = c0 + kk, r = r0 + pb;
      int best = INT_MAX;
      for (int i = r + tid; i < n; i += kT)
        if (m[(int64_t)perm[i] * n + c] != 0) {
          best = i;
          break;
        }
      best = __reduce_min_sync(0xffffffffu, best);
      if (lane == 0) S.red[warp] = best;
      __syncthreads();
      if (tid == 0) {
        int b = INT_MAX;
        for (int w = 0; w < kNW; ++w) b = min(b, S.red[w]);
        S.found = b != INT_MAX;
        if (b != INT_MAX) {
          const int t = perm[r];
          perm[r] = perm[b];
          perm[b] = t;
          S.pcol[pb] = c;
          S.inv = fp_inv_binary(m[(int64_t)perm[r] * n + c], p);
        }
      }
      __syncthreads();
      if (!S.found) continue;
      const uint64_t* P = m + (int64_t)perm[r] * n + c0;
      if (tid < W) S.prow[tid] = P[tid];
      __syncthreads();
      // Rows below, kG per warp at a time: lane l holds panel entries l and
      // l + 32 of each of its rows (coalesced loads, all issued before any
      // is used), so each group costs one memory round trip.
      const uint64_t inv = S.inv;
      const uint64_t pv0 = lane > kk && lane < W ? S.prow[lane] : 0;
      const uint64_t pv1 = lane + 32 > kk && lane + 32 < W ? S.prow[lane + 32] : 0;
      for (int base = r + 1 + warp; base < n; base += kNW * kG) {
        uint64_t* R[kG];
        uint64_t x0[kG], x1[kG];
#pragma unroll
        for (int g = 0; g < kG; ++g) {
          const int i = base + g * kNW;
          R[g] = i < n ? m + (int64_t)perm[i] * n + c0 : nullptr;
          x0[g] = R[g] && lane < W ? R[g][lane] : 0;
          x1[g] = R[g] && lane + 32 < W ? R[g][lane + 32] : 0;
        }
#pragma unroll
        for (int g = 0; g < kG; ++g) {
          const uint64_t e = __shfl_sync(0xffffffffu, kk < 32 ? x0[g] : x1[g], kk & 31);
          if (e == 0) continue;  // uniform across the warp
          const uint64_t fm = f.mul(e, inv);
          if (lane > kk && lane < W) R[g][lane] = f.sub(x0[g], f.mul(fm, pv0));
          if (lane + 32 > kk && lane + 32 < W) R[g][lane + 32] = f.sub(x1[g], f.mul(fm, pv1));
          if (lane == (kk & 31)) R[g][kk] = fm;
        }
      }
      __syncthreads();
      ++pb;
    }
    if (pb == 0) continue;
    const int jend = c0 + W;
    if (jend < n && r0 + pb < n) {
      // ---- B + C. per 64-column tile: U block, then the trailing rows ------
      const int tx = tid & 15, ty = tid >> 4;
      for (int ct = jend; ct < n; ct += kP) {
        // Pivot rows' multipliers F[k][k2] (k2 < k) and their tile of U.
        for (int idx = tid; idx < pb * pb; idx += kT) {
          const int k = idx / pb, k2 = idx - k * pb;
          S.LF[k][k2] = k2 < k ? m[(int64_t)perm[r0 + k] * n + S.pcol[k2]] : 0;
        }
        for (int idx = tid; idx < pb * kP; idx += kT) {
          const int k = idx >> 6, ci = idx & 63;
          const int cc = ct + ci;
          S.Us[k][ci] = cc < n ? m[(int64_t)perm[r0 + k] * n + cc] : 0;
        }
        __syncthreads();
        {
          // U_k -= sum_{k2<k} F[k][k2] U_k2, four threads per column.
          const int ci = tid >> 2, q = tid & 3;
          for (int k = 1; k < pb; ++k) {
            AT acc = 0;
            uint64_t tot = 0, cnt = 0;
            for (int k2 = q; k2 < k; k2 += 4) {
              acc += A::prod(f, S.LF[k][k2], S.Us[k2][ci]);
              if (++cnt >= sb) {
                tot = f.add(tot, A::reduce(f, acc));
                acc = 0;
                cnt = 0;
              }
            }
            uint64_t part = f.add(tot, A::reduce(f, acc));
            part = f.add(part, __shfl_xor_sync(0xffffffffu, part, 1));
            part = f.add(part, __shfl_xor_sync(0xffffffffu, part, 2));
            if (q == 0) S.Us[k][ci] = f.sub(S.Us[k][ci], part);
            __syncwarp();
          }
        }
        __syncthreads();
        for (int rt = r0 + pb; rt < n; rt += kP) {
          // Multipliers of the row tile: LF[k][ri] = m[row][pcol[k]].
          for (int idx = tid; idx < pb * kP; idx += kT) {
            const int ri = idx / pb, k = idx - ri * pb;
            const int rr = rt + ri;
            S.LF[k][ri] = rr < n ? m[(int64_t)perm[rr] * n + S.pcol[k]] : 0;
          }
          __syncthreads();
          // A reduced accumulator (< p <= (p-1)^2 + 1) counts as one product,
          // so sb terms never overflow the u128.
          // The tile's C entries are loaded before the products so that
          // their latency overlaps the arithmetic.
          uint64_t cv[4][4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int rr = rt + ty + 16 * i;
            const uint64_t* R = rr < n ? m + (int64_t)perm[rr] * n : nullptr;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int cc = ct + tx + 16 * q;
              cv[i][q] = R && cc < n ? R[cc] : 0;
            }
          }
          AT acc[4][4];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][q] = 0;
          uint64_t cnt = 0;
          for (int k = 0; k < pb; ++k) {
            uint64_t a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = S.LF[k][ty + 16 * i];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = S.Us[k][tx + 16 * q];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int q = 0; q < 4; ++q) acc[i][q] += A::prod(f, a[i], b[q]);
            if (++cnt >= sb) {
#pragma unroll
              for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[i][q] = A::reduce(f, acc[i][q]);
              cnt = 1;
            }
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int rr = rt + ty + 16 * i;
            if (rr >= n) continue;
            uint64_t* R = m + (int64_t)perm[rr] * n;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int cc = ct + tx + 16 * q;
              if (cc < n) R[cc] = f.sub(cv[i][q], A::reduce(f, acc[i][q]));
            }
          }
          __syncthreads();
        }
      }
    }
    r0 += pb;
  }
  return r0;
}

__global__ void __launch_bounds__(kT, 2)
    rank_batch_kernel(const RankJob* __restrict__ jobs, int64_t count, unsigned long long* next, int64_t* out) {
  extern __shared__ __align__(16) unsigned char rb_smem[];
  BatchSmem& S = *reinterpret_cast<BatchSmem*>(rb_smem);
  int* perm = reinterpret_cast<int*>(rb_smem + sizeof(BatchSmem));
  for (;;) {
    if (threadIdx.x == 0) S.job = (long long)atomicAdd(next, 1ULL);
    __syncthreads();
    const long long q = S.job;
    __syncthreads();
    if (q >= count) break;
    const RankJob J = jobs[q];
    const FieldParams fp{J.p, J.mu_lo, J.mu_hi, J.safe_batch};
    int r;
    if (J.p == kM61)
      r = rank_one(FpM61(fp), J.m, (int)J.n, perm, S);
    else if (J.p < (1ULL << 32))
      r = rank_one(FpSmall(fp), J.m, (int)J.n, perm, S);
    else
      r = rank_one(FpBarrett(fp), J.m, (int)J.n, perm, S);
    if (threadIdx.x == 0) out[J.slot] = r;
    __syncthreads();
  }
}

}  // namespace

size_t rank_batch_smem_bytes(int64_t max_n) { return sizeof(BatchSmem) + (size_t)max_n * sizeof(int); }

// The kernel's dynamic shared memory cap is set once to what the largest
// side needs, so launches of any batch (graph-captured ones included) need no
// attribute call.
static cudaError_t rank_batch_attr() {
  static cudaError_t e = [] {
    cudaError_t r = cudaFuncSetAttribute(rank_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rank_batch_smem_bytes(kRankBatchMaxN));
    return r;
  }();
  return e;
}

int rank_batch_blocks_per_sm(int64_t max_n) {
  const size_t smem = rank_batch_smem_bytes(max_n);
  if (rank_batch_attr() != cudaSuccess) return 0;
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rank_batch_kernel, kT, smem);
  return nb;
}

cudaError_t launch_rank_batch(const RankJob* d_jobs, int64_t count, unsigned long long* d_next, int64_t max_n,
                              int blocks, int64_t* d_out, cudaStream_t st) {
  const size_t smem = rank_batch_smem_bytes(max_n);
  cudaError_t e = rank_batch_attr();
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  rank_batch_kernel<<<blocks, kT, smem, st>>>(d_jobs, count, d_next, d_out);
  return cudaGetLastError();
}

}  // namespace modlin
