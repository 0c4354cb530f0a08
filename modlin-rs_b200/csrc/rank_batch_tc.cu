// Batched rank with the trailing updates on the tensor cores: one CTA per
// matrix (persistent, largest first), the same panel method as
// rank_batch.cu (src/fp.rs:125-255): in-panel elimination with a logical row
// permutation, the U block solved per 64-column tile and written back over
// the pivot rows (they are finished after the panel), and the rank-pb update
// of the rows below as exact INT8-limb GEMMs on this SM's tensor cores:
//   * A operand: the 128 x 64 multiplier tile of 128 rows, split into LIMBS
//     u8 planes in shared memory (UMMA K-major, no swizzle);
//   * B operand: a 16·(8/LIMBS)-column subtile of U, its LIMBS planes stacked
//     along N (N = 128);
//   * tcgen05.mma kind::i8 per A plane writes TMEM columns [i·NS, i·NS+128),
//     so the 2·LIMBS-1 diagonal sums accumulate in TMEM; the epilogue folds
//     them to an exact residue and subtracts it from C.
// Every residue is exact, so the rank is the reference's bit for bit.
#include <cuda_runtime.h>

#include <climits>
#include <type_traits>

#include "field.cuh"
#include "rank_batch.cuh"
#include "tc_ptx.cuh"

namespace modlin {

namespace {

using namespace tc;

constexpr int kT = 256;  // threads per CTA (8 warps: 2 per TMEM lane quadrant)
constexpr int kNW = kT / 32;
constexpr int kP = 64;                   // panel width = K of the update
constexpr int kPlane = 128 * kP;         // one 128-row x 64-byte limb plane (8 KiB)
constexpr uint32_t kTmemCols = 256;      // one accumulator buffer per CTA (two CTAs per SM)
constexpr int kRegionBytes = 2 * kP * (kP + 1) * 8;  // Phase B (F and U tiles) / Phase C (A planes)

struct TcSmem {
  uint64_t prow[kP];
  int pcol[kP];
  int red[kNW];
  uint64_t inv;
  int found;
  long long job;
  uint64_t mbar;
  uint32_t tmem;
  int err;
};

// Byte offset of (n-row or m-row r, K byte k) in a UMMA K-major no-swizzle
// tile of 64-byte rows: 8-row x 16-byte core matrices, 4 along K.
__device__ __forceinline__ int core_off(int r, int k) { return ((r >> 3) * 4 + (k >> 4)) * 128 + (r & 7) * 16 + (k & 15); }

// Four consecutive K values of one row split into LIMBS planes (u32 per plane).
template <int LIMBS>
__device__ __forceinline__ void put_limbs(uint8_t* base, int plane_stride, int off, const uint64_t (&v)[4]) {
#pragma unroll
  for (int i = 0; i < LIMBS; ++i) {
    uint32_t x = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) x |= (uint32_t)((v[b] >> (8 * i)) & 0xFF) << (8 * b);
    *reinterpret_cast<uint32_t*>(base + i * plane_stride + off) = x;
  }
}

template <class F, int LIMBS>
__device__ int rank_one_tc(const F& f, uint64_t* __restrict__ m, const int n, int* perm, TcSmem& S, uint8_t* region,
                           uint8_t* sB, uint8_t* sZ, uint32_t& phase, const int* err) {
  constexpr int NS = 128 / LIMBS;      // output columns per subtile
  constexpr int DIAG = 2 * LIMBS - 1;  // diagonal accumulators
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t p = f.modulus();
  const uint64_t sb = f.safe_batch();
  const uint64_t r64 = (uint64_t)(((u128)1 << 64) % p);
  uint64_t(*Fs)[kP + 1] = reinterpret_cast<uint64_t(*)[kP + 1]>(region);
  uint64_t(*Us)[kP + 1] = reinterpret_cast<uint64_t(*)[kP + 1]>(region + kP * (kP + 1) * 8);
  for (int i = tid; i < n; i += kT) perm[i] = i;
  __syncthreads();
  int r0 = 0;
  for (int c0 = 0; c0 < n && r0 < n; c0 += kP) {
    const int W = min(kP, n - c0);
    int pb = 0;
    // ---- A. in-panel elimination (src/fp.rs:146-178) ----------------------
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
      const uint64_t inv = S.inv;
      for (int i = r + 1 + warp; i < n; i += kNW) {
        uint64_t* R = m + (int64_t)perm[i] * n;
        const uint64_t e = R[c];
        if (e == 0) continue;
        const uint64_t fm = f.mul(e, inv);
        for (int cc = c + 1 + lane; cc < c0 + W; cc += 32) R[cc] = f.sub(R[cc], f.mul(fm, S.prow[cc - c0]));
        __syncwarp();
        if (lane == 0) R[c] = fm;
      }
      __syncthreads();
      ++pb;
    }
    if (pb == 0) continue;
    const int jend = c0 + W;
    if (jend < n && r0 + pb < n) {
      // ---- B. U block (src/fp.rs:181-200), tile by tile, over the pivot rows
      for (int ct = jend; ct < n; ct += kP) {
        for (int idx = tid; idx < pb * pb; idx += kT) {
          const int k = idx / pb, k2 = idx - k * pb;
          Fs[k][k2] = k2 < k ? m[(int64_t)perm[r0 + k] * n + S.pcol[k2]] : 0;
        }
        for (int idx = tid; idx < pb * kP; idx += kT) {
          const int k = idx >> 6, ci = idx & 63;
          const int cc = ct + ci;
          Us[k][ci] = cc < n ? m[(int64_t)perm[r0 + k] * n + cc] : 0;
        }
        __syncthreads();
        {
          const int ci = tid >> 2, q = tid & 3;  // 4 threads per column, 64 columns
          for (int k = 1; k < pb; ++k) {
            u128 acc = 0;
            uint64_t tot = 0, cnt = 0;
            for (int k2 = q; k2 < k; k2 += 4) {
              acc += f.prod(Fs[k][k2], Us[k2][ci]);
              if (++cnt == sb) {
                tot = f.add(tot, f.reduce(acc));
                acc = 0;
                cnt = 0;
              }
            }
            uint64_t part = f.add(tot, f.reduce(acc));
            part = f.add(part, __shfl_xor_sync(0xffffffffu, part, 1));
            part = f.add(part, __shfl_xor_sync(0xffffffffu, part, 2));
            if (q == 0) Us[k][ci] = f.sub(Us[k][ci], part);
            __syncwarp();
          }
        }
        __syncthreads();
        // U replaces the pivot rows' trailing entries (finished rows).
        for (int idx = tid; idx < pb * kP; idx += kT) {
          const int k = idx >> 6, ci = idx & 63;
          const int cc = ct + ci;
          if (cc < n) m[(int64_t)perm[r0 + k] * n + cc] = Us[k][ci];
        }
        __syncthreads();
      }
      // ---- C. trailing rows -= multipliers x U on the tensor cores ----------
      uint8_t* sA = region;
      for (int rt = r0 + pb; rt < n; rt += 128) {
        // A planes: row i of the tile = logical row rt + i, K = the pivots.
        for (int u = tid; u < 128 * (kP / 4); u += kT) {
          const int i = u >> 4, k4 = (u & 15) * 4;
          const int rr = rt + i;
          uint64_t v[4];
#pragma unroll
          for (int b = 0; b < 4; ++b)
            v[b] = (rr < n && k4 + b < pb) ? m[(int64_t)perm[rr] * n + S.pcol[k4 + b]] : 0;
          put_limbs<LIMBS>(sA, kPlane, core_off(i, k4), v);
        }
        for (int cs = jend; cs < n; cs += NS) {
          // B planes: N-row j·NS + cc of plane j = U column cs + cc.
          for (int u = tid; u < NS * (kP / 4); u += kT) {
            const int cc = u >> 4, k4 = (u & 15) * 4;
            const int col = cs + cc;
            uint64_t v[4];
#pragma unroll
            for (int b = 0; b < 4; ++b)
              v[b] = (col < n && k4 + b < pb) ? m[(int64_t)perm[r0 + k4 + b] * n + col] : 0;
            put_limbs<LIMBS>(sB, NS * kP, core_off(cc, k4), v);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          fence_before();
          __syncthreads();
          fence_after();
          if (tid == 0) {
            const uint32_t id_full = idesc_i8(LIMBS * NS);
            if (LIMBS > 1)  // zero the upper diagonal blocks: (zero A) x B, no accumulate
              mma_i8(S.tmem + LIMBS * NS, smem_desc(sZ, 256), smem_desc(sB, 512), idesc_i8((LIMBS - 1) * NS), 0);
#pragma unroll
            for (int i = 0; i < LIMBS; ++i)
#pragma unroll
              for (int ks = 0; ks < kP / 32; ++ks)
                mma_i8(S.tmem + i * NS, smem_desc(sA + i * kPlane + ks * 256, 512), smem_desc(sB + ks * 256, 512),
                       id_full, (i > 0 || ks > 0) ? 1u : 0u);
            mma_commit(&S.mbar);
          }
          // One thread polls the MMA barrier; the CTA acts on its outcome.
          const bool ok = __syncthreads_and(tid == 0 ? mbar_poll(&S.mbar, phase & 1, err) : true);
          ++phase;
          if (!ok) {
            if (tid == 0) S.err = 1;
            return -1;
          }
          fence_after();
          // Epilogue: warp w reads TMEM lanes 32 (w % 4).. (tile rows) and the
          // column half w / 4 of the subtile, four columns at a time.
          const int quad = warp & 3, half = warp >> 2;
          const int row = quad * 32 + lane;
          const int rr = rt + row;
          const uint32_t lane_base = S.tmem + ((uint32_t)(quad * 32) << 16);
          uint64_t* crow = rr < n ? m + (int64_t)perm[rr] * n : nullptr;
          for (int c4 = half * (NS / 2); c4 < (half + 1) * (NS / 2); c4 += 4) {
            const int col = cs + c4;
            uint64_t res[4];
            if constexpr (std::is_same<F, FpM61>::value) {
              uint32_t a[15][4];
#pragma unroll
              for (int d = 0; d < 15; ++d) tmem_ld4(lane_base + d * NS + c4, a[d]);
              tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < 4; ++c) {
                // 2^(8(d+8)) = 8 * 2^(8d) mod 2^61-1: V_d = S_d + 8 S_(d+8).
                uint32_t V[8];
#pragma unroll
                for (int d = 0; d < 7; ++d) V[d] = a[d][c] + 8u * a[d + 8][c];
                V[7] = a[7][c];
                const uint64_t W0 = (uint64_t)V[3] * 16777216u +
                                    ((uint64_t)V[2] * 65536u + ((uint64_t)V[1] * 256u + (uint64_t)V[0]));
                const uint64_t W1 = (uint64_t)V[7] * 16777216u +
                                    ((uint64_t)V[6] * 65536u + ((uint64_t)V[5] * 256u + (uint64_t)V[4]));
                uint64_t x = W0 + ((uint64_t)((uint32_t)W1 & 0x1FFFFFFFu) << 32) + (W1 >> 29);
                x = (x & kM61) + (x >> 61);
                res[c] = x >= kM61 ? x - kM61 : x;
              }
            } else {
              u128 lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
#pragma unroll
              for (int d = 0; d < DIAG; ++d) {
                uint32_t a[4];
                tmem_ld4(lane_base + d * NS + c4, a);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                  if (d < 8)
                    lo[c] += (u128)a[c] << (8 * d);
                  else
                    hi[c] += (u128)a[c] << (8 * (d - 8));
                }
              }
#pragma unroll
              for (int c = 0; c < 4; ++c) res[c] = f.add(f.reduce(lo[c]), f.mul(f.reduce(hi[c]), r64));
            }
            if (crow) {
#pragma unroll
              for (int c = 0; c < 4; ++c)
                if (col + c < n) crow[col + c] = f.sub(crow[col + c], res[c]);
            }
          }
          fence_before();
          __syncthreads();  // TMEM drained and B planes free for the next subtile
          fence_after();
        }
      }
    }
    r0 += pb;
  }
  return r0;
}

__global__ void __launch_bounds__(kT, 2)
    rank_batch_tc_kernel(const RankJob* __restrict__ jobs, int64_t count, unsigned long long* next, int64_t* out,
                         int* err) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  uint8_t* region = tc_smem;                      // kRegionBytes
  uint8_t* sB = tc_smem + kRegionBytes;           // 8 KiB: B planes of one subtile
  uint8_t* sZ = sB + kPlane;                      // 4 KiB of zeros (128 x 32 B A tile)
  TcSmem& S = *reinterpret_cast<TcSmem*>(sZ + 4096);
  int* perm = reinterpret_cast<int*>(sZ + 4096 + ((sizeof(TcSmem) + 15) / 16) * 16);
  const int warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < 4096 / 16; i += kT) reinterpret_cast<uint4*>(sZ)[i] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    mbar_init(&S.mbar, 1);
    S.err = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  fence_before();
  __syncthreads();
  fence_after();
  uint32_t phase = 0;
  for (;;) {
    if (threadIdx.x == 0) S.job = (long long)atomicAdd(next, 1ULL);
    __syncthreads();
    const long long q = S.job;
    __syncthreads();
    if (q >= count || S.err) break;
    const RankJob J = jobs[q];
    const FieldParams fp{J.p, J.mu_lo, J.mu_hi, J.safe_batch};
    const int bits = 64 - __clzll((long long)(J.p - 1));
    int r;
    if (J.p == kM61)
      r = rank_one_tc<FpM61, 8>(FpM61(fp), J.m, (int)J.n, perm, S, region, sB, sZ, phase, err);
    else if (bits <= 8)
      r = rank_one_tc<FpSmall, 1>(FpSmall(fp), J.m, (int)J.n, perm, S, region, sB, sZ, phase, err);
    else if (bits <= 16)
      r = rank_one_tc<FpSmall, 2>(FpSmall(fp), J.m, (int)J.n, perm, S, region, sB, sZ, phase, err);
    else if (bits <= 32)
      r = rank_one_tc<FpSmall, 4>(FpSmall(fp), J.m, (int)J.n, perm, S, region, sB, sZ, phase, err);
    else
      r = rank_one_tc<FpBarrett, 8>(FpBarrett(fp), J.m, (int)J.n, perm, S, region, sB, sZ, phase, err);
    __syncthreads();
    if (S.err) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    if (threadIdx.x == 0) out[J.slot] = r;
  }
  // An abandoned wait may leave MMAs in flight: let them finish (bounded)
  // before TMEM is released.
  if (S.err && threadIdx.x == 0) mbar_poll(&S.mbar, (phase - 1) & 1, err + 1);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace

size_t rank_batch_tc_smem_bytes(int64_t max_n) {
  return (size_t)kRegionBytes + kPlane + 4096 + ((sizeof(TcSmem) + 15) / 16) * 16 + (size_t)max_n * sizeof(int);
}

static cudaError_t rank_batch_tc_attr() {
  static cudaError_t e = [] {
    cudaError_t r = cudaFuncSetAttribute(rank_batch_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rank_batch_tc_smem_bytes(kRankBatchMaxN));
    return r;
  }();
  return e;
}

int rank_batch_tc_blocks_per_sm(int64_t max_n) {
  if (rank_batch_tc_attr() != cudaSuccess) return 0;
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rank_batch_tc_kernel, kT, rank_batch_tc_smem_bytes(max_n));
  return nb < 2 ? nb : 2;  // two CTAs own all 512 TMEM columns
}

cudaError_t launch_rank_batch_tc(const RankJob* d_jobs, int64_t count, unsigned long long* d_next, int64_t max_n,
                                 int blocks, int64_t* d_out, int* d_err, cudaStream_t st) {
  cudaError_t e = rank_batch_tc_attr();
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  rank_batch_tc_kernel<<<blocks, kT, rank_batch_tc_smem_bytes(max_n), st>>>(d_jobs, count, d_next, d_out, d_err);
  return cudaGetLastError();
}

}  // namespace modlin
