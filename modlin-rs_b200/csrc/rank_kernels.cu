// Panel kernels and the plain trailing update of the blocked GPU rank.
// See rank_plain.cuh for the algorithm and its correspondence to the
// reference's src/fp.rs:125-255.
#include <cuda_runtime.h>

#include "launch.cuh"
#include "rank_plain.cuh"
#include "rank_kernels.cuh"
#include "tc_ptx.cuh"

namespace modlin {

// ---------------------------------------------------------------------------
// window_kernel — one CTA, kWindowThreads threads.
// Candidates: round 0 -> rows [r0, r0 + min(64, n - r0)); later rounds ->
// ps->cand[0 .. min(ps->ncand, 64)). Their panel columns [col, col + W) are
// eliminated in shared memory with first-nonzero pivoting in candidate order
// (src/fp.rs:150-157), fraction-free, while recording for each candidate
// alpha and its coefficients g against this round's new pivots, so that a
// pivot row k satisfies  U_k = alpha_k * row_k - sum_{k2<k} G[k][k2] * U_k2.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(kWindowThreads) window_kernel(F f, const uint64_t* __restrict__ m, int64_t ld,
                                                                 int32_t n, int32_t r0, int32_t col, int32_t W,
                                                                 int32_t round, PanelState* ps, uint64_t* Upanel,
                                                                 uint64_t* G, const uint64_t* Lbuf,
                                                                 uint8_t* is_pivot) {
  extern __shared__ __align__(16) uint64_t smem_w[];
  uint64_t(*A)[kPanel] = reinterpret_cast<uint64_t(*)[kPanel]>(smem_w);                  // [64][64]
  uint64_t(*Gc)[kPanel] = reinterpret_cast<uint64_t(*)[kPanel]>(smem_w + kWindow * kPanel);  // [64][64]
  __shared__ uint64_t alph[kWindow];
  __shared__ int32_t rowidx[kWindow], ispiv[kWindow], pivcand[kPanel], pivc[kPanel];
  __shared__ uint32_t ballots[2][2];
  __shared__ int32_t sh_nc, sh_pb_old;
  __shared__ uint64_t sh_mask;

  const int tid = threadIdx.x;
  if (tid == 0) {
    int nc = round == 0 ? min(kWindow, n - r0) : min(ps->ncand, kWindow);
    sh_nc = nc < 0 ? 0 : nc;
    sh_pb_old = ps->pb;
    sh_mask = ps->colmask;
  }
  __syncthreads();
  const int nc = sh_nc, pb_old = sh_pb_old;
  const uint64_t mask0 = sh_mask;
  if (tid < kWindow) {
    rowidx[tid] = tid < nc ? (round == 0 ? r0 + tid : ps->cand[tid]) : -1;
    ispiv[tid] = 0;
    alph[tid] = 1;
  }
  for (int idx = tid; idx < kWindow * kPanel; idx += blockDim.x) {
    (&Gc[0][0])[idx] = 0;
    (&A[0][0])[idx] = 0;
  }
  __syncthreads();
  for (int idx = tid; idx < nc * W; idx += blockDim.x) {
    const int i = idx / W, c = idx - (idx / W) * W;
    A[i][c] = m[(int64_t)rowidx[i] * ld + col + c];
  }
  __syncthreads();

  int npiv = 0, nb = 0;
  uint64_t newmask = 0;
  const int j = tid >> 3, sub = tid & 7;
  for (int c = 0; c < W; ++c) {
    if ((mask0 >> c) & 1ULL) continue;
    if (tid < kWindow) {
      const bool nz = tid < nc && !ispiv[tid] && A[tid][c] != 0;
      const uint32_t bal = __ballot_sync(0xffffffffu, nz);
      if ((tid & 31) == 0) ballots[nb & 1][tid >> 5] = bal;
    }
    __syncthreads();
    const uint32_t b0 = ballots[nb & 1][0], b1 = ballots[nb & 1][1];
    ++nb;
    const int piv = b0 ? __ffs(b0) - 1 : (b1 ? 31 + __ffs(b1) : -1);
    if (piv < 0) continue;
    const int t = npiv++;
    newmask |= 1ULL << c;
    const uint64_t e = A[piv][c];
    uint64_t h = 0;
    if (j < nc && j != piv && !ispiv[j]) h = A[j][c];
    __syncwarp();
    if (h != 0) {
      for (int cc = c + 1 + sub; cc < W; cc += 8) A[j][cc] = f.sub(f.mul(e, A[j][cc]), f.mul(h, A[piv][cc]));
      for (int t2 = sub; t2 < t; t2 += 8) Gc[j][t2] = f.mul(e, Gc[j][t2]);
      if (sub == 0) {
        alph[j] = f.mul(e, alph[j]);
        Gc[j][t] = h;
        A[j][c] = 0;
      }
    }
    if (tid == 0) {
      ispiv[piv] = 1;
      pivcand[t] = piv;
      pivc[t] = c;
    }
    __syncthreads();
  }
  __syncthreads();

  // Outputs: pivot bookkeeping, reduced pivot rows, transformation rows.
  for (int t = tid; t < npiv; t += blockDim.x) {
    const int k = pb_old + t, i = pivcand[t];
    ps->prow[k] = rowidx[i];
    ps->pcol[k] = col + pivc[t];
    ps->alpha[k] = alph[i];
    ps->inv[k] = fp_inv(f, A[i][pivc[t]]);
    is_pivot[rowidx[i]] = 1;
  }
  for (int idx = tid; idx < npiv * kPanel; idx += blockDim.x) {
    const int t = idx / kPanel, cc = idx % kPanel;
    Upanel[(int64_t)(pb_old + t) * kPanel + cc] = cc < W ? A[pivcand[t]][cc] : 0;
  }
  for (int idx = tid; idx < npiv * kPanel; idx += blockDim.x) {
    const int t = idx / kPanel, k2 = idx % kPanel, k = pb_old + t, i = pivcand[t];
    uint64_t v = 0;
    if (k2 < pb_old)
      v = f.mul(alph[i], Lbuf[(int64_t)(rowidx[i] - r0) * kPanel + k2]);
    else if (k2 < k)
      v = Gc[i][k2 - pb_old];
    G[(int64_t)k * kPanel + k2] = v;
  }
  if (tid == 0) {
    ps->pb = pb_old + npiv;
    ps->colmask = mask0 | newmask;
    ps->ncand = 0;
  }
}

// ---------------------------------------------------------------------------
// bulk_kernel — a warp per active non-pivot row: reference-style elimination
// of this round's new pivots pb_lo .. ps->pb from the row's panel part
// (f = e * inv, row -= f * U_k; src/fp.rs:163-175), multipliers to Lbuf,
// residual written back and, if nonzero, the row offered as a candidate.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(256) bulk_kernel(F f, uint64_t* __restrict__ m, int64_t ld, int32_t n, int32_t r0,
                                                    int32_t col, int32_t W, int32_t pb_lo, PanelState* ps,
                                                    const uint64_t* __restrict__ Upanel, uint64_t* Lbuf,
                                                    const uint8_t* __restrict__ is_pivot) {
  __shared__ uint64_t Us[kPanel][kPanel];
  __shared__ uint64_t invs[kPanel];
  __shared__ int32_t pcs[kPanel];
  const int pb_hi = ps->pb;
  const int nk = pb_hi - pb_lo;
  for (int idx = threadIdx.x; idx < nk * kPanel; idx += blockDim.x) {
    const int t = idx / kPanel, c = idx % kPanel;
    Us[t][c] = c < W ? Upanel[(int64_t)(pb_lo + t) * kPanel + c] : 0;
  }
  for (int t = threadIdx.x; t < nk; t += blockDim.x) {
    invs[t] = ps->inv[pb_lo + t];
    pcs[t] = ps->pcol[pb_lo + t] - col;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * (blockDim.x >> 5);
  for (int r = r0 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps_total) {
    if (is_pivot[r]) continue;
    uint64_t* row = m + (int64_t)r * ld + col;
    uint64_t x0 = lane < W ? row[lane] : 0;
    uint64_t x1 = lane + 32 < W ? row[lane + 32] : 0;
    for (int t = 0; t < nk; ++t) {
      const int pc = pcs[t];
      const uint64_t e = __shfl_sync(0xffffffffu, pc < 32 ? x0 : x1, pc & 31);
      const uint64_t fm = e ? f.mul(e, invs[t]) : 0;
      if (lane == 0) Lbuf[(int64_t)(r - r0) * kPanel + pb_lo + t] = fm;
      if (fm) {
        if (lane < W) x0 = f.sub(x0, f.mul(fm, Us[t][lane]));
        if (lane + 32 < W) x1 = f.sub(x1, f.mul(fm, Us[t][lane + 32]));
      }
    }
    if (nk > 0) {
      if (lane < W) row[lane] = x0;
      if (lane + 32 < W) row[lane + 32] = x1;
    }
    const bool nz = __any_sync(0xffffffffu, (x0 | x1) != 0);
    if (nz && lane == 0) {
      const int s = atomicAdd(&ps->ncand, 1);
      if (s < kWindow) ps->cand[s] = r;
    }
  }
}

// ---------------------------------------------------------------------------
// couple_kernel — U block (src/fp.rs:184-200): for every trailing column c,
// U_k[c] = alpha_k * row_{prow_k}[c] - sum_{k2<k} G[k][k2] * U_k2[c],
// sequential in k, a thread per column; the column's coupled values stay in
// registers (fully unrolled triangular loop), u128 lazy accumulation.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(128) couple_kernel(F f, const uint64_t* __restrict__ m, int64_t ld, int32_t n,
                                                      int32_t jend, const PanelState* __restrict__ ps,
                                                      const uint64_t* __restrict__ G, uint64_t* Ubuf, int64_t ldU) {
  extern __shared__ __align__(16) uint64_t smem_c[];
  uint64_t(*Us)[128] = reinterpret_cast<uint64_t(*)[128]>(smem_c);            // [64][128]: my column's U_k
  uint64_t(*Gs)[kPanel] = reinterpret_cast<uint64_t(*)[kPanel]>(smem_c + kPanel * 128);  // [64][64]
  __shared__ uint64_t al[kPanel];
  __shared__ int32_t prs[kPanel];
  const int pb = ps->pb;
  for (int idx = threadIdx.x; idx < pb * kPanel; idx += blockDim.x) Gs[idx / kPanel][idx % kPanel] = G[idx];
  for (int k = threadIdx.x; k < pb; k += blockDim.x) {
    al[k] = ps->alpha[k];
    prs[k] = ps->prow[k];
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int64_t c = (int64_t)jend + (int64_t)blockIdx.x * blockDim.x + t;
  const bool valid = c < n;
  const uint64_t sb = f.safe_batch();
  for (int k = 0; k < pb; ++k) {
    const uint64_t v = valid ? f.mul(al[k], m[(int64_t)prs[k] * ld + c]) : 0;
    u128 acc = 0;
    uint64_t tot = 0, cnt = 0;
#pragma unroll 8
    for (int k2 = 0; k2 < k; ++k2) {
      acc += (u128)Gs[k][k2] * Us[k2][t];
      if (++cnt == sb) {
        tot = f.add(tot, f.reduce(acc));
        acc = 0;
        cnt = 0;
      }
    }
    const uint64_t u = f.sub(v, f.add(tot, f.reduce(acc)));
    Us[k][t] = u;
    if (valid) Ubuf[(int64_t)k * ldU + c] = u;
  }
}

// ---------------------------------------------------------------------------
// move_rows_kernel — compaction of the active block: a non-pivot row that sits
// in [r0, r0 + pb) is copied (trailing part and multiplier row) into the slot
// of a pivot row that sits in [r0 + pb, n). blockIdx.y = move.
// ---------------------------------------------------------------------------
__global__ void move_rows_kernel(uint64_t* m, int64_t ld, int32_t n, int32_t jend, const int2* moves,
                                 uint64_t* Lbuf, int32_t r0, int32_t pb) {
  const int2 mv = moves[blockIdx.y];
  const int64_t src = mv.x, dst = mv.y;
  for (int64_t c = (int64_t)jend + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    m[dst * ld + c] = m[src * ld + c];
  if (blockIdx.x == 0)
    for (int k = threadIdx.x; k < pb; k += blockDim.x)
      Lbuf[(dst - r0) * kPanel + k] = Lbuf[(src - r0) * kPanel + k];
}

__global__ void clear_pivot_flags_kernel(const PanelState* ps, uint8_t* is_pivot) {
  const int k = threadIdx.x;
  if (k < ps->pb) is_pivot[ps->prow[k]] = 0;
}

// ---------------------------------------------------------------------------
// trailing_plain_kernel — A[rbeg.., jend..cend) -= L * U mod p on the integer
// pipes (src/fp.rs:208-248): 64x64 output tile per CTA, 4x4 per thread,
// u128 accumulators, one reduction per safe_batch products. The operands of
// the whole depth K are staged in shared memory by bulk copies
// (cp.async.bulk, completion counted on one mbarrier) that warp 0 issues:
// the tile's 64 rows of L (row stride 64, so one contiguous block) and K rows
// of 64 columns of U (one 512-byte copy each). U rows that are not 16-byte
// aligned or run past cend, and an unaligned L, are loaded by the threads.
// The mbarrier wait is bounded; on expiry the CTA records err[0] = 1, waits
// (bounded) for its own copies and returns without writing C.
// ---------------------------------------------------------------------------
constexpr int kPlainSmem = 2 * 64 * 64 * 8;  // L tile + U tile

template <class F>
__global__ void __launch_bounds__(256) trailing_plain_kernel(F f, uint64_t* __restrict__ m, int64_t ld, int32_t rbeg,
                                                              int32_t n, int32_t jend, int32_t cend,
                                                              const uint64_t* __restrict__ Lbuf, int32_t r0,
                                                              const uint64_t* __restrict__ Ubuf, int64_t ldU,
                                                              int32_t K, int* err) {
  extern __shared__ __align__(128) uint64_t smem_plain[];
  uint64_t* Ls = smem_plain;            // [64][64]: tile row ri, depth k
  uint64_t* Us = smem_plain + 64 * 64;  // [64][64]: depth k, tile column ci
  __shared__ __align__(8) uint64_t bar;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int64_t rt = (int64_t)rbeg + (int64_t)blockIdx.y * 64;
  const int64_t ct = (int64_t)jend + (int64_t)blockIdx.x * 64;
  const int rows = n - rt < 64 ? (int)(n - rt) : 64;
  const uint64_t* lsrc = Lbuf + (rt - r0) * kPanel;
  const bool bulk_l = ((uintptr_t)lsrc & 15) == 0;
  const bool bulk_u = ct + 64 <= cend && ((uintptr_t)(Ubuf + ct) & 15) == 0 && (ldU & 1) == 0;
  const uint32_t bytes = (bulk_l ? (uint32_t)rows * 512u : 0u) + (bulk_u ? (uint32_t)K * 512u : 0u);
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid < 32 && bytes) {
    if (tid == 0) tc::mbar_arrive_expect_tx(&bar, bytes);
    __syncwarp();
    if (bulk_l && tid == 0) tc::bulk_g2s(Ls, lsrc, (uint32_t)rows * 512u, &bar);
    if (bulk_u)
      for (int k = tid; k < K; k += 32) tc::bulk_g2s(Us + k * 64, Ubuf + (int64_t)k * ldU + ct, 512u, &bar);
  }
  if (!bulk_l)
    for (int idx = tid; idx < rows * 64; idx += 256) Ls[idx] = lsrc[(idx >> 6) * kPanel + (idx & 63)];
  if (!bulk_u)
    for (int idx = tid; idx < K * 64; idx += 256) {
      const int k = idx >> 6, ci = idx & 63;
      Us[idx] = ct + ci < cend ? Ubuf[(int64_t)k * ldU + ct + ci] : 0;
    }
  bool ok = true;
  if (bytes) ok = tc::mbar_wait(&bar, 0, err);
  if (!__syncthreads_and(ok)) {
    if (tid == 0) {
      atomicExch(err, 1);
      if (bytes) tc::mbar_wait(&bar, 0, err + 1);  // this CTA's copies land before it exits
    }
    return;
  }
  const uint64_t sb = f.safe_batch();
  uint64_t tot[4][4];
  u128 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      tot[i][q] = 0;
      acc[i][q] = 0;
    }
  uint64_t cnt = 0;
  for (int k = 0; k < K; ++k) {
    uint64_t a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = Ls[(ty + 16 * i) * 64 + k];
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = Us[k * 64 + tx + 16 * q];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][q] += (u128)a[i] * b[q];
    if (++cnt == sb) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          tot[i][q] = f.add(tot[i][q], f.reduce(acc[i][q]));
          acc[i][q] = 0;
        }
      cnt = 0;
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t r = rt + ty + 16 * i;
    if (r >= n) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t c = ct + tx + 16 * q;
      if (c < cend) {
        uint64_t* p = m + r * ld + c;
        *p = f.sub(*p, f.add(tot[i][q], f.reduce(acc[i][q])));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// plain_mac_peak_kernel — the roofline of trailing_plain_kernel: its inner
// loop (4x4 u128 accumulators per thread, operands read from shared memory,
// one reduction per safe_batch products) run `iters` times over a 64-deep
// tile that stays in shared memory, with no global traffic. The sums are
// written out so that nothing is optimised away.
// ---------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(256) plain_mac_peak_kernel(F f, int iters, uint64_t* out) {
  extern __shared__ __align__(128) uint64_t smem_peak[];
  uint64_t* Ls = smem_peak;
  uint64_t* Us = smem_peak + 64 * 64;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const uint64_t p = f.modulus();
  for (int idx = tid; idx < 64 * 64; idx += 256) {
    Ls[idx] = (0x9E3779B97F4A7C15ull * (uint64_t)(idx + 1 + blockIdx.x)) % p;
    Us[idx] = (0xBF58476D1CE4E5B9ull * (uint64_t)(idx + 7)) % p;
  }
  __syncthreads();
  const uint64_t sb = f.safe_batch();
  uint64_t tot[4][4];
  u128 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      tot[i][q] = 0;
      acc[i][q] = 0;
    }
  uint64_t cnt = 0;
  for (int it = 0; it < iters; ++it)
    for (int k = 0; k < 64; ++k) {
      uint64_t a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = Ls[(ty + 16 * i) * 64 + k];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = Us[k * 64 + tx + 16 * q];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] += (u128)a[i] * b[q];
      if (++cnt == sb) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            tot[i][q] = f.add(tot[i][q], f.reduce(acc[i][q]));
            acc[i][q] = 0;
          }
        cnt = 0;
      }
    }
  uint64_t s = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) s ^= f.add(tot[i][q], f.reduce(acc[i][q]));
  out[(int64_t)blockIdx.x * 256 + tid] = s;
}

template <class F>
cudaError_t launch_plain_mac_peak(const F& f, int blocks, int iters, uint64_t* out, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(plain_mac_peak_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kPlainSmem);
  if (e != cudaSuccess) return e;
  plain_mac_peak_kernel<F><<<blocks, 256, kPlainSmem, st>>>(f, iters, out);
  return cudaGetLastError();
}

template <class F>
int plain_blocks_per_sm() {
  cudaFuncSetAttribute(trailing_plain_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPlainSmem);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, trailing_plain_kernel<F>, 256, kPlainSmem);
  return nb;
}

// ---------------------------------------------------------------------------
// gj64_inverse — one CTA of 1024 threads (16 per block row): the inverse of
// the 64 x 64 block P = A[r0 .. r0+64, col .. col+64), or status = 1 when P
// is singular. In-place fraction-free Gauss-Jordan: at
// column c with pivot row `piv` (the first row not yet used whose entry is
// nonzero) every other row j becomes e * row_j - h * row_piv (e = P[piv][c],
// h = P[j][c]: one reduction of the two-product sum per entry), and column c,
// now zero outside the pivot, stores column `piv` of the accumulated row
// operations E instead (-h s and s in the pivot row, s = the scale row piv
// took while it was not a pivot). Row j's remaining left entry d_j is tracked
// apart. At the end P^-1 [pc_j][i] = E[j][i] / d_j with
// E[j][i] stored at column pc_i. One block barrier per column: the owner of
// column c+1 in each row flags a nonzero entry before it, and every warp then
// finds the pivot by itself with a ballot over the flags.
// Output: Vneg[c][i] = -(P^-1)[c][i] (row c = panel column, column i =
// block row), the B operand of the multiplier GEMM H = X_P * P^-1.
// ---------------------------------------------------------------------------
template <class F>
__device__ void gj64_inverse(const F& f, const uint64_t* __restrict__ m, int64_t ld, int32_t r0, int32_t col,
                             uint64_t* __restrict__ Vneg, int* status, const Guard& g, uint64_t* smem_inv) {
  uint64_t(*M)[kPanel + 1] = reinterpret_cast<uint64_t(*)[kPanel + 1]>(smem_inv);
  __shared__ uint64_t d[kPanel], dinv[kPanel], sc[kPanel];
  __shared__ int32_t pc[kPanel];
  __shared__ uint8_t nz[2][kPanel];  // nz[c & 1][j]: row j's entry in column c is nonzero
  const uint64_t p = f.modulus();
  const int tid = threadIdx.x, j = tid >> 4, s = tid & 15;
#pragma unroll
  for (int q = 0; q < 4; ++q) M[j][s + 16 * q] = m[(int64_t)(r0 + j) * ld + col + s + 16 * q];
  if (s == 0) {
    d[j] = 0;
    sc[j] = 1;
    nz[0][j] = M[j][0] != 0;  // written by this thread just above
  }
  __syncthreads();
  const int lane = tid & 31;
  unsigned long long used = 0;  // rows that are pivots already (same in every thread)
  int last_piv = -1;     // the previous column's pivot row: its column gets E's entry now
  uint64_t last_sc = 0;  // that entry: the pivot row's scale
  for (int c = 0; c < kPanel; ++c) {
    // Deferred from the previous column, after every thread has read the
    // pivot value there; only this thread reads this entry before the next
    // barrier.
    if (j == last_piv && s == ((c - 1) & 15)) M[j][c - 1] = last_sc;
    // Every warp finds the pivot itself: the first row not yet used with a
    // nonzero entry in column c (a ballot over the 64 rows' flags, set before
    // the barrier by the thread that owns column c of each row).
    const bool lo = !((used >> lane) & 1) && nz[c & 1][lane];
    const bool hi = !((used >> (lane + 32)) & 1) && nz[c & 1][lane + 32];
    const uint32_t b0 = __ballot_sync(0xffffffffu, lo), b1 = __ballot_sync(0xffffffffu, hi);
    if ((b0 | b1) == 0) {  // no pivot in column c: P is singular
      if (tid == 0) {
        if (status) *status = 1;
        if (g.bad) atomicMin(g.bad, g.step + 1);  // the chain of step g.step + 1 failed
      }
      return;
    }
    const int piv = b0 ? __ffs(b0) - 1 : 31 + __ffs(b1);
    const uint64_t e = M[piv][c];
    const uint64_t spiv = sc[piv];  // E[piv][piv]: the scale row piv took while unused
    const uint64_t h = j != piv ? M[j][c] : 0;
    __syncwarp();  // every read of M[j][c] precedes its overwrite below
    if (h != 0) {
      const uint64_t nh = p - h;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = s + 16 * q;
        M[j][k] = f.reduce2(f.prod(e, M[j][k]) + f.prod(nh, M[piv][k]));
      }
      if (s == (c & 15)) M[j][c] = f.mul(nh, spiv);  // column c now holds E's column piv
      if (s == 0) {
        if ((used >> j) & 1)
          d[j] = f.mul(e, d[j]);
        else
          sc[j] = f.mul(e, sc[j]);
      }
    }
    if (j == piv && s == 0) {
      d[j] = e;
      pc[j] = c;
    }
    const int cn = c + 1;
    if (cn < kPanel && s == (cn & 15)) nz[cn & 1][j] = M[j][cn] != 0;
    last_piv = piv;
    last_sc = spiv;
    used |= 1ULL << piv;
    __syncthreads();
  }
  if (j == last_piv && s == ((kPanel - 1) & 15)) M[j][kPanel - 1] = last_sc;
  if (tid < kPanel) dinv[tid] = fp_inv_binary(d[tid], p);
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = s + 16 * q;
    const uint64_t v = f.mul(M[j][pc[i]], dinv[j]);
    Vneg[(int64_t)pc[j] * kPanel + i] = v ? p - v : 0;
  }
}


// ---------------------------------------------------------------------------
// Recursive fraction-free inverse of the 64 x 64 block (the fast path of
// block_inverse_kernel). With P = [[A, B], [C, D]] in h x h blocks and
// A^-1 = N1 / d1 (numerator, scalar denominator):
//   S' = d1 D - (C N1) B  (= d1 S, S the Schur complement), S'^-1 = N2 / d2,
//   W' = (N1 B) N2, V = N2 (C N1),
//   P^-1 = [[d2 N1 + W' (C N1), -d1 W'], [-d1 V, d1^2 N2]] / (d1 d2).
// Blocks of 32 recurse the same way; blocks of 16 are fraction-free
// Gauss-Jordan on [X | I] with diagonal pivots (256 threads, two entries
// each, one named barrier per column), after which row j reads
// [D_j at column j | D_j X^-1 row j], and the per-row D_j are brought to
// their product. No modular inverse until the single one of the final
// denominator. The diagonal pivots and the leading 16- and 32-blocks and
// their Schur complements must be nonzero / invertible (for large p all
// fail with probability about 100/p); when one is not, the caller falls
// back to gj64_inverse (first-nonzero pivoting over all 64 rows), so the
// result never depends on that. Every product sum is exact (lazy u128 accumulation, one reduction
// per safe_batch products).
// ---------------------------------------------------------------------------
constexpr int kRecWords = 64 * 64 * 2 + 7 * 32 * 32 + 7 * 16 * 16 + 16 * 16;  // X, Out, scratch, base's I

struct RecShared {
  uint64_t pe[16];
  int fail;
};

__device__ __forceinline__ void bar_base() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

template <class F, int K>
__device__ __forceinline__ uint64_t rec_dot(const F& f, const uint64_t* A, const uint64_t* B, int ldb) {
  const uint64_t sb = f.safe_batch();
  u128 acc = 0;
  if (sb >= (uint64_t)K) {
#pragma unroll 16
    for (int k = 0; k < K; ++k) acc += f.prod(A[k], B[k * ldb]);
  } else {
    uint64_t cnt = 0;
    for (int k = 0; k < K; ++k) {
      acc += f.prod(A[k], B[k * ldb]);
      if (++cnt == sb) {
        acc = f.reduce(acc);
        cnt = 1;
      }
    }
  }
  return f.reduce(acc);
}

// The dot product of this thread's output with K split over SPLIT adjacent
// lanes (part = lane's share), summed across them by shuffles.
template <class F, int K, int SPLIT>
__device__ __forceinline__ uint64_t rec_dot_split(const F& f, const uint64_t* A, const uint64_t* B, int ldb, int part) {
  constexpr int KP = K / SPLIT;
  uint64_t v = rec_dot<F, KP>(f, A + part * KP, B + part * KP * ldb, ldb);
#pragma unroll
  for (int o = 1; o < SPLIT; o <<= 1) v = f.add(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// 16 x 16 block X (clobbered) -> Out = X^-1 * delta, delta = product of the
// rows' final diagonal entries. All threads call; threads 0..255 work.
template <class F>
__device__ void rec_base16(const F& f, uint64_t* X, int ldx, uint64_t* R, uint64_t* Out, int ldo, uint64_t* delta,
                           RecShared& S) {
  const uint64_t p = f.modulus();
  const int tid = threadIdx.x;
  if (tid < 256) {
    const int j = tid >> 4, k = tid & 15, lane = tid & 31;
    uint64_t x = X[j * ldx + k], y = j == k;
    R[j * 16 + k] = y;
    bar_base();
    bool ok = true;
#pragma unroll 1
    for (int c = 0; c < 16; ++c) {
      const uint64_t e = X[c * ldx + c], h = X[j * ldx + c];
      if (e == 0) {  // the same in every thread
        ok = false;
        break;
      }
      const uint64_t xp = X[c * ldx + k], yp = R[c * 16 + k];
      __syncwarp();  // row j's reads of X[j][c] precede its owner's write below
      if (j != c && h != 0) {
        const uint64_t nh = p - h;
        x = f.reduce2(f.prod(e, x) + f.prod(nh, xp));
        y = f.reduce2(f.prod(e, y) + f.prod(nh, yp));
        X[j * ldx + k] = x;
        R[j * 16 + k] = y;
      }
      bar_base();
    }
    if (!ok) {
      if (tid == 0) S.fail = 1;
    } else {
      if (tid < 32) {  // pe[j] = product of the other rows' diagonal entries
        const uint64_t xd = lane < 16 ? X[lane * ldx + lane] : 1;
        uint64_t pre = xd, suf = xd;
#pragma unroll
        for (int off = 1; off < 16; off <<= 1) {
          const uint64_t a = __shfl_up_sync(0xffffffffu, pre, off), b2 = __shfl_down_sync(0xffffffffu, suf, off);
          if (lane >= off) pre = f.mul(pre, a);
          if (lane + off < 16) suf = f.mul(suf, b2);
        }
        const uint64_t ex_pre = __shfl_up_sync(0xffffffffu, pre, 1), ex_suf = __shfl_down_sync(0xffffffffu, suf, 1);
        const uint64_t all = __shfl_sync(0xffffffffu, pre, 15);
        if (lane < 16) S.pe[lane] = f.mul(lane ? ex_pre : 1, lane < 15 ? ex_suf : 1);
        if (lane == 0) *delta = all;
      }
      bar_base();
      Out[j * ldo + k] = f.mul(y, S.pe[j]);
    }
  }
  __syncthreads();
}

// N x N block X (N = 32 or 64; its top-left h x h block is clobbered) ->
// Out = X^-1 * delta. Scratch: 7 h x h buffers at scr, then the next level's.
template <class F, int N>
__device__ void rec_inverse(const F& f, uint64_t* X, int ldx, uint64_t* Out, int ldo, uint64_t* delta, uint64_t* scr,
                            uint64_t* R, RecShared& S, uint64_t* dl) {
  constexpr int H = N / 2, HH = H * H;
  const uint64_t p = f.modulus();
  uint64_t *N1 = scr, *CN = scr + HH, *NB = scr + 2 * HH, *Sp = scr + 3 * HH, *N2 = scr + 4 * HH, *Wp = scr + 5 * HH,
           *V = scr + 6 * HH;
  uint64_t* A = X;
  const uint64_t *B = X + H, *C = X + H * ldx, *D = X + H * ldx + H;
  if constexpr (H == 16)
    rec_base16(f, A, ldx, R, N1, H, &dl[0], S);
  else
    rec_inverse<F, H>(f, A, ldx, N1, H, &dl[0], scr + 7 * HH, R, S, dl + 2);
  if (S.fail) return;
  // Small levels split each dot product over SP lanes (all threads busy).
  constexpr int SP = H == 16 ? 2 : 1;
  const uint64_t d1 = dl[0];
  for (int tt = threadIdx.x; tt < SP * 2 * HH; tt += blockDim.x) {  // CN = C N1, NB = N1 B
    const int t = tt / SP, part = tt % SP, u = t & (HH - 1), i = u / H, j = u % H;
    const uint64_t v = t < HH ? rec_dot_split<F, H, SP>(f, C + i * ldx, N1 + j, H, part)
                              : rec_dot_split<F, H, SP>(f, N1 + i * H, B + j, ldx, part);
    if (part == 0) (t < HH ? CN : NB)[u] = v;
  }
  __syncthreads();
  for (int tt = threadIdx.x; tt < SP * HH; tt += blockDim.x) {  // S' = d1 D - CN B
    const int t = tt / SP, part = tt % SP, i = t / H, j = t % H;
    const uint64_t v = rec_dot_split<F, H, SP>(f, CN + i * H, B + j, ldx, part);
    if (part == 0) Sp[t] = f.sub(f.mul(d1, D[i * ldx + j]), v);
  }
  __syncthreads();
  if constexpr (H == 16)
    rec_base16(f, Sp, H, R, N2, H, &dl[1], S);
  else
    rec_inverse<F, H>(f, Sp, H, N2, H, &dl[1], scr + 7 * HH, R, S, dl + 2);
  if (S.fail) return;
  const uint64_t d2 = dl[1];
  for (int tt = threadIdx.x; tt < SP * 2 * HH; tt += blockDim.x) {  // W' = NB N2, V = N2 CN
    const int t = tt / SP, part = tt % SP, u = t & (HH - 1), i = u / H, j = u % H;
    const uint64_t v = t < HH ? rec_dot_split<F, H, SP>(f, NB + i * H, N2 + j, H, part)
                              : rec_dot_split<F, H, SP>(f, N2 + i * H, CN + j, H, part);
    if (part == 0) (t < HH ? Wp : V)[u] = v;
  }
  __syncthreads();
  const uint64_t d11 = f.mul(d1, d1);
  for (int tt = threadIdx.x; tt < SP * HH; tt += blockDim.x) {  // top left: d2 N1 + W' CN
    const int t = tt / SP, part = tt % SP, i = t / H, j = t % H;
    const uint64_t v = rec_dot_split<F, H, SP>(f, Wp + i * H, CN + j, H, part);
    if (part == 0) Out[i * ldo + j] = f.add(f.mul(d2, N1[t]), v);
  }
  for (int t = threadIdx.x + HH; t < 4 * HH; t += blockDim.x) {  // [[., -d1 W'], [-d1 V, d1^2 N2]]
    const int q = t / HH, u = t & (HH - 1), i = u / H, j = u % H;
    uint64_t v;
    if (q == 3) {
      v = f.mul(d11, N2[u]);
    } else {
      v = f.mul(d1, q == 1 ? Wp[u] : V[u]);
      v = v ? p - v : 0;
    }
    Out[(i + (q >> 1) * H) * ldo + j + (q & 1) * H] = v;
  }
  if (threadIdx.x == 0) *delta = f.mul(d1, d2);
  __syncthreads();
}

// block_inverse_kernel: the recursive path when `rec` (large p, where it
// fails with probability about 100/p), else or on its failure the pivoting
// Gauss-Jordan. Output as gj64_inverse.
template <class F>
__global__ void __launch_bounds__(kInvThreads) block_inverse_kernel(F f, const uint64_t* __restrict__ m, int64_t ld,
                                                                     int32_t r0, int32_t col,
                                                                     uint64_t* __restrict__ Vneg, int* status, int rec,
                                                                     int reset_status, Guard g) {
  extern __shared__ __align__(16) uint64_t smem_inv[];
  pdl_wait();
  if (guard_skip(g)) return;  // an earlier step of the pipeline failed
  if (reset_status && status && threadIdx.x == 0) *status = 0;
  if (rec) {
    __shared__ RecShared S;
    __shared__ uint64_t dl[5];  // level 64: d1, d2; level 32: d1, d2; the result's denominator
    __shared__ uint64_t invd;
    uint64_t* X = smem_inv;
    uint64_t* Out = X + 64 * 64;
    uint64_t* scr = Out + 64 * 64;
    uint64_t* R = scr + 7 * 32 * 32 + 7 * 16 * 16;
    for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x)
      X[t] = m[(int64_t)(r0 + (t >> 6)) * ld + col + (t & 63)];
    if (threadIdx.x == 0) S.fail = 0;
    __syncthreads();
    rec_inverse<F, 64>(f, X, 64, Out, 64, &dl[4], scr, R, S, dl);
    if (!S.fail) {
      const uint64_t p = f.modulus();
      if (threadIdx.x == 0) invd = std::is_same<F, FpM61>::value ? fp_inv_m61(dl[4]) : fp_inv_binary(dl[4], p);
      __syncthreads();
      const uint64_t inv = invd;
      for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x) {
        const uint64_t v = f.mul(Out[t], inv);
        Vneg[t] = v ? p - v : 0;
      }
      return;
    }
    __syncthreads();
  }
  gj64_inverse(f, m, ld, r0, col, Vneg, status, g, smem_inv);
}

// ---------------------------------------------------------------------------
// small_gemm64_kernel — C = D - A * B (negate) or C = D + A * B on 64 x 64
// blocks mod p (D may be null: zero), or the copy C = D when A is null; up to
// kSgMaxProbs independent problems per launch, 16 CTAs of 256 threads each,
// one 16 x 16 output tile per CTA (one output per thread, one reduction per
// output), so the products spread over the SMs a finished trailing update
// leaves free.
// ---------------------------------------------------------------------------
constexpr int kSgTile = 16;
struct SgBatch {
  SgProb p[kSgMaxProbs];
  Guard g;
};
template <class F>
__global__ void __launch_bounds__(256) small_gemm64_kernel(F f, SgBatch batch) {
  __shared__ uint64_t As[kSgTile][2 * kPanel + 1], Bs[2 * kPanel][kSgTile + 1];
  pdl_wait();
  if (guard_skip(batch.g)) return;
  const SgProb& P = batch.p[blockIdx.x >> 4];
  const int tid = threadIdx.x, i = tid >> 4, j = tid & 15;
  const int ti = (blockIdx.x >> 2) & 3, tj = blockIdx.x & 3;
  const int r = ti * kSgTile + i, c = tj * kSgTile + j;
  if (!P.A) {  // copy
    P.C[(int64_t)r * P.ldc + c] = P.D[(int64_t)r * P.ldd + c];
    return;
  }
  const int K = P.k == 2 * kPanel ? 2 * kPanel : kPanel;
  for (int q = 0; q < K / 16; ++q) {
    const int kk = j + 16 * q;
    As[i][kk] = P.A[(int64_t)(ti * kSgTile + i) * P.lda + kk];
    Bs[i + 16 * q][j] = P.B[(int64_t)(i + 16 * q) * P.ldb + tj * kSgTile + j];
  }
  __syncthreads();
  const uint64_t p = f.modulus(), sb = f.safe_batch();
  u128 acc = 0;
  if (sb >= (uint64_t)K) {
#pragma unroll 16
    for (int k = 0; k < K; ++k) acc += f.prod(As[i][k], Bs[k][j]);
  } else {
    uint64_t cnt = 0;
    for (int k = 0; k < K; ++k) {
      acc += f.prod(As[i][k], Bs[k][j]);
      if (++cnt == sb) {
        acc = f.reduce(acc);  // counts as one product from here on
        cnt = 1;
      }
    }
  }
  uint64_t v = f.reduce(acc);
  if (P.negate && v) v = p - v;
  if (P.D) v = f.add(v, P.D[(int64_t)r * P.ldd + c]);
  P.C[(int64_t)r * P.ldc + c] = v;
}

__global__ void zero_kernel(uint64_t* __restrict__ p, int64_t n, Guard g) {
  pdl_wait();
  if (guard_skip(g)) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0;
}

// ---------------------------------------------------------------------------
// Launch wrappers (explicit instantiation for both field policies).
// ---------------------------------------------------------------------------
template <class F>
void launch_window(const F& f, const uint64_t* m, int64_t ld, int n, int r0, int col, int W, int round,
                   PanelState* ps, uint64_t* Upanel, uint64_t* G, const uint64_t* Lbuf, uint8_t* is_pivot,
                   cudaStream_t st) {
  const size_t smem = 2 * kWindow * kPanel * sizeof(uint64_t);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(window_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set = true;
  }
  window_kernel<F><<<1, kWindowThreads, smem, st>>>(f, m, ld, n, r0, col, W, round, ps, Upanel, G, Lbuf, is_pivot);
}

template <class F>
void launch_bulk(const F& f, uint64_t* m, int64_t ld, int n, int r0, int col, int W, int pb_lo, PanelState* ps,
                 const uint64_t* Upanel, uint64_t* Lbuf, const uint8_t* is_pivot, int num_sms, cudaStream_t st) {
  const int rows = n - r0;
  int blocks = (rows + 7) / 8;
  const int cap = num_sms * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  bulk_kernel<F><<<blocks, 256, 0, st>>>(f, m, ld, n, r0, col, W, pb_lo, ps, Upanel, Lbuf, is_pivot);
}

template <class F>
void launch_couple(const F& f, const uint64_t* m, int64_t ld, int n, int jend, const PanelState* ps,
                   const uint64_t* G, uint64_t* Ubuf, int64_t ldU, cudaStream_t st) {
  const int cols = n - jend;
  const size_t smem = (size_t)(kPanel * 128 + kPanel * kPanel) * sizeof(uint64_t);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(couple_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set = true;
  }
  couple_kernel<F><<<(cols + 127) / 128, 128, smem, st>>>(f, m, ld, n, jend, ps, G, Ubuf, ldU);
}

void launch_moves(uint64_t* m, int64_t ld, int n, int jend, const int2* moves, int nmoves, uint64_t* Lbuf, int r0,
                  int pb, cudaStream_t st) {
  if (nmoves <= 0) return;
  const int cols = n - jend;
  int bx = (cols + 255) / 256;
  if (bx > 64) bx = 64;
  if (bx < 1) bx = 1;
  move_rows_kernel<<<dim3(bx, nmoves), 256, 0, st>>>(m, ld, n, jend, moves, Lbuf, r0, pb);
}

void launch_clear_flags(const PanelState* ps, uint8_t* is_pivot, cudaStream_t st) {
  clear_pivot_flags_kernel<<<1, kPanel, 0, st>>>(ps, is_pivot);
}

template <class F>
void launch_trailing_plain(const F& f, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend,
                           const uint64_t* Lbuf, int r0, const uint64_t* Ubuf, int64_t ldU, int K, int* err,
                           cudaStream_t st) {
  if (rbeg >= rend || jend >= cend || K <= 0) return;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(trailing_plain_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPlainSmem);
    attr = true;
  }
  dim3 grid((cend - jend + 63) / 64, (rend - rbeg + 63) / 64);
  trailing_plain_kernel<F><<<grid, 256, kPlainSmem, st>>>(f, m, ld, rbeg, rend, jend, cend, Lbuf, r0, Ubuf, ldU, K,
                                                           err);
}

template <class F>
void launch_block_inverse(const F& f, const uint64_t* m, int64_t ld, int r0, int col, uint64_t* Vneg, int* status,
                          cudaStream_t st, bool reset_status, const Guard& g) {
  const size_t smem = kRecWords * sizeof(uint64_t);  // >= the pivoting path's kPanel * (kPanel + 1) words
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(block_inverse_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set = true;
  }
  const int rec = f.modulus() > (1ULL << 20);
  launch_k(block_inverse_kernel<F>, dim3(1), dim3(kInvThreads), smem, st, 1, f, m, ld, (int32_t)r0, (int32_t)col,
           Vneg, status, rec, reset_status ? 1 : 0, g);
}

template <class F>
void launch_small_gemm64_batch(const F& f, const SgProb* probs, int count, cudaStream_t st, const Guard& g) {
  SgBatch b = {};
  b.g = g;
  for (int i = 0; i < count && i < kSgMaxProbs; ++i) b.p[i] = probs[i];
  const int n = count < kSgMaxProbs ? count : kSgMaxProbs;
  launch_k(small_gemm64_kernel<F>, dim3(16 * n), dim3(256), 0, st, 1, f, b);
}

template <class F>
void launch_small_gemm64(const F& f, const uint64_t* A, int64_t lda, const uint64_t* B, int64_t ldb, const uint64_t* D,
                         int64_t ldd, uint64_t* C, int64_t ldc, bool negate, cudaStream_t st, const Guard& g) {
  const SgProb pr = {A, B, D, C, lda, ldb, ldd, ldc, negate ? 1 : 0, kPanel};
  launch_small_gemm64_batch<F>(f, &pr, 1, st, g);
}

void launch_zero(uint64_t* p, int64_t n, cudaStream_t st, const Guard& g) {
  if (n <= 0) return;
  int64_t blocks = (n + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  launch_k(zero_kernel, dim3((unsigned)blocks), dim3(256), 0, st, 1, p, n, g);
}

#define INSTANTIATE(F)                                                                                          \
  template void launch_small_gemm64<F>(const F&, const uint64_t*, int64_t, const uint64_t*, int64_t,            \
                                       const uint64_t*, int64_t, uint64_t*, int64_t, bool, cudaStream_t,        \
                                       const Guard&);                                                           \
  template void launch_block_inverse<F>(const F&, const uint64_t*, int64_t, int, int, uint64_t*, int*,          \
                                        cudaStream_t, bool, const Guard&);                                      \
  template void launch_small_gemm64_batch<F>(const F&, const SgProb*, int, cudaStream_t, const Guard&);         \
  template void launch_window<F>(const F&, const uint64_t*, int64_t, int, int, int, int, int, PanelState*,       \
                                 uint64_t*, uint64_t*, const uint64_t*, uint8_t*, cudaStream_t);                \
  template void launch_bulk<F>(const F&, uint64_t*, int64_t, int, int, int, int, int, PanelState*,              \
                               const uint64_t*, uint64_t*, const uint8_t*, int, cudaStream_t);                  \
  template void launch_couple<F>(const F&, const uint64_t*, int64_t, int, int, const PanelState*,               \
                                 const uint64_t*, uint64_t*, int64_t, cudaStream_t);                            \
  template void launch_trailing_plain<F>(const F&, uint64_t*, int64_t, int, int, int, int, const uint64_t*, int, \
                                         const uint64_t*, int64_t, int, int*, cudaStream_t);                        \
  template cudaError_t launch_plain_mac_peak<F>(const F&, int, int, uint64_t*, cudaStream_t);                      \
  template int plain_blocks_per_sm<F>();

INSTANTIATE(FpBarrett)
INSTANTIATE(FpM61)

}  // namespace modlin
