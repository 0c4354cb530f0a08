// Exact modular trailing update on the 5th-generation tensor cores.
//
//   C[rbeg.., jend..] -= L * U  (mod p),   L: M x K,  U: K x N,  K <= 128,
//
// the rank-K update of the reference's blocked elimination
// (src/fp.rs:202-248), recast as integer GEMMs that are exact:
//
// * Every residue x < p is split into LIMBS unsigned 8-bit limbs,
//   x = sum_i 2^(8i) x_i (LIMBS = 1, 2, 4, 8 for p below 2^8, 2^16, 2^32,
//   2^63). Then L*U = sum_d 2^(8d) S_d with S_d = sum_{i+j=d} L_i U_j.
// * tcgen05.mma kind::i8 (u8 x u8 -> s32) computes the limb products. The B
//   operand of one MMA is the LIMBS planes U_0..U_{LIMBS-1} of an NS-column
//   subtile stacked along N (N = LIMBS*NS = 128); for plane i of L the MMA
//   writes TMEM columns [i*NS, i*NS + 128), so the product L_i U_j lands in
//   column block i+j: the diagonal sums S_d accumulate in TMEM for free.
//   2*LIMBS-1 blocks of NS columns (240 of the 256 allocated for LIMBS = 8).
//   Plane 0 initialises blocks 0..LIMBS-1 and the first K step of plane
//   LIMBS-1 is split in two MMAs so that it initialises the upper blocks.
// * No overflow: S_d <= LIMBS * K * 255^2 < 2^27 for K <= 128.
// * Epilogue: T = sum_d 2^(8d) S_d reduced exactly mod p (for 2^61 - 1 the
//   weights are powers of two mod p, so the 15 blocks fold into one value
//   below 2^62 with 32-bit multiply-adds), then C = C - T mod p. Bit-exact
//   against the u64 Barrett path.
//
// Operands are staged by cp.async.bulk in the canonical K-major, no-swizzle
// UMMA layout: 8-row x 16-byte core matrices, LBO = 128 B between the core
// matrices along K, SBO = 8 K B between 8-row groups. The limb planes are
// written to global memory in exactly that layout by the split kernels, so
// each stage is one contiguous bulk copy.
//
// CTA = 18 warps: warp 0 issues the bulk copies, warp 1 owns TMEM and issues
// the MMAs (one thread), warps 2-17 drain TMEM. Each CTA takes a contiguous
// range of the (M tile, N subtile) space; it keeps the 128-row A tile (all
// limb planes) resident and streams B subtiles through a ring; one CTA per SM
// owns all 512 TMEM columns as two accumulator buffers, so the MMAs of
// subtile s+1 run while the epilogue drains subtile s. Over 2^61 - 1 the
// epilogue is two 8-warp groups, one per accumulator buffer, and C moves by
// 2D TMA (128 x 16 tiles, 128-byte swizzle) through one shared buffer per
// group; other primes use 16 warps and C staged by cp.async. Every mbarrier
// wait is bounded; on expiry the kernel records an error, drains its own
// copies and MMAs (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <climits>
#include <cstring>
#include <cstdint>
#include <type_traits>

#include "field.cuh"
#include "rank_tc.cuh"
#include "launch.cuh"
#include "tc_ptx.cuh"

namespace modlin {

namespace tc {

constexpr int kKMax = 128;      // largest K of one update (two panels), zero padded to 64 or 128
constexpr int kEpiWarps = 16;                // TMEM-draining warps (4 per lane quadrant)
constexpr int kThreads = 32 * (2 + kEpiWarps);  // producer warp, MMA warp, epilogue warps
constexpr uint32_t kTmemCols = 512;  // two accumulator buffers of 256 columns
constexpr int kCStride = 18;         // padded row stride (words) of a staged 128 x 16 C tile (16-byte rows)

// KK = 64 (one panel) or 128 (two panels per pass: half the epilogue work
// per modMAC). A plane tile is 128 rows x KK bytes in 8-row x 16-byte core
// matrices; SBO (next 8-row group) = KK * 8 bytes.
template <int LIMBS, int KK>
struct Shape {
  static constexpr int NS = 128 / LIMBS;             // output columns per subtile
  static constexpr int DIAG = 2 * LIMBS - 1;         // diagonal accumulators
  static constexpr int TILE = 128 * KK;              // one limb plane tile
  static constexpr int KC = KK / 16;                 // 16-byte core matrices along K
  static constexpr uint32_t SBO = KK * 8;
  static constexpr int STAGES = KK == 64 ? 6 : 3;    // B ring depth
  static constexpr int CDEPTH = KK == 64 ? 4 : 2;    // staged C tiles (subtiles) in shared memory
  static constexpr int A_BYTES = LIMBS * TILE;       // resident A tile
  static constexpr int B_BYTES = TILE;               // one B subtile (all planes)
  static constexpr int ZERO_BYTES = 0;
  static constexpr int C_BYTES = LIMBS == 8 ? CDEPTH * 128 * kCStride * 8 : 0;  // staged C tiles
  static constexpr int SMEM = A_BYTES + STAGES * B_BYTES + ZERO_BYTES + 1024 + C_BYTES;
  static_assert(SMEM <= 227 * 1024, "shared memory");
  // p = 2^61 - 1: the epilogue stages C by TMA, one 128 x 16 tile per group.
  static constexpr int STAGES_M61 = KK == 64 ? 8 : 2;
  static constexpr int C_TMA_BYTES = 4 * 128 * 16 * 8;  // two 128 x 16 C tiles per epilogue group
  static constexpr int SMEM_M61 = A_BYTES + STAGES_M61 * B_BYTES + ZERO_BYTES + 1024 + C_TMA_BYTES;
  static_assert(SMEM_M61 <= 227 * 1024, "shared memory");
};

struct Sched {
  int mtiles, nsub;
};

// ---------------------------------------------------------------------------
// Limb split of L (A operand): Aw[mt][i][g][kc][rr][kb], thread per (row, kc).
// ---------------------------------------------------------------------------
template <int LIMBS, int KK>
__global__ void split_a_kernel(const uint64_t* __restrict__ Lbuf, int64_t lda, int32_t r0, int32_t rbeg, int32_t rend,
                               int32_t K, int32_t mpad, uint8_t* __restrict__ Aw, Guard g) {
  using SH = Shape<LIMBS, KK>;
  pdl_wait();
  if (guard_skip(g)) return;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)mpad * SH::KC) return;
  const int ri_all = (int)(idx / SH::KC), kc = (int)(idx % SH::KC);
  const int mt = ri_all >> 7, ri = ri_all & 127;
  const int64_t r = (int64_t)rbeg + ri_all;
  uint64_t v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int k = kc * 16 + q;
    v[q] = (r < rend && k < K) ? Lbuf[(r - r0) * lda + k] : 0;
  }
  const int64_t tile_off = ((int64_t)mt * LIMBS) * SH::TILE + (((ri >> 3) * SH::KC + kc) * 8 + (ri & 7)) * 16;
#pragma unroll
  for (int i = 0; i < LIMBS; ++i) {
    uint32_t w[4];
#pragma unroll
    for (int q4 = 0; q4 < 4; ++q4) {
      uint32_t x = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) x |= (uint32_t)((v[q4 * 4 + b] >> (8 * i)) & 0xFF) << (8 * b);
      w[q4] = x;
    }
    *reinterpret_cast<uint4*>(Aw + tile_off + (int64_t)i * SH::TILE) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// ---------------------------------------------------------------------------
// Limb split of U (B operand): Bw[sub][j][g2][kc][rr][kb], thread per
// (column, kc); reads Ubuf[k][c] (coalesced over c).
// ---------------------------------------------------------------------------
template <int LIMBS, int KK>
__global__ void split_b_kernel(const uint64_t* __restrict__ Ubuf, int64_t ldU, int32_t jend, int32_t cend, int32_t K,
                               int32_t npad, uint8_t* __restrict__ Bw, Guard g) {
  pdl_wait();
  if (guard_skip(g)) return;
  using SH = Shape<LIMBS, KK>;
  constexpr int NS = SH::NS;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)npad * SH::KC) return;
  const int kc = (int)(idx / npad), ci = (int)(idx - (int64_t)kc * npad);
  const int64_t c = (int64_t)jend + ci;
  uint64_t v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int k = kc * 16 + q;
    v[q] = (c < cend && k < K) ? Ubuf[(int64_t)k * ldU + c] : 0;
  }
  const int sub = ci / NS, cc = ci % NS;
  const int64_t base = (int64_t)sub * SH::TILE + (((cc >> 3) * SH::KC + kc) * 8 + (cc & 7)) * 16;
#pragma unroll
  for (int j = 0; j < LIMBS; ++j) {
    uint32_t w[4];
#pragma unroll
    for (int q4 = 0; q4 < 4; ++q4) {
      uint32_t x = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) x |= (uint32_t)((v[q4 * 4 + b] >> (8 * j)) & 0xFF) << (8 * b);
      w[q4] = x;
    }
    *reinterpret_cast<uint4*>(Bw + base + (int64_t)j * NS * KK) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Exact residue of sum_d 2^(8d) S_d for one output column (S in registers
// acc_lo/acc_hi = the two 128-bit halves prepared by the fold).
template <class F>
__device__ __forceinline__ uint64_t finish(const F& f, u128 lo, u128 hi, uint64_t r64) {
  if constexpr (std::is_same<F, FpM61>::value) {
    return f.reduce(lo);  // already folded into one 128-bit value
  } else {
    return f.add(f.reduce(lo), f.mul(f.reduce(hi), r64));
  }
}

__device__ __forceinline__ uint64_t mad_wide_u32(uint32_t a, uint32_t b, uint64_t c) {
  uint64_t d;
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

// x = sum_{d<15} 2^(8d) a[d][c] mod 2^61 - 1, lazily: x < 2^62 and congruent.
// The diagonal sums are a[d][c] <= 8 * 128 * 255^2 < 2^26 (K <= 128), and
// 2^(8(d+8)) = 8 * 2^(8d) (mod p), so V_d = a_d + 8 a_(d+8) <= 57 * 128 * 255^2
// < 2^29 (d < 7; V_7 = a_7). L = sum_{d<4} 2^(8d) V_d and H = sum_{d<4}
// 2^(8d) V_(d+4) are < 2^54, and 2^32 H = 2^32 (H mod 2^29) + (H >> 29) (mod p)
// since 2^61 = 1, so x = L + 2^32 (H mod 2^29) + (H >> 29) < 2^62.
__device__ __forceinline__ uint64_t m61_fold15(const uint32_t (&a)[15][4], int c) {
  uint32_t V[8];
#pragma unroll
  for (int d = 0; d < 7; ++d) V[d] = a[d][c] + 8u * a[d + 8][c];
  V[7] = a[7][c];
  const uint64_t L = mad_wide_u32(V[3], 1u << 24, mad_wide_u32(V[2], 1u << 16, mad_wide_u32(V[1], 1u << 8, V[0])));
  const uint64_t H = mad_wide_u32(V[7], 1u << 24, mad_wide_u32(V[6], 1u << 16, mad_wide_u32(V[5], 1u << 8, V[4])));
  return L + ((uint64_t)((uint32_t)H & 0x1FFFFFFFu) << 32) + (H >> 29);
}

// (cv - x) mod 2^61 - 1 for a canonical cv and any x < 2^62:
// y = cv + 4p - x lies in (0, 2^64), one fold leaves y1 <= p + 7, and one
// conditional subtraction makes it canonical.
__device__ __forceinline__ uint64_t m61_sub_lazy(uint64_t cv, uint64_t x) {
  const uint64_t y = cv + (4 * kM61) - x;
  const uint64_t y1 = (y & kM61) + (y >> 61);
  return y1 >= kM61 ? y1 - kM61 : y1;
}

// In place 8 x 8 byte transpose: afterwards byte c of t[i] is the former
// byte i of t[c] (swap the off-diagonal 4 x 4, then 2 x 2, then 1 x 1
// blocks).
__device__ __forceinline__ void bytes_transpose8(uint64_t (&t)[8]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint64_t x = ((t[j] >> 32) ^ t[j + 4]) & 0x00000000FFFFFFFFull;
    t[j] ^= x << 32;
    t[j + 4] ^= x;
  }
#pragma unroll
  for (int j = 0; j < 8; j += (j & 1) ? 3 : 1) {  // 0, 1, 4, 5
    const uint64_t x = ((t[j] >> 16) ^ t[j + 2]) & 0x0000FFFF0000FFFFull;
    t[j] ^= x << 16;
    t[j + 2] ^= x;
  }
#pragma unroll
  for (int j = 0; j < 8; j += 2) {
    const uint64_t x = ((t[j] >> 8) ^ t[j + 1]) & 0x00FF00FF00FF00FFull;
    t[j] ^= x << 8;
    t[j + 1] ^= x;
  }
}

// Writes the 8 residues v (columns kcol .. kcol+7 of K, kcol a multiple of
// 8, of limb row lr) as bytes of the 8 limb planes in the A-operand layout
// of a K = kk update (split_a_kernel's layout).
__device__ __forceinline__ void store_limbs8(uint8_t* Aw, int kk, int64_t lr, int kcol, const uint64_t (&v)[8]) {
  uint64_t t[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) t[c] = v[c];
  bytes_transpose8(t);
  const int64_t tile = 128 * (int64_t)kk;
  const int lmt = (int)(lr >> 7), lri = (int)(lr & 127);
  uint8_t* base = Aw + (int64_t)lmt * 8 * tile + (((lri >> 3) * (kk >> 4) + (kcol >> 4)) * 8 + (lri & 7)) * 16 +
                  (kcol & 15);
#pragma unroll
  for (int i = 0; i < 8; ++i) *reinterpret_cast<uint64_t*>(base + i * tile) = t[i];
}

template <class F, int LIMBS, int KK>
__global__ void __launch_bounds__(kThreads, 1)
    trailing_tc_kernel(F f, const uint8_t* __restrict__ Aw, const uint8_t* __restrict__ Bw, uint64_t* m, int64_t ld,
                       int32_t rbeg, int32_t rend, int32_t jend, int32_t cend, Sched S, uint64_t r64, int* err,
                       const __grid_constant__ CUtensorMap cmap, int use_tma, Guard guard, LimbOut lo) {
  using SH = Shape<LIMBS, KK>;
  constexpr int NS = SH::NS;
  // p = 2^61 - 1: two epilogue groups of 8 warps, one per accumulator buffer.
  constexpr bool kM61Path = std::is_same<F, FpM61>::value;
  constexpr int kStages = kM61Path ? SH::STAGES_M61 : SH::STAGES;
  constexpr int kCDepth = SH::CDEPTH;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;                        // A_BYTES
  uint8_t* sB = smem + SH::A_BYTES;          // kStages * 8 KB
  uint8_t* sZ = sB + kStages * SH::B_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sZ + SH::ZERO_BYTES);
  uint64_t* sC = reinterpret_cast<uint64_t*>(sZ + SH::ZERO_BYTES + 1024);  // [kCDepth][128][kCStride]
  uint64_t* a_full = bars + 0;
  uint64_t* a_empty = bars + 1;
  uint64_t* acc_full = bars + 2;   // [2]: accumulator buffer b holds a finished subtile
  uint64_t* acc_empty = bars + 4;  // [2]: the epilogue has drained buffer b
  uint64_t* mma_done = bars + 6;
  uint64_t* b_full = bars + 8;
  uint64_t* b_empty = bars + 8 + kStages;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int skip_sh;

  pdl_wait();
  if (threadIdx.x == 0) skip_sh = guard_skip(guard);
  __syncthreads();
  if (skip_sh) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(a_full, 1);
    mbar_init(a_empty, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, kM61Path ? kEpiWarps / 2 : kEpiWarps);
    }
    mbar_init(mma_done, 1);
    for (int q = 0; q < 4; ++q) mbar_init(bars + 40 + q, 1);  // c_full of (epilogue group, C buffer), 2^61 - 1
    for (int st = 0; st < kStages; ++st) {
      mbar_init(b_full + st, 1);
      mbar_init(b_empty + st, 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base_sh;
  // This CTA's contiguous range of the (M tile, N subtile) space, row-major:
  // balanced to one subtile, and an A tile is loaded once per M tile touched.
  const int64_t total = (int64_t)S.mtiles * S.nsub;
  const int64_t g0 = total * blockIdx.x / gridDim.x, g1 = total * (blockIdx.x + 1) / gridDim.x;

  if (warp == 0) {
    // ---------------- producer: bulk copies -------------------------------
    if (lane == 0) {
      int cur = -1, nload = 0, it = 0;
      int mt = (int)(g0 / S.nsub), sb = (int)(g0 - (int64_t)mt * S.nsub);
      bool ok = true;
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        if (mt != cur) {
          if (nload > 0 && !(ok = mbar_wait(a_empty, (nload - 1) & 1, err))) break;
          mbar_arrive_expect_tx(a_full, SH::A_BYTES);
          bulk_g2s(sA, Aw + (int64_t)mt * SH::A_BYTES, SH::A_BYTES, a_full);
          cur = mt;
          ++nload;
        }
        const int st = it % kStages;
        if (it >= kStages && !(ok = mbar_wait(b_empty + st, ((it / kStages) - 1) & 1, err))) break;
        mbar_arrive_expect_tx(b_full + st, SH::B_BYTES);
        bulk_g2s(sB + st * SH::B_BYTES, Bw + (int64_t)sb * SH::B_BYTES, SH::B_BYTES, b_full + st);
      }
      if (!ok) {
        atomicExch(err, 1);
        // Let this CTA's own copies land before the CTA can exit.
        if (nload > 0) mbar_wait(a_full, (nload - 1) & 1, err + 1);
        for (int st = 0; st < kStages; ++st)
          if (it > st) mbar_wait(b_full + st, ((it - 1 - st) / kStages) & 1, err + 1);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ------------------------------------------
    if (lane == 0) {
      int cur = -1, nload = 0, it = 0;
      bool ok = true;
      const uint32_t id_full = idesc_i8(LIMBS * NS);
      const uint32_t id_upper = idesc_i8(LIMBS > 1 ? (LIMBS - 1) * NS : 16);  // B planes 1 .. LIMBS-1
      const uint32_t id_plane = idesc_i8(NS);                                  // B plane 0
      int mt = (int)(g0 / S.nsub), sb = (int)(g0 - (int64_t)mt * S.nsub);
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        if (mt != cur) {
          if (nload > 0) mma_commit(a_empty);  // the previous A tile is free once these MMAs finish
          if (!(ok = mbar_wait(a_full, nload & 1, err))) break;
          fence_after();
          cur = mt;
          ++nload;
        }
        const int st = it % kStages;
        const int ab = it & 1;  // accumulator buffer
        if (it >= 2 && !(ok = mbar_wait(acc_empty + ab, ((it >> 1) - 1) & 1, err))) break;
        if (!(ok = mbar_wait(b_full + st, (it / kStages) & 1, err))) break;
        fence_after();
        const uint8_t* bt = sB + st * SH::B_BYTES;
        const uint32_t dacc = tmem + ab * 256;
        // Plane 0 (first K step without accumulate) initialises diagonal
        // blocks 0 .. LIMBS-1. The first K step of plane LIMBS-1 is split so
        // that it initialises blocks LIMBS .. 2 LIMBS-2 (B planes 1 .. LIMBS-1,
        // no accumulate) and adds into block LIMBS-1 (B plane 0); every other
        // MMA accumulates.
        auto adesc = [&](int i, int ks) { return smem_desc(sA + i * SH::TILE + ks * 256, SH::SBO); };
#pragma unroll
        for (int ks = 0; ks < KK / 32; ++ks)
          mma_i8(dacc, adesc(0, ks), smem_desc(bt + ks * 256, SH::SBO), id_full, ks > 0 ? 1u : 0u);
        if (LIMBS > 1) {
          mma_i8(dacc + LIMBS * NS, adesc(LIMBS - 1, 0), smem_desc(bt + NS * KK, SH::SBO), id_upper, 0);
          mma_i8(dacc + (LIMBS - 1) * NS, adesc(LIMBS - 1, 0), smem_desc(bt, SH::SBO), id_plane, 1);
#pragma unroll
          for (int ks = 1; ks < KK / 32; ++ks)
            mma_i8(dacc + (LIMBS - 1) * NS, adesc(LIMBS - 1, ks), smem_desc(bt + ks * 256, SH::SBO), id_full, 1);
        }
#pragma unroll
        for (int i = 1; i < LIMBS - 1; ++i)
#pragma unroll
          for (int ks = 0; ks < KK / 32; ++ks)
            mma_i8(dacc + i * NS, adesc(i, ks), smem_desc(bt + ks * 256, SH::SBO), id_full, 1);
        mma_commit(b_empty + st);
        mma_commit(acc_full + ab);
      }
      if (!ok) atomicExch(err, 1);
      mma_commit(mma_done);
      mbar_wait(mma_done, 0, err + 1);
    }
    __syncwarp();
  } else if constexpr (kM61Path) {
    // ---------------- epilogue, p = 2^61 - 1 ----------------------------------
    // Two groups of 8 warps: group g drains accumulator buffer g, i.e. the
    // subtiles it = g, g + 2, ... of this CTA's range, so each group has two
    // MMA periods per subtile and the groups' phases interleave. In a group,
    // warp w reads TMEM lanes 32*(w%4)..+32 (its 32 rows) and one half (8
    // columns) of the 16-column subtile, so every thread owns one row x 8
    // columns. It folds the 15 diagonal sums of each column and releases the
    // accumulator buffer first; then C - T is formed against C.
    // C moves by TMA (use_tma): the group's leader thread loads the 128 x 16
    // C tile of its next subtile into the group's shared buffer (128-byte
    // swizzle, so the threads' row-wise accesses are conflict-free), the
    // threads replace it in place by C - T, and the leader stores it back
    // with one tensor copy, then loads the group's next tile. Without TMA
    // (a row stride or column offset that is not 16-byte aligned) every
    // thread reads and writes its 8 values directly.
    const int ew = warp - 2;
    const int grp = ew >> 3;          // accumulator buffer this group drains
    const int quad = warp & 3;        // TMEM lane quadrant
    const int half = (ew >> 2) & 1;   // column half of the subtile
    const int row = quad * 32 + lane;
    const bool leader = (ew & 7) == 0 && lane == 0;
    const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16) + grp * 256 + half * 8;
    // Two C buffers per group: the tile of the group's next subtile loads
    // while the current one is computed and stored.
    uint64_t* cbuf0 = reinterpret_cast<uint64_t*>(sZ + SH::ZERO_BYTES + 1024) + grp * 2 * (128 * 16);
    uint64_t* c_full0 = bars + 40 + 2 * grp;
    const int64_t nsub = S.nsub;
    // Subtile it = grp + 2 k of [g0, g1): (mt, sb) tracked incrementally.
    int64_t g = g0 + grp;
    int64_t mt = g / nsub, sb = g - mt * nsub;
    auto advance = [&]() {
      g += 2;
      sb += 2;
      while (sb >= nsub) {
        sb -= nsub;
        ++mt;
      }
    };
    int loads = 0;  // TMA loads issued by the leader; load j goes to buffer j & 1
    auto tma_load = [&]() {
      uint64_t* cf = c_full0 + (loads & 1);
      mbar_arrive_expect_tx(cf, 128 * 16 * 8);
      tma_load_2d(cbuf0 + (loads & 1) * (128 * 16), &cmap, (int32_t)(jend + sb * NS), (int32_t)(rbeg + mt * 128), cf);
      ++loads;
    };
    auto load_c = [&](uint64_t (&cv)[8]) {
      const int64_t r = (int64_t)rbeg + mt * 128 + row;
      const int64_t c0 = (int64_t)jend + sb * NS + half * 8;
      const uint64_t* src = m + r * ld + c0;
#pragma unroll
      for (int c = 0; c < 8; ++c) cv[c] = (r < rend && c0 + c < cend) ? __ldcs(src + c) : 0;
    };
    // lo.c_zero: C is zero and not written (only the limb planes are).
    const bool czero = lo.c_zero != 0;
    const bool tma = use_tma && !czero;
    auto put_limbs = [&](uint64_t (&res)[8]) {
      const int64_t r = (int64_t)rbeg + mt * 128 + row;
      const int64_t c0 = (int64_t)jend + sb * NS + half * 8;
      const int64_t lr = r - lo.row0;
      if (r >= rend || lr < 0) return;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c0 + c >= cend) res[c] = 0;
      store_limbs8(lo.Aw, lo.kk, lr, (int)(c0 - jend), res);
    };
    uint64_t cv[8];
    if (g < g1 && !czero) {
      if (!use_tma) {
        load_c(cv);
      } else if (leader) {
        tma_load();  // subtile 0 into buffer 0
        if (g + 2 < g1) {
          advance();
          tma_load();  // subtile 1 into buffer 1
          g -= 2;      // back to subtile 0
          sb -= 2;
          while (sb < 0) {
            sb += nsub;
            --mt;
          }
        }
      }
    }
    bool ok = true;
    for (int k = 0; g < g1; ++k) {
      bool okw = __all_sync(0xffffffffu, mbar_wait(acc_full + grp, k & 1, err));
      uint64_t x[8];
      if (okw) {
        fence_after();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          uint32_t a[15][4];
#pragma unroll
          for (int d = 0; d < 15; ++d) tmem_ld4(lane_base + d * NS + q * 4, a[d]);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 4; ++c) x[4 * q + c] = m61_fold15(a, c);
        }
        fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty + grp);
      }
      uint64_t res[8];
      if (tma) {
        uint64_t* const cbuf = cbuf0 + (k & 1) * (128 * 16);
        if (okw) okw = __all_sync(0xffffffffu, mbar_wait(c_full0 + (k & 1), (k >> 1) & 1, err));
        if (okw) {
          // Row `row`, 16-byte chunks 4 half .. +4 of the 128-byte row; the
          // 128-byte swizzle XORs the chunk index (address bits 4-6) with
          // address bits 7-9.
          uint64_t* rp = cbuf + row * 16;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint64_t* lp = rp + (half * 4 + q) * 2;
            const uint32_t a = smem_u32(lp);
            const int delta = (int)((a ^ (a >> 3)) & 0x70u) - (int)(a & 0x70u);
            ulonglong2* pq = reinterpret_cast<ulonglong2*>(reinterpret_cast<uint8_t*>(lp) + delta);
            const ulonglong2 v = *pq;
            res[2 * q] = m61_sub_lazy(v.x, x[2 * q]);
            res[2 * q + 1] = m61_sub_lazy(v.y, x[2 * q + 1]);
            *pq = make_ulonglong2(res[2 * q], res[2 * q + 1]);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        // Every thread of the group reaches this barrier, failed or not; the
        // group leaves together when any of them failed.
        if (!group_bar_and(1 + grp, okw)) {
          ok = false;
          break;
        }
        if (leader) {
          tma_store_2d(&cmap, (int32_t)(jend + sb * NS), (int32_t)(rbeg + mt * 128), cbuf);
          bulk_commit();
        }
        if (lo.Aw) put_limbs(res);
        advance();
        if (leader && g < g1 && loads == k + 1) {
          // The tile after next goes to the other buffer once the store
          // issued from it one subtile ago has read it (this subtile's store
          // may still be reading).
          asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
          tma_load();
        }
      } else {
        if (!okw) {
          ok = false;
          break;
        }
        const int64_t r = (int64_t)rbeg + mt * 128 + row;
        const int64_t c0 = (int64_t)jend + sb * NS + half * 8;
#pragma unroll
        for (int c = 0; c < 8; ++c) res[c] = m61_sub_lazy(czero ? 0 : cv[c], x[c]);
        if (!czero && r < rend) {
          uint64_t* dst = m + r * ld + c0;
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c0 + c < cend) dst[c] = res[c];
        }
        if (lo.Aw) put_limbs(res);
        advance();
        if (g < g1 && !czero) load_c(cv);
      }
    }
    if (leader && tma) {
      bulk_wait_all0();  // stores complete
      if (!ok) {  // loads still landing: the last one into each buffer
        for (int j = loads - 2 > 0 ? loads - 2 : 0; j < loads; ++j) mbar_wait(c_full0 + (j & 1), (j >> 1) & 1, err + 1);
      }
    }
    if (!ok) atomicExch(err, 1);
  } else {
    // ---------------- epilogue: TMEM -> exact residue -> C -= T -------------
    // kEpiWarps warps: warp w reads TMEM lanes 32*(w%4)..+32 (its rows) and
    // the 4-column quarter (w-2)/4 of every 16-column chunk; the accumulator
    // buffer is released as soon as its columns are in registers.
    const int ew = warp - 2;
    const int quad = warp & 3;
    const int qc = ew >> 2;  // column quarter
    const int row = quad * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16) + qc * 4;
    int it = 0;
    bool ok = true;
    if constexpr (LIMBS == 8) {
      // C goes through shared memory so that global accesses are coalesced.
      // The 4 warps of a TMEM lane quadrant form a group that owns rows
      // 32*quad..+32 of the 128 x 16 tile: warp (quad, qc) copies rows
      // 32*quad + 8*qc..+8 kCDepth - 1 subtiles ahead with cp.async, every
      // thread then works on its own row in shared memory, and the results
      // leave the same way. Each group synchronises on its own named barrier
      // (1 + quad), so the four groups drift and their phases overlap.
      constexpr int kRowsPerWarp = 8;
      const int rbase_w = quad * 32 + qc * kRowsPerWarp;
      const int rr = lane >> 4, cc = lane & 15, rr4 = lane >> 3, cc2 = (lane & 7) * 2;
      auto epi_bar = [quad]() { asm volatile("bar.sync %0, 128;" ::"r"(1 + quad) : "memory"); };
      // 16-byte copies when every row start is 16-byte aligned and the
      // subtile is complete, else 8-byte copies.
      const bool vec_ld = (ld & 1) == 0 && ((uintptr_t)m & 15) == 0 && (jend & 1) == 0;
      int64_t pg = g0;
      int pmt = (int)(g0 / S.nsub), psb = (int)(g0 - (int64_t)pmt * S.nsub);
      int pcount = 0;
      auto pf_issue = [&]() {
        if (pg < g1) {
          const int mt = pmt, sb = psb;
          const int64_t pbase = (int64_t)rbeg + (int64_t)mt * 128;
          uint64_t* slot = sC + (size_t)(pcount % kCDepth) * 128 * kCStride;
          const int64_t sc0 = (int64_t)jend + (int64_t)sb * NS;
          if (vec_ld && sc0 + 16 <= cend) {
#pragma unroll
            for (int i = 0; i < kRowsPerWarp / 4; ++i) {
              const int lr = rbase_w + 4 * i + rr4;
              const int64_t gr = pbase + lr;
              if (gr < rend) cp_async16(slot + lr * kCStride + cc2, m + gr * ld + sc0 + cc2);
            }
          } else {
            const int64_t gc = sc0 + cc;
#pragma unroll
            for (int i = 0; i < kRowsPerWarp / 2; ++i) {
              const int lr = rbase_w + 2 * i + rr;
              const int64_t gr = pbase + lr;
              if (gr < rend && gc < cend) cp_async8(slot + lr * kCStride + cc, m + gr * ld + gc);
            }
          }
          ++pg;
          if (++psb == S.nsub) {
            psb = 0;
            ++pmt;
          }
        }
        cp_async_commit();
        ++pcount;
      };
      for (int k = 0; k < kCDepth - 1; ++k) pf_issue();
      int mt = (int)(g0 / S.nsub), sb = (int)(g0 - (int64_t)mt * S.nsub);
      for (int64_t g = g0; g < g1; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        const int64_t base = (int64_t)rbeg + (int64_t)mt * 128;
        const bool row_ok = base + row < rend;
        const int ab = it & 1;
        const uint32_t lane_addr = lane_base + ab * 256;
        cp_async_wait<kCDepth - 2>();
        epi_bar();  // this subtile's C is in shared memory; the previous one has been stored
        pf_issue();
        uint64_t* slot = sC + (size_t)(it % kCDepth) * 128 * kCStride;
        uint64_t* my = slot + row * kCStride + qc * 4;
        const int64_t c0 = (int64_t)jend + (int64_t)sb * NS + qc * 4;
        uint64_t cv[4];
        {
          const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(my);
          const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(my + 2);
          cv[0] = v0.x;
          cv[1] = v0.y;
          cv[2] = v1.x;
          cv[3] = v1.y;
        }
        if (ok) ok = __all_sync(0xffffffffu, mbar_wait(acc_full + ab, (it >> 1) & 1, err));
        if (ok) {
          fence_after();
          uint64_t res[4];
          {
            u128 lo[4], hi[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) lo[c] = hi[c] = 0;
#pragma unroll 1
            for (int d = 0; d < SH::DIAG; ++d) {
              uint32_t a[4];
              tmem_ld4(lane_addr + d * NS, a);
              tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < 4; ++c) {
                asm volatile("" : "+r"(a[c]));
                if (d < 8)
                  lo[c] += (u128)a[c] << (8 * d);
                else
                  hi[c] += (u128)a[c] << (8 * (d - 8));
              }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty + ab);
#pragma unroll
            for (int c = 0; c < 4; ++c) res[c] = f.sub(cv[c], finish(f, lo[c], hi[c], r64));
          }
          if (row_ok) {
            if (c0 + 4 <= cend) {
              *reinterpret_cast<ulonglong2*>(my) = make_ulonglong2(res[0], res[1]);
              *reinterpret_cast<ulonglong2*>(my + 2) = make_ulonglong2(res[2], res[3]);
            } else {
#pragma unroll
              for (int c = 0; c < 4; ++c)
                if (c0 + c < cend) my[c] = res[c];
            }
          }
        }
        epi_bar();  // results of all rows in shared memory
        if (ok) {
          const int64_t sc0 = (int64_t)jend + (int64_t)sb * NS;
          if (vec_ld && sc0 + 16 <= cend) {
#pragma unroll
            for (int i = 0; i < kRowsPerWarp / 4; ++i) {
              const int lr = rbase_w + 4 * i + rr4;
              const int64_t gr = base + lr;
              if (gr < rend)
                *reinterpret_cast<ulonglong2*>(m + gr * ld + sc0 + cc2) =
                    *reinterpret_cast<const ulonglong2*>(slot + lr * kCStride + cc2);
            }
          } else {
            const int64_t gc = sc0 + cc;
#pragma unroll
            for (int i = 0; i < kRowsPerWarp / 2; ++i) {
              const int lr = rbase_w + 2 * i + rr;
              const int64_t gr = base + lr;
              if (gr < rend && gc < cend) m[gr * ld + gc] = slot[lr * kCStride + cc];
            }
          }
        }
      }
    } else {
      // Fewer limbs (p < 2^32): NS >= 32 columns per subtile; direct access.
      int mt = (int)(g0 / S.nsub), sb = (int)(g0 - (int64_t)mt * S.nsub);
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        const int64_t r = (int64_t)rbeg + (int64_t)mt * 128 + row;
        const bool row_ok = r < rend;
        const int ab = it & 1;
        const uint32_t lane_addr = lane_base + ab * 256;
        ok = __all_sync(0xffffffffu, mbar_wait(acc_full + ab, (it >> 1) & 1, err));
        if (!ok) break;
        fence_after();
        for (int q = 0; q < NS / 16; ++q) {
          const int64_t c0 = (int64_t)jend + (int64_t)sb * NS + q * 16 + qc * 4;
          uint64_t* crow = m + r * ld + c0;
          uint64_t cv[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) cv[c] = (row_ok && c0 + c < cend) ? crow[c] : 0;
          u128 lo[4], hi[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) lo[c] = hi[c] = 0;
#pragma unroll 1
          for (int d = 0; d < SH::DIAG; ++d) {
            uint32_t a[4];
            tmem_ld4(lane_addr + d * NS + q * 16, a);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              asm volatile("" : "+r"(a[c]));
              if (d < 8)
                lo[c] += (u128)a[c] << (8 * d);
              else
                hi[c] += (u128)a[c] << (8 * (d - 8));
            }
          }
          if (q == NS / 16 - 1) {
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty + ab);
          }
          if (row_ok) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
              if (c0 + c < cend) crow[c] = f.sub(cv[c], finish(f, lo[c], hi[c], r64));
          }
        }
      }
    }
    cp_async_wait<0>();  // no prefetch may still target this CTA's shared memory
    if (!ok) atomicExch(err, 1);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// The same update over 2^61 - 1 on CTA pairs (cta_group::2, cluster of 2):
// the pair computes 256-row x 16-column subtiles with M = 256 MMAs issued by
// the even CTA; each CTA keeps its own 128 rows of A resident and streams its
// half of every B subtile (limb planes 0..3 in the even CTA, 4..7 in the odd
// one), so each SM reads 6 KB of operands from shared memory per 64 tensor
// cycles instead of 8 KB. Each CTA's TMEM holds its rows' accumulators; its
// epilogue is the 1-CTA kernel's (two 8-warp groups, C by 2D TMA). The even
// CTA's MMA thread learns that the odd CTA's copies have landed from that
// CTA's relay thread (a remote mbarrier arrive), and the odd CTA's epilogue
// releases TMEM buffers by remote arrives; MMA completions reach both CTAs
// through multicast commits. The upper diagonal blocks 8..14 are zeroed by
// the epilogue (TMEM stores) after it drains a buffer, and once at start.
// ---------------------------------------------------------------------------
template <int KK>
struct PairShape {
  static constexpr int NS = 16;
  static constexpr int TILE = 128 * KK;  // one limb plane of 128 rows
  static constexpr int KC = KK / 16;
  static constexpr uint32_t SBO = KK * 8;
  static constexpr int A_BYTES = 8 * TILE;   // this CTA's 128 rows, 8 planes
  static constexpr int BH_BYTES = 4 * 16 * KK;  // half a B subtile: 4 limb planes x 16 columns x KK
  static constexpr int STAGES = KK == 64 ? 8 : 6;
  static constexpr int C_BYTES = 2 * 128 * 16 * 8;
  static constexpr int SMEM = A_BYTES + STAGES * BH_BYTES + 1024 + C_BYTES;
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

template <int KK>
__global__ void __launch_bounds__(kThreads, 1)
    trailing_tc_pair_kernel(const uint8_t* __restrict__ Aw, const uint8_t* __restrict__ Bw, int32_t rbeg,
                            int32_t jend, Sched S, int* err, const __grid_constant__ CUtensorMap cmap,
                            Guard guard) {
  using SH = PairShape<KK>;
  constexpr int NS = SH::NS;
  constexpr int kStages = SH::STAGES;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;
  uint8_t* sB = smem + SH::A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kStages * SH::BH_BYTES);
  uint64_t* sC = bars + 128;  // 1 KB of barriers, then the C tiles (1024-byte aligned)
  uint64_t* a_full = bars + 0;
  uint64_t* a_empty = bars + 1;
  uint64_t* acc_full = bars + 2;   // [2]
  uint64_t* acc_empty = bars + 4;  // [2], even CTA: 8 local + 8 remote arrivals
  uint64_t* mma_done = bars + 6;
  uint64_t* a_peer = bars + 7;     // even CTA: the odd CTA's A tile has landed
  uint64_t* b_full = bars + 8;
  uint64_t* b_empty = bars + 8 + kStages;
  uint64_t* b_peer = bars + 8 + 2 * kStages;  // even CTA: the odd CTA's B half has landed
  __shared__ uint32_t tmem_base_sh;
  __shared__ int skip_sh;

  pdl_wait();
  // Both CTAs of a pair read the same word (it cannot change during the launch).
  if (threadIdx.x == 0) skip_sh = guard_skip(guard);
  __syncthreads();
  if (skip_sh) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t crank = cluster_rank();
  const int pair = blockIdx.x >> 1;
  const int npairs = gridDim.x >> 1;
  if (threadIdx.x == 0) {
    mbar_init(a_full, 1);
    mbar_init(a_empty, 1);
    mbar_init(a_peer, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, kEpiWarps);  // both CTAs' group of 8 warps
    }
    mbar_init(mma_done, 1);
    mbar_init(bars + 40, 1);  // c_full of epilogue group 0
    mbar_init(bars + 41, 1);  // c_full of epilogue group 1
    for (int st = 0; st < kStages; ++st) {
      mbar_init(b_full + st, 1);
      mbar_init(b_empty + st, 1);
      mbar_init(b_peer + st, 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_base_sh;
  if (warp >= 2) {
    // Zero the upper diagonal blocks (8 .. 14) of this group's buffer.
    const int ew = warp - 2, grp = ew >> 3, quad = warp & 3, half = (ew >> 2) & 1;
    const uint32_t lb = tmem + ((uint32_t)(quad * 32) << 16) + grp * 256 + half * 8;
#pragma unroll
    for (int d = 8; d < 15; ++d) tmem_st8_zero(lb + d * NS);
    tmem_wait_st();
  }
  fence_before();
  cluster_sync_all();  // both CTAs' barriers initialised and their buffers zeroed
  fence_after();
  const int64_t total = (int64_t)S.mtiles * S.nsub;  // (256-row tile, subtile) pairs
  const int64_t g0 = total * pair / npairs, g1 = total * (pair + 1) / npairs;

  if (warp == 0) {
    // ---------------- producer (both CTAs): this CTA's A rows and B half ----
    if (lane == 0) {
      int cur = -1, nload = 0, it = 0;
      int64_t mt = g0 / S.nsub, sb = g0 - mt * S.nsub;
      bool ok = true;
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        if (mt != cur) {
          if (nload > 0 && !(ok = mbar_wait(a_empty, (nload - 1) & 1, err))) break;
          mbar_arrive_expect_tx(a_full, SH::A_BYTES);
          bulk_g2s(sA, Aw + (2 * mt + crank) * (int64_t)SH::A_BYTES, SH::A_BYTES, a_full);
          cur = (int)mt;
          ++nload;
        }
        const int st = it % kStages;
        if (it >= kStages && !(ok = mbar_wait(b_empty + st, ((it / kStages) - 1) & 1, err))) break;
        mbar_arrive_expect_tx(b_full + st, SH::BH_BYTES);
        bulk_g2s(sB + st * SH::BH_BYTES, Bw + sb * (int64_t)(2 * SH::BH_BYTES) + crank * SH::BH_BYTES, SH::BH_BYTES,
                 b_full + st);
      }
      if (!ok) {
        atomicExch(err, 1);
        if (nload > 0) mbar_wait(a_full, (nload - 1) & 1, err + 1);
        for (int st = 0; st < kStages; ++st)
          if (it > st) mbar_wait(b_full + st, ((it - 1 - st) / kStages) & 1, err + 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && crank == 1) {
      // ---------------- relay (odd CTA): tell the even CTA's MMA thread ------
      const uint32_t peer_a = cluster_addr(a_peer, 0);
      int cur = -1, nload = 0, it = 0;
      int64_t mt = g0 / S.nsub, sb = g0 - mt * S.nsub;
      bool ok = true;
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        if (mt != cur) {
          if (!(ok = mbar_wait(a_full, nload & 1, err))) break;
          mbar_arrive_cluster(peer_a);
          cur = (int)mt;
          ++nload;
        }
        const int st = it % kStages;
        if (!(ok = mbar_wait(b_full + st, (it / kStages) & 1, err))) break;
        mbar_arrive_cluster(cluster_addr(b_peer + st, 0));
      }
      if (!ok) atomicExch(err, 1);
    } else if (lane == 0) {
      // ---------------- MMA issuer (even CTA) --------------------------------
      int cur = -1, nload = 0, it = 0;
      bool ok = true;
      const uint32_t id = idesc_i8_m256(8 * NS);
      int64_t mt = g0 / S.nsub, sb = g0 - mt * S.nsub;
      for (int64_t g = g0; g < g1 && ok; ++g, ++it, sb = sb + 1 == S.nsub ? (++mt, 0) : sb + 1) {
        if (mt != cur) {
          if (nload > 0) mma_commit_pair(a_empty);  // both CTAs' A tiles are free once these MMAs finish
          if (!(ok = mbar_wait(a_full, nload & 1, err))) break;
          if (!(ok = mbar_wait(a_peer, nload & 1, err))) break;
          fence_after();
          cur = (int)mt;
          ++nload;
        }
        const int st = it % kStages;
        const int ab = it & 1;
        if (it >= 2 && !(ok = mbar_wait(acc_empty + ab, ((it >> 1) - 1) & 1, err))) break;
        if (!(ok = mbar_wait(b_full + st, (it / kStages) & 1, err))) break;
        if (!(ok = mbar_wait(b_peer + st, (it / kStages) & 1, err))) break;
        fence_after();
        const uint8_t* bt = sB + st * SH::BH_BYTES;
        const uint32_t dacc = tmem + ab * 256;
        // Plane 0's first K step initialises blocks 0..7; blocks 8..14 were
        // zeroed by the epilogue; every other MMA accumulates.
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int ks = 0; ks < KK / 32; ++ks)
            mma_i8_pair(dacc + i * NS, smem_desc(sA + i * SH::TILE + ks * 256, SH::SBO),
                        smem_desc(bt + ks * 256, SH::SBO), id, (i > 0 || ks > 0) ? 1u : 0u);
        mma_commit_pair(b_empty + st);
        mma_commit_pair(acc_full + ab);
      }
      if (!ok) atomicExch(err, 1);
      mma_commit_pair(mma_done);
      mbar_wait(mma_done, 0, err + 1);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (both CTAs): this CTA's 128 rows -------------
    const int ew = warp - 2;
    const int grp = ew >> 3;
    const int quad = warp & 3;
    const int half = (ew >> 2) & 1;
    const int row = quad * 32 + lane;
    const bool leader = (ew & 7) == 0 && lane == 0;
    const uint32_t lane_base = tmem + ((uint32_t)(quad * 32) << 16) + grp * 256 + half * 8;
    uint64_t* cbuf = sC + grp * (128 * 16);
    uint64_t* c_full = bars + 40 + grp;
    const uint32_t release = crank == 0 ? 0u : cluster_addr(acc_empty + grp, 0);
    const int64_t nsub = S.nsub;
    int64_t g = g0 + grp;
    int64_t mt = g / nsub, sb = g - mt * nsub;
    auto advance = [&]() {
      g += 2;
      sb += 2;
      while (sb >= nsub) {
        sb -= nsub;
        ++mt;
      }
    };
    auto rowbase = [&]() { return (int32_t)(rbeg + mt * 256 + crank * 128); };
    int loads = 0;
    auto tma_load = [&]() {
      mbar_arrive_expect_tx(c_full, 128 * 16 * 8);
      tma_load_2d(cbuf, &cmap, (int32_t)(jend + sb * NS), rowbase(), c_full);
      ++loads;
    };
    if (g < g1 && leader) tma_load();
    bool ok = true;
    for (int k = 0; g < g1; ++k) {
      bool okw = __all_sync(0xffffffffu, mbar_wait(acc_full + grp, k & 1, err));
      uint64_t x[8];
      if (okw) {
        fence_after();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          uint32_t a[15][4];
#pragma unroll
          for (int d = 0; d < 15; ++d) tmem_ld4(lane_base + d * NS + q * 4, a[d]);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 4; ++c) x[4 * q + c] = m61_fold15(a, c);
        }
#pragma unroll
        for (int d = 8; d < 15; ++d) tmem_st8_zero(lane_base + d * NS);
        tmem_wait_st();
        fence_before();
        __syncwarp();
        if (lane == 0) {
          if (crank == 0)
            mbar_arrive(acc_empty + grp);
          else
            mbar_arrive_cluster(release);
        }
      }
      if (okw) okw = __all_sync(0xffffffffu, mbar_wait(c_full, k & 1, err));
      if (okw) {
        uint64_t* rp = cbuf + row * 16;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint64_t* lp = rp + (half * 4 + q) * 2;
          const uint32_t a = smem_u32(lp);
          const int delta = (int)((a ^ (a >> 3)) & 0x70u) - (int)(a & 0x70u);
          ulonglong2* pq = reinterpret_cast<ulonglong2*>(reinterpret_cast<uint8_t*>(lp) + delta);
          const ulonglong2 v = *pq;
          *pq = make_ulonglong2(m61_sub_lazy(v.x, x[2 * q]), m61_sub_lazy(v.y, x[2 * q + 1]));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      if (!group_bar_and(1 + grp, okw)) {
        ok = false;
        break;
      }
      if (leader) {
        tma_store_2d(&cmap, (int32_t)(jend + sb * NS), rowbase(), cbuf);
        bulk_commit();
        bulk_wait_read0();
      }
      advance();
      if (leader && g < g1) tma_load();
    }
    if (leader) {
      bulk_wait_all0();
      if (!ok && loads > 0) mbar_wait(c_full, (loads - 1) & 1, err + 1);
    }
    if (!ok) atomicExch(err, 1);
  }
  fence_before();
  __syncthreads();
  cluster_sync_all();  // no CTA leaves while its peer may still signal it or write its TMEM
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

int limbs_for(uint64_t p) {
  const int bits = 64 - __builtin_clzll(p - 1);
  return bits <= 8 ? 1 : bits <= 16 ? 2 : bits <= 32 ? 4 : 8;
}

template <int LIMBS, int KK>
void split_a_t(const uint64_t* A, int64_t lda, int r0, int rbeg, int rend, int K, uint8_t* Aw, cudaStream_t st,
               const Guard& g) {
  // Padded to 256 rows (zero rows past rend), so CTA pairs find both of a
  // 256-row tile's halves.
  const int mpad = ((rend - rbeg + 255) / 256) * 256;
  const int64_t threads = (int64_t)mpad * Shape<LIMBS, KK>::KC;
  launch_k(split_a_kernel<LIMBS, KK>, dim3((unsigned)((threads + 255) / 256)), dim3(256), 0, st, 1, A, lda,
           (int32_t)r0, (int32_t)rbeg, (int32_t)rend, (int32_t)K, (int32_t)mpad, Aw, g);
}

template <int LIMBS, int KK>
void split_b_t(const uint64_t* B, int64_t ldb, int jend, int cend, int K, uint8_t* Bw, cudaStream_t st,
               const Guard& g) {
  constexpr int NS = Shape<LIMBS, KK>::NS;
  const int npad = ((cend - jend + NS - 1) / NS) * NS;
  const int64_t threads = (int64_t)npad * Shape<LIMBS, KK>::KC;
  launch_k(split_b_kernel<LIMBS, KK>, dim3((unsigned)((threads + 255) / 256)), dim3(256), 0, st, 1, B, ldb,
           (int32_t)jend, (int32_t)cend, (int32_t)K, (int32_t)npad, Bw, g);
}

// Tensor map of C = m[0 .. rend) x [0 .. cend) (row stride ld) for 128 x 16
// boxes of u64 with the 128-byte swizzle; false when the driver entry point
// is unavailable or the encoding fails.
static bool make_c_map(CUtensorMap* map, uint64_t* m, int64_t ld, int rend, int cend) {
  static PFN_cuTensorMapEncodeTiled encode = []() -> PFN_cuTensorMapEncodeTiled {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  }();
  if (!encode) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cend, (cuuint64_t)rend};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
  const cuuint32_t box[2] = {16, 128};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, m, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class F, int LIMBS, int KK>
void update_t(const F& f, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend, const uint8_t* Aw,
              const uint8_t* Bw, int max_ctas, uint64_t r64, int* err, cudaStream_t st, const Guard& g,
              const LimbOut& lo) {
  using SH = Shape<LIMBS, KK>;
  Sched S;
  S.mtiles = (rend - rbeg + 127) / 128;
  S.nsub = (cend - jend + SH::NS - 1) / SH::NS;
  const int64_t total = (int64_t)S.mtiles * S.nsub;
  const int grid = total < max_ctas ? (int)total : max_ctas;  // one CTA per SM: it owns all 512 TMEM columns
  constexpr int smem = std::is_same<F, FpM61>::value ? SH::SMEM_M61 : SH::SMEM;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(trailing_tc_kernel<F, LIMBS, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr = true;
  }
  // C through TMA (p = 2^61 - 1): 16-byte aligned rows and column offset.
  CUtensorMap cmap;
  std::memset(&cmap, 0, sizeof cmap);
  int use_tma = 0;
  if (std::is_same<F, FpM61>::value && !lo.c_zero && (ld & 1) == 0 && ((uintptr_t)m & 15) == 0 && (jend & 1) == 0)
    use_tma = make_c_map(&cmap, m, ld, rend, cend) ? 1 : 0;
  launch_k(trailing_tc_kernel<F, LIMBS, KK>, dim3(grid), dim3(kThreads), smem, st, 1, f, Aw, Bw, m, ld,
           (int32_t)rbeg, (int32_t)rend, (int32_t)jend, (int32_t)cend, S, r64, err, cmap, use_tma, g, lo);
}

// The pair kernel over 2^61 - 1 (C through TMA, so the caller checked the
// alignment and made the tensor map): grid = 2 x the pairs that fit at once.
template <int KK>
cudaError_t update_pair_t(const uint8_t* Aw, const uint8_t* Bw, int rbeg, int rend, int jend, int cend, int max_ctas,
                          int* err, const CUtensorMap& cmap, cudaStream_t st, const Guard& g) {
  using SH = PairShape<KK>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(trailing_tc_pair_kernel<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SH::SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  Sched S;
  S.mtiles = (rend - rbeg + 255) / 256;
  S.nsub = (cend - jend + SH::NS - 1) / SH::NS;
  const int64_t total = (int64_t)S.mtiles * S.nsub;
  int pairs = max_ctas / 2;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = SH::SMEM;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  static int fit = 0;  // clusters of two that can be resident at once
  if (!fit) {
    cfg.gridDim = dim3(2 * pairs);
    int c = 0;
    if (cudaOccupancyMaxActiveClusters(&c, trailing_tc_pair_kernel<KK>, &cfg) != cudaSuccess || c < 1) {
      cudaGetLastError();
      c = 1;
    }
    fit = c;
  }
  if (pairs > fit) pairs = fit;
  if (total < pairs) pairs = (int)total;
  if (pairs < 1) pairs = 1;
  return launch_k(trailing_tc_pair_kernel<KK>, dim3(2 * pairs), dim3(kThreads), SH::SMEM, st, 2, Aw, Bw,
                  (int32_t)rbeg, (int32_t)jend, S, err, cmap, g);
}

// (limb count, K tile) of a prime and an update depth.
inline int limbs_of(uint64_t p) { return p == kM61 ? 8 : limbs_for(p); }

}  // namespace tc

int tc_crossover_n(uint64_t) { return 512; }

// Whether updates over 2^61 - 1 run on CTA pairs (modlin_set_tc_pairs; off
// by default: measured 1.5 % slower than single CTAs in the 16384^2 rank).
bool g_tc_pairs = false;

// Calls OP(limbs, K tile) for fp.p and K, both compile-time constants.
#define MODLIN_TC_DISPATCH(OP)                      \
  do {                                              \
    const bool k128 = K > 64;                       \
    switch (tc::limbs_of(fp.p)) {                   \
      case 1: k128 ? OP(1, 128) : OP(1, 64); break; \
      case 2: k128 ? OP(2, 128) : OP(2, 64); break; \
      case 4: k128 ? OP(4, 128) : OP(4, 64); break; \
      default: k128 ? OP(8, 128) : OP(8, 64); break; \
    }                                               \
  } while (0)

size_t tc_a_bytes(int rows) { return (size_t)((rows + 127) / 128 + 1) * 128 * tc::kKMax * 8; }
size_t tc_b_bytes(int cols) { return (size_t)((cols + 127) / 128 + 1) * 128 * tc::kKMax * 8; }

cudaError_t tc_split_a(const FieldParams& fp, const uint64_t* A, int64_t lda, int r0, int rbeg, int rend, int K,
                       uint8_t* Aw, cudaStream_t st, const Guard& g) {
  if (rbeg >= rend) return cudaSuccess;
  if (K <= 0 || K > tc::kKMax) return cudaErrorInvalidValue;
#define MODLIN_SPLIT_A(LL, KK) tc::split_a_t<LL, KK>(A, lda, r0, rbeg, rend, K, Aw, st, g)
  MODLIN_TC_DISPATCH(MODLIN_SPLIT_A);
#undef MODLIN_SPLIT_A
  return cudaGetLastError();
}

cudaError_t tc_split_b(const FieldParams& fp, const uint64_t* B, int64_t ldb, int jend, int cend, int K, uint8_t* Bw,
                       cudaStream_t st, const Guard& g) {
  if (jend >= cend) return cudaSuccess;
  if (K <= 0 || K > tc::kKMax) return cudaErrorInvalidValue;
#define MODLIN_SPLIT_B(LL, KK) tc::split_b_t<LL, KK>(B, ldb, jend, cend, K, Bw, st, g)
  MODLIN_TC_DISPATCH(MODLIN_SPLIT_B);
#undef MODLIN_SPLIT_B
  return cudaGetLastError();
}

cudaError_t tc_update(const FieldParams& fp, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend, int K,
                      const uint8_t* Aw, const uint8_t* Bw, int max_ctas, int* err, cudaStream_t st,
                      const Guard& g, const LimbOut& lo) {
  if (rbeg >= rend || jend >= cend) return cudaSuccess;
  if (lo.Aw && (fp.p != kM61 || (lo.kk != 64 && lo.kk != 128))) return cudaErrorInvalidValue;
  if (K <= 0 || K > tc::kKMax) return cudaErrorInvalidValue;
  const uint64_t r64 = (uint64_t)(((u128)1 << 64) % fp.p);
  if (fp.p == kM61) {
    // CTA pairs when C can move by TMA and there are rows for both halves.
    CUtensorMap cmap;
    if (g_tc_pairs && !lo.Aw && rend - rbeg > 128 && max_ctas >= 2 && (ld & 1) == 0 && ((uintptr_t)m & 15) == 0 &&
        (jend & 1) == 0 && tc::make_c_map(&cmap, m, ld, rend, cend))
      return K > 64 ? tc::update_pair_t<128>(Aw, Bw, rbeg, rend, jend, cend, max_ctas, err, cmap, st, g)
                    : tc::update_pair_t<64>(Aw, Bw, rbeg, rend, jend, cend, max_ctas, err, cmap, st, g);
    if (K > 64)
      tc::update_t<FpM61, 8, 128>(FpM61(fp), m, ld, rbeg, rend, jend, cend, Aw, Bw, max_ctas, r64, err, st, g, lo);
    else
      tc::update_t<FpM61, 8, 64>(FpM61(fp), m, ld, rbeg, rend, jend, cend, Aw, Bw, max_ctas, r64, err, st, g, lo);
    return cudaGetLastError();
  }
  const FpBarrett f(fp);
#define MODLIN_UPDATE(LL, KK) \
  tc::update_t<FpBarrett, LL, KK>(f, m, ld, rbeg, rend, jend, cend, Aw, Bw, max_ctas, r64, err, st, g, lo)
  MODLIN_TC_DISPATCH(MODLIN_UPDATE);
#undef MODLIN_UPDATE
  return cudaGetLastError();
}

cudaError_t launch_trailing_tc(const FieldParams& fp, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend,
                               const uint64_t* Lbuf, int64_t lda, int r0, const uint64_t* Ubuf, int64_t ldU, int K,
                               uint8_t* Aw, uint8_t* Bw, int num_sms, int* err, cudaStream_t st, const Guard& g) {
  if (rbeg >= rend || jend >= cend || K <= 0) return cudaSuccess;
  if (K > tc::kKMax) return cudaErrorInvalidValue;
  cudaError_t e = tc_split_a(fp, Lbuf, lda, r0, rbeg, rend, K, Aw, st, g);
  if (e == cudaSuccess) e = tc_split_b(fp, Ubuf, ldU, jend, cend, K, Bw, st, g);
  if (e == cudaSuccess) e = tc_update(fp, m, ld, rbeg, rend, jend, cend, K, Aw, Bw, num_sms, err, st, g);
  return e;
}

}  // namespace modlin
