// Device fill of the generators under test.
//
// MIXMAX (src/prng.rs:133-270, ROOT's MixMaxEngine) is linear over
// F_p, p = 2^61 - 1: one iteration maps the state (sumtot, v[1..N-1]) by a
// fixed N x N matrix, so the state any number of iterations ahead is a matrix
// power times the starting state (the host builds the matrix; powers come
// from m61_gemm). Each warp then runs one segment of the stream from its
// jump-ahead state. Within an iteration the two running sums of ROOT's loop
// (tp = v[1] + ... + v[i], tv = sumtot + tp_1 + ... + tp_i, plus the
// rotated-tp term when SPECIALMUL != 0) are two prefix scans over the state,
// 8 entries per lane and five shuffle steps across the warp.
//
// Bit parity with ROOT's arithmetic: ROOT folds each sum once
// (MOD_MERSENNE), which is exact mod p but can leave 2^61 - 1 where the
// canonical residue is 0, and that representation reaches the outputs
// (raw << 3). Every folded sum is below 3 * 2^61, so its result is at most
// 2^61 - 1 and equals it only when the sum is = 0 (mod p). Hence if no
// intermediate of an iteration (tp_i, tv_i, the special term, the corrected
// v[2]) is = 0 and no input entry is 2^61 - 1, ROOT's values are the
// canonical residues the scans compute; sumtot is ROOT's own formula on the
// exact 128-bit sum. Any other iteration is run by lane 0 exactly as ROOT
// runs it. A segment that ends on an entry 2^61 - 1 flags the next one, whose
// canonical jump-ahead start may then differ from ROOT's state in
// representation; the host reruns it from the flagged segment's exact end.
//
// xoroshiro128++ (src/prng.rs:48-83): the state transition is linear over
// GF(2) (the host computes the jump-ahead states); one thread per segment,
// outputs staged 32 per thread in shared memory and written row by row.
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"
#include "prng_kernels.cuh"

namespace modlin {

namespace {

constexpr uint64_t kP = kM61;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint64_t padd(uint64_t a, uint64_t b) {
  const uint64_t s = a + b;
  return s >= kP ? s - kP : s;
}
__device__ __forceinline__ uint64_t fold61(uint64_t k) { return (k & kP) + (k >> 61); }
__device__ __forceinline__ uint64_t rot61(uint64_t x, int s) { return ((x << s) & kP) | (x >> (61 - s)); }

// ---- reductions of outputs to the field ------------------------------------
struct RedRaw {
  __device__ __forceinline__ uint64_t operator()(uint64_t x) const { return x; }
};
struct RedM61 {
  __device__ __forceinline__ uint64_t operator()(uint64_t x) const {
    const uint64_t y = fold61(x);
    return y >= kP ? y - kP : y;
  }
};
struct RedBarrett {
  FpBarrett f;
  __device__ __forceinline__ uint64_t operator()(uint64_t x) const { return f.reduce((u128)x); }
};
struct RedSmall {
  FpSmall f;
  __device__ __forceinline__ uint64_t operator()(uint64_t x) const { return f.reduce64(x); }
};

// ---- C = A * B mod 2^61 - 1 ------------------------------------------------
constexpr int kGT = 32;  // output tile kGT x kGT, 256 threads, 4 outputs each

__global__ void __launch_bounds__(256) m61_gemm_kernel(const uint64_t* __restrict__ A, const uint64_t* __restrict__ B,
                                                       uint64_t* __restrict__ C, int M, int K, int N) {
  __shared__ uint64_t As[kGT][kGT + 1], Bs[kGT][kGT + 1];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // ty 0..7
  const int r0 = blockIdx.y * kGT, c0 = blockIdx.x * kGT;
  u128 acc[4] = {0, 0, 0, 0};
  for (int k0 = 0; k0 < K; k0 += kGT) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ty + 8 * q;
      As[r][tx] = (r0 + r < M && k0 + tx < K) ? A[(int64_t)(r0 + r) * K + k0 + tx] : 0;
      Bs[r][tx] = (k0 + r < K && c0 + tx < N) ? B[(int64_t)(k0 + r) * N + c0 + tx] : 0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kGT; ++kk) {
      const uint64_t b = Bs[kk][tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const u128 t = (u128)As[ty + 8 * q][kk] * b;  // < 2^122
        const uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
        acc[q] += (lo & kP) + ((lo >> 61) | (hi << 3));  // < 2^62 each, K of them < 2^126
      }
    }
    __syncthreads();
  }
  const FpM61 f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = r0 + ty + 8 * q;
    if (r < M && c0 + tx < N) C[(int64_t)r * N + c0 + tx] = f.reduce(acc[q]);
  }
}

// ---- MIXMAX ---------------------------------------------------------------------
template <int N>
struct MixTraits;
template <>
struct MixTraits<17> {  // TRandomMixMax17: SPECIALMUL 36, no special term, no skip
  static constexpr int E = 1, SM = 36, SKIP = 0, SK = 0;
};
template <>
struct MixTraits<240> {  // TRandomMixMax: SPECIALMUL 51, special * v[1], no skip
  static constexpr int E = 8, SM = 51, SKIP = 0, SK = 2;
};
template <>
struct MixTraits<256> {  // TRandomMixMax256: no SPECIALMUL, special -1, skip 2
  static constexpr int E = 8, SM = 0, SKIP = 2, SK = 1;
};

constexpr int kMixWarps = 4;

// Inclusive prefix sum mod p across the warp, returned exclusive.
__device__ __forceinline__ uint64_t warp_excl_scan(uint64_t v, int lane) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, v, off);
    if (lane >= off) v = padd(v, y);
  }
  const uint64_t ex = __shfl_up_sync(kFull, v, 1);
  return lane ? ex : 0;
}

// ROOT's iteration, run by one thread on the state s[0] = sumtot,
// s[1..N-1] = v[1..N-1] (src/prng.rs:191-222).
template <int N>
__device__ void mix_iterate_exact(uint64_t* s, uint64_t special) {
  using T = MixTraits<N>;
  const uint64_t temp2 = s[1];
  uint64_t tv = s[0], acc = tv, ovf = 0, tp = 0;
  for (int i = 1; i < N; ++i) {
    if (T::SM) {
      const uint64_t tpo = ((tp << T::SM) & kP) | (tp >> (61 - T::SM));
      tp = fold61(tp + s[i]);
      tv = fold61(tv + tp + tpo);
    } else {
      tp = fold61(tp + s[i]);
      tv = fold61(tv + tp);
    }
    s[i] = tv;
    const uint64_t t = acc + tv;
    ovf += t < acc;
    acc = t;
  }
  if (T::SK) {
    uint64_t t2;
    if (T::SK == 1) {
      t2 = kP - temp2;
    } else {
      const u128 m = (u128)special * temp2;
      const uint64_t lo = (uint64_t)m, hi = (uint64_t)(m >> 64);
      t2 = fold61((lo & kP) + hi * 8 + (lo >> 61));
    }
    s[2] = fold61(s[2] + t2);
    const uint64_t t = acc + t2;
    ovf += t < acc;
    acc = t;
  }
  s[0] = fold61(fold61(acc) + (ovf << 3));
}

// One iteration of the warp's state x (entry idx = lane * E + k).
template <int N>
__device__ __forceinline__ void mix_iterate(uint64_t (&x)[MixTraits<N>::E], uint64_t& v0, uint64_t* s, int lane,
                                            uint64_t special) {
  using T = MixTraits<N>;
  constexpr int E = T::E;
  bool bad = false;
#pragma unroll
  for (int k = 0; k < E; ++k) bad |= x[k] == kP;
  const uint64_t sum_old = __shfl_sync(kFull, x[0], 0);
  const uint64_t temp2 = __shfl_sync(kFull, x[1 % E], 1 / E);
  // tp_i = v[1] + ... + v[i]
  uint64_t tp[E];
  uint64_t run = 0;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int idx = lane * E + k;
    run = padd(run, (idx >= 1 && idx < N) ? x[k] : 0);
    tp[k] = run;
  }
  const uint64_t ex1 = warp_excl_scan(run, lane);
  // u_0 = sumtot, u_i = tp_i (+ 2^SM tp_{i-1}); tv_i = u_0 + ... + u_i
  uint64_t tv[E];
  uint64_t prev = ex1;
  run = 0;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int idx = lane * E + k;
    const uint64_t t = padd(tp[k], ex1);
    uint64_t u = 0;
    if (idx == 0) {
      u = sum_old;
    } else if (idx < N) {
      bad |= t == 0;
      u = T::SM ? padd(t, rot61(prev, T::SM)) : t;
    }
    prev = t;
    run = padd(run, u);
    tv[k] = run;
  }
  const uint64_t ex2 = warp_excl_scan(run, lane);
  uint64_t t2 = 0;
  if (T::SK == 1) {
    t2 = temp2 ? kP - temp2 : 0;
    bad |= temp2 == 0;
  } else if (T::SK == 2) {
    t2 = FpM61().mul(special, temp2);
    bad |= t2 == 0;
  }
  uint64_t lo = 0, hi = 0;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int idx = lane * E + k;
    tv[k] = padd(tv[k], ex2);
    if (idx < N) {
      if (idx >= 1) bad |= tv[k] == 0;
      lo += tv[k];
      hi += lo < tv[k];
    }
  }
  if (lane == 0) {
    lo += t2;
    hi += lo < t2;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const uint64_t olo = __shfl_xor_sync(kFull, lo, off), ohi = __shfl_xor_sync(kFull, hi, off);
    const uint64_t l2 = lo + olo;
    hi += ohi + (l2 < lo);
    lo = l2;
  }
  if (T::SK) {
#pragma unroll
    for (int k = 0; k < E; ++k)
      if (lane * E + k == 2) {
        tv[k] = padd(tv[k], t2);
        bad |= tv[k] == 0;
      }
  }
  if (!__any_sync(kFull, bad)) {
    const uint64_t sumtot = fold61(fold61(lo) + (hi << 3));
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const int idx = lane * E + k;
      x[k] = idx == 0 ? sumtot : (idx < N ? tv[k] : 0);
    }
  } else {
#pragma unroll
    for (int k = 0; k < E; ++k)
      if (lane * E + k < N) s[lane * E + k] = x[k];
    __syncwarp();
    if (lane == 0) mix_iterate_exact<N>(s, special);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < E; ++k) x[k] = lane * E + k < N ? s[lane * E + k] : 0;
    __syncwarp();
  }
  v0 = sum_old;
}

template <int N, class R>
__global__ void __launch_bounds__(kMixWarps * 32) mixmax_fill_kernel(MixFill a, R red) {
  using T = MixTraits<N>;
  constexpr int E = T::E;
  __shared__ uint64_t sh[kMixWarps][N];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t seg = a.seg_begin + (int64_t)blockIdx.x * kMixWarps + w;
  if (seg >= a.seg_end) return;
  uint64_t* s = sh[w];
  uint64_t x[E];
  const uint64_t* st = a.starts + seg * N;
#pragma unroll
  for (int k = 0; k < E; ++k) x[k] = lane * E + k < N ? st[lane * E + k] : 0;
  uint64_t v0 = 0;
  if (seg == 0 && a.h0 > 0) {  // the rest of the starting block
#pragma unroll
    for (int k = 0; k < E; ++k)
      if (lane * E + k < N) s[lane * E + k] = x[k];
    __syncwarp();
    for (int64_t j = lane; j < a.h0; j += 32) a.out[j] = red(s[a.c0 + j] << 3);
    __syncwarp();
  }
  const int64_t b0 = seg * a.G + 1, b1 = (seg + 1) * a.G < a.nbk ? (seg + 1) * a.G : a.nbk;
  for (int64_t b = b0; b <= b1; ++b) {
#pragma unroll 1
    for (int it = 0; it <= T::SKIP; ++it) mix_iterate<N>(x, v0, s, lane, a.special);
#pragma unroll
    for (int k = 0; k < E; ++k)
      if (lane * E + k < N) s[lane * E + k] = x[k];
    __syncwarp();
    const int64_t base = a.h0 + (b - 1) * (N - 1) - 1;  // output index of v[e] is base + e
    if (base + N <= a.count) {
      for (int e = lane; e < N; e += 32)
        if (e >= 1) a.out[base + e] = red(s[e] << 3);
    } else {
      for (int e = lane; e < N; e += 32)
        if (e >= 1 && base + e < a.count) a.out[base + e] = red(s[e] << 3);
    }
    __syncwarp();
  }
  uint64_t* en = a.ends + seg * (N + 1);
  bool kmp = false;
#pragma unroll
  for (int k = 0; k < E; ++k)
    if (lane * E + k < N) {
      en[lane * E + k] = x[k];
      kmp |= x[k] == kP;
    }
  if (lane == 0) en[N] = v0;
  if (__any_sync(kFull, kmp) && lane == 0 && seg + 1 < a.S) {
    a.flags[seg + 1] = 1;
    atomicAdd(a.any, 1);
  }
}

template <int N, class R>
cudaError_t launch_mix(const MixFill& a, R red, cudaStream_t st) {
  const int64_t segs = a.seg_end - a.seg_begin;
  if (segs <= 0) return cudaSuccess;
  const int64_t blocks = (segs + kMixWarps - 1) / kMixWarps;
  mixmax_fill_kernel<N, R><<<(unsigned)blocks, kMixWarps * 32, 0, st>>>(a, red);
  return cudaGetLastError();
}

template <int N>
cudaError_t mix_dispatch(const MixFill& a, uint64_t p, const FieldParams& fp, cudaStream_t st) {
  if (p == 0) return launch_mix<N>(a, RedRaw{}, st);
  if (p == kM61) return launch_mix<N>(a, RedM61{}, st);
  if (p < (1ULL << 32)) return launch_mix<N>(a, RedSmall{FpSmall(fp)}, st);
  return launch_mix<N>(a, RedBarrett{FpBarrett(fp)}, st);
}

// ---- xoroshiro128++ ----------------------------------------------------------------
constexpr int kXoroWarps = 4;

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

template <class R>
__global__ void __launch_bounds__(kXoroWarps * 32) xoro_fill_kernel(XoroFill a, R red) {
  __shared__ uint64_t sh[kXoroWarps][32][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, t0 = t - lane;
  if (t0 >= a.S) return;
  const bool act = t < a.S;
  uint64_t s0 = 0, s1 = 0;
  if (act) {
    s0 = a.starts[2 * t];
    s1 = a.starts[2 * t + 1];
  }
  const int64_t beg = t * a.L, cnt = act ? ((a.count - beg) < a.L ? (a.count - beg) : a.L) : 0;
  const int64_t nch = (a.L + 31) / 32;
  for (int64_t c = 0; c < nch; ++c) {
#pragma unroll 4
    for (int i = 0; i < 32; ++i) {
      if (c * 32 + i < cnt) {  // src/prng.rs:75-83
        const uint64_t r = rotl64(s0 + s1, 17) + s0;
        const uint64_t b = s1 ^ s0;
        s0 = rotl64(s0, 49) ^ b ^ (b << 21);
        s1 = rotl64(b, 28);
        sh[w][lane][i] = red(r);
      }
    }
    __syncwarp();
    for (int r = 0; r < 32; ++r) {
      const int64_t tr = t0 + r;
      if (tr >= a.S) break;
      const int64_t rb = tr * a.L, rc = (a.count - rb) < a.L ? (a.count - rb) : a.L;
      const int64_t off = c * 32 + lane;
      if (off < rc) a.out[rb + off] = sh[w][r][lane];
    }
    __syncwarp();
  }
  if (t == a.S - 1) {
    a.ends[0] = s0;
    a.ends[1] = s1;
  }
}

template <class R>
cudaError_t launch_xoro(const XoroFill& a, R red, cudaStream_t st) {
  if (a.S <= 0) return cudaSuccess;
  const int64_t threads = kXoroWarps * 32;
  xoro_fill_kernel<R><<<(unsigned)((a.S + threads - 1) / threads), (unsigned)threads, 0, st>>>(a, red);
  return cudaGetLastError();
}

}  // namespace

cudaError_t m61_gemm(const uint64_t* A, const uint64_t* B, uint64_t* C, int M, int K, int N, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
  const dim3 grid((N + kGT - 1) / kGT, (M + kGT - 1) / kGT);
  m61_gemm_kernel<<<grid, 256, 0, st>>>(A, B, C, M, K, N);
  return cudaGetLastError();
}

cudaError_t mixmax_fill(const MixFill& a, uint64_t p, const FieldParams& fp, cudaStream_t st) {
  switch (a.N) {
    case 17: return mix_dispatch<17>(a, p, fp, st);
    case 240: return mix_dispatch<240>(a, p, fp, st);
    case 256: return mix_dispatch<256>(a, p, fp, st);
    default: return cudaErrorInvalidValue;
  }
}

int mixmax_resident_warps(int N, int num_sms) {
  int per_sm = 0;
  cudaError_t e = cudaErrorInvalidValue;
  if (N == 17) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixmax_fill_kernel<17, RedM61>, kMixWarps * 32, 0);
  if (N == 240) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixmax_fill_kernel<240, RedM61>, kMixWarps * 32, 0);
  if (N == 256) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixmax_fill_kernel<256, RedM61>, kMixWarps * 32, 0);
  if (e != cudaSuccess || per_sm < 1) per_sm = 1;
  return per_sm * kMixWarps * num_sms;
}

cudaError_t xoro_fill(const XoroFill& a, uint64_t p, const FieldParams& fp, cudaStream_t st) {
  if (p == 0) return launch_xoro(a, RedRaw{}, st);
  if (p == kM61) return launch_xoro(a, RedM61{}, st);
  if (p < (1ULL << 32)) return launch_xoro(a, RedSmall{FpSmall(fp)}, st);
  return launch_xoro(a, RedBarrett{FpBarrett(fp)}, st);
}

}  // namespace modlin

// ---------------------------------------------------------------------------
// Host side: jump-ahead states, launches, the boundary repair, write-back.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <vector>

#include "../host/prng.h"

namespace modlin {

namespace {

constexpr int kPowMax = 64;

uint64_t hmul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % kM61); }
uint64_t hadd(uint64_t a, uint64_t b) { return (a + b) % kM61; }

// One MIXMAX iteration as the linear map it is over F_p (canonical
// residues): the state x = [sumtot, v[1..N-1]] (src/prng.rs:191-222).
void mix_linear_step(const modlin_prng_impl::MixMax& m, const uint64_t* x, uint64_t* y) {
  const int N = m.N;
  const uint64_t sum_old = x[0], temp2 = x[1];
  const uint64_t two_sm = m.specialmul ? (1ULL << m.specialmul) % kM61 : 0;
  uint64_t tp = 0, tv = sum_old, tot = sum_old;
  for (int i = 1; i < N; ++i) {
    const uint64_t tpo = m.specialmul ? hmul(tp, two_sm) : 0;
    tp = hadd(tp, x[i]);
    tv = hadd(hadd(tv, tp), tpo);
    y[i] = tv;
    tot = hadd(tot, tv);
  }
  if (m.special) {
    const uint64_t t2 = m.special == UINT64_MAX ? (kM61 - temp2) % kM61 : hmul(m.special % kM61, temp2);
    y[2] = hadd(y[2], t2);
    tot = hadd(tot, t2);
  }
  y[0] = tot;
}

int kind_slot(int N) { return N == 17 ? 0 : N == 240 ? 1 : 2; }

#define PCK(x)                                                        \
  do {                                                                \
    cudaError_t e_ = (x);                                             \
    if (e_ != cudaSuccess) {                                          \
      cudaGetLastError();                                             \
      return e_ == cudaErrorMemoryAllocation ? MODLIN_ENOMEM : MODLIN_ECUDA; \
    }                                                                 \
  } while (0)

int ensure_ws(PrngCache& c, size_t bytes) {
  if (bytes <= c.ws_bytes) return MODLIN_OK;
  if (c.ws) cudaFree(c.ws);
  c.ws = nullptr;
  c.ws_bytes = 0;
  PCK(cudaMalloc(&c.ws, bytes));
  c.ws_bytes = bytes;
  return MODLIN_OK;
}

// B^(2^k) for k <= kmax in the cache (B built on the host, squared here).
int ensure_pows(PrngCache& c, const modlin_prng_impl::MixMax& m, int kmax, cudaStream_t st, uint64_t* launches) {
  const int slot = kind_slot(m.N), N = m.N;
  const size_t mat = (size_t)N * N;
  if (!c.pow[slot]) {
    PCK(cudaMalloc(&c.pow[slot], mat * kPowMax * sizeof(uint64_t)));
    std::vector<uint64_t> Q(mat), x(N), y(N);
    for (int j = 0; j < N; ++j) {  // row j = B e_j
      std::fill(x.begin(), x.end(), 0);
      x[j] = 1;
      for (int it = 0; it <= m.skip; ++it) {
        mix_linear_step(m, x.data(), y.data());
        x.swap(y);
      }
      std::copy(x.begin(), x.end(), Q.begin() + (size_t)j * N);
    }
    PCK(cudaMemcpyAsync(c.pow[slot], Q.data(), mat * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    PCK(cudaStreamSynchronize(st));
    c.have[slot] = 1;
  }
  for (int k = c.have[slot]; k <= kmax; ++k) {
    const uint64_t* P = c.pow[slot] + (size_t)(k - 1) * mat;
    PCK(m61_gemm(P, P, c.pow[slot] + (size_t)k * mat, N, N, N, st));
    ++*launches;
    c.have[slot] = k + 1;
  }
  return MODLIN_OK;
}

int mix_fill(PrngCache& c, int num_sms, modlin_prng_impl::MixMax& m, uint64_t p, const FieldParams& fp,
             uint64_t* d_out, uint64_t count, cudaStream_t st, uint64_t* launches) {
  const int N = m.N;
  const size_t mat = (size_t)N * N;
  const int64_t c0 = m.counter;
  const int64_t h0 = c0 < N ? std::min<int64_t>(N - c0, (int64_t)count) : 0;
  const int64_t rest = (int64_t)count - h0;
  const int64_t nbk = rest > 0 ? (rest + N - 2) / (N - 1) : 0;
  int64_t S = 1, G = 1;
  if (nbk > 0) {
    const int64_t R = mixmax_resident_warps(N, num_sms);
    G = (nbk + std::min<int64_t>(nbk, R) - 1) / std::min<int64_t>(nbk, R);
    S = (nbk + G - 1) / G;
  }
  // workspace: starts S x N | ends S x (N+1) | 3 matrices | flags S + 1 ints
  const size_t o_ends = (size_t)S * N, o_mat = o_ends + (size_t)S * (N + 1), o_flags = o_mat + 3 * mat;
  int rc = ensure_ws(c, (o_flags + 1) * sizeof(uint64_t) + (size_t)(S + 1) * sizeof(int));
  if (rc) return rc;
  uint64_t* ws = static_cast<uint64_t*>(c.ws);
  uint64_t *starts = ws, *ends = ws + o_ends, *J = ws + o_mat, *Jt = J + mat, *Jn = Jt + mat;
  int* flags = reinterpret_cast<int*>(ws + o_flags);
  int* any = flags + S;

  // The exact host state; its canonical form seeds the jump-ahead.
  std::vector<uint64_t> x0(N);
  x0[0] = m.sumtot;
  for (int i = 1; i < N; ++i) x0[i] = m.v[i];
  if (S > 1) {
    int bits = 0;
    while ((G >> bits) > 1) ++bits;  // floor(log2 G)
    rc = ensure_pows(c, m, bits, st, launches);
    if (rc) return rc;
    // J = B^G from the cached powers (they commute).
    bool first = true;
    for (int k = 0; k <= bits; ++k) {
      if (!((G >> k) & 1)) continue;
      const uint64_t* P = c.pow[kind_slot(N)] + (size_t)k * mat;
      if (first) {
        PCK(cudaMemcpyAsync(J, P, mat * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
        first = false;
      } else {
        PCK(m61_gemm(J, P, Jn, N, N, N, st));
        ++*launches;
        std::swap(J, Jn);
      }
    }
    std::vector<uint64_t> xc(x0);
    for (auto& v : xc) v %= kM61;
    PCK(cudaMemcpyAsync(starts, xc.data(), N * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    // Doubling: states [have, 2 have) = states [0, have) * B^(G have).
    for (int64_t have = 1; have < S;) {
      const int64_t w = std::min(have, S - have);
      PCK(m61_gemm(starts, J, starts + (size_t)have * N, (int)w, N, N, st));
      ++*launches;
      have += w;
      if (have < S) {
        PCK(m61_gemm(J, J, Jt, N, N, N, st));
        ++*launches;
        std::swap(J, Jt);
      }
    }
  }
  PCK(cudaMemcpyAsync(starts, x0.data(), N * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  PCK(cudaMemsetAsync(flags, 0, (size_t)(S + 1) * sizeof(int), st));
  MixFill a{};
  a.N = N;
  a.special = m.special == UINT64_MAX ? 0 : m.special;
  a.starts = starts;
  a.ends = ends;
  a.flags = flags;
  a.any = any;
  a.out = d_out;
  a.count = (int64_t)count;
  a.h0 = h0;
  a.nbk = nbk;
  a.G = G;
  a.S = S;
  a.c0 = (int)c0;
  a.seg_begin = 0;
  a.seg_end = S;
  PCK(mixmax_fill(a, p, fp, st));
  ++*launches;
  int h_any = 0;
  PCK(cudaMemcpyAsync(&h_any, any, sizeof(int), cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  if (h_any) {
    // A segment ended on an entry 2^61 - 1: rerun the next one from that
    // exact end (its canonical start differs in representation), in order.
    std::vector<int> hf(S);
    PCK(cudaMemcpyAsync(hf.data(), flags, S * sizeof(int), cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    for (int64_t s = 1; s < S; ++s) {
      if (!hf[s]) continue;
      PCK(cudaMemcpyAsync(starts + (size_t)s * N, ends + (size_t)(s - 1) * (N + 1), N * sizeof(uint64_t),
                          cudaMemcpyDeviceToDevice, st));
      if (s + 1 < S) PCK(cudaMemsetAsync(flags + s + 1, 0, sizeof(int), st));
      a.seg_begin = s;
      a.seg_end = s + 1;
      PCK(mixmax_fill(a, p, fp, st));
      ++*launches;
      if (s + 1 < S) {
        PCK(cudaMemcpyAsync(&hf[s + 1], flags + s + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        PCK(cudaStreamSynchronize(st));
      }
    }
  }
  if (nbk == 0) {
    PCK(cudaStreamSynchronize(st));
    m.counter = (int)(c0 + (int64_t)count);
    return MODLIN_OK;
  }
  std::vector<uint64_t> e(N + 1);
  PCK(cudaMemcpyAsync(e.data(), ends + (size_t)(S - 1) * (N + 1), (N + 1) * sizeof(uint64_t),
                      cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  m.sumtot = e[0];
  for (int i = 1; i < N; ++i) m.v[i] = e[i];
  m.v[0] = e[N];
  m.counter = (int)((rest - 1) % (N - 1) + 2);  // one past the last element output
  return MODLIN_OK;
}

// GF(2) 128 x 128 matrices over the xoroshiro state (s0 = bits 0..63,
// s1 = bits 64..127), stored by columns.
struct V128 {
  uint64_t lo, hi;
};
struct M128 {
  V128 col[128];
};

V128 gf2_apply(const M128& A, V128 v) {
  V128 r{0, 0};
  for (int j = 0; j < 64; ++j)
    if ((v.lo >> j) & 1) {
      r.lo ^= A.col[j].lo;
      r.hi ^= A.col[j].hi;
    }
  for (int j = 0; j < 64; ++j)
    if ((v.hi >> j) & 1) {
      r.lo ^= A.col[64 + j].lo;
      r.hi ^= A.col[64 + j].hi;
    }
  return r;
}
void gf2_mul(const M128& A, const M128& B, M128* C) {  // C = A B
  for (int j = 0; j < 128; ++j) C->col[j] = gf2_apply(A, B.col[j]);
}

int xoro_fill_host(PrngCache& c, int num_sms, modlin_prng_impl::Xoroshiro& x, uint64_t p, const FieldParams& fp,
                   uint64_t* d_out, uint64_t count, cudaStream_t st, uint64_t* launches) {
  int64_t S = std::min<int64_t>(((int64_t)count + 63) / 64, (int64_t)num_sms * 256);
  if (S < 1) S = 1;
  const int64_t L = ((int64_t)count + S - 1) / S;
  S = ((int64_t)count + L - 1) / L;
  // T: one step; J = T^L.
  M128 T, J, P, tmp;
  for (int j = 0; j < 128; ++j) {
    modlin_prng_impl::Xoroshiro u;
    u.s0 = j < 64 ? 1ULL << j : 0;
    u.s1 = j < 64 ? 0 : 1ULL << (j - 64);
    u.step();
    T.col[j] = V128{u.s0, u.s1};
  }
  P = T;
  bool have = false;
  for (int64_t e = L; e; e >>= 1) {
    if (e & 1) {
      if (!have) {
        J = P;
        have = true;
      } else {
        gf2_mul(J, P, &tmp);
        J = tmp;
      }
    }
    if (e > 1) {
      gf2_mul(P, P, &tmp);
      P = tmp;
    }
  }
  std::vector<uint64_t> starts(2 * S);
  V128 v{x.s0, x.s1};
  for (int64_t t = 0; t < S; ++t) {
    starts[2 * t] = v.lo;
    starts[2 * t + 1] = v.hi;
    if (t + 1 < S) v = gf2_apply(J, v);
  }
  const int rc = ensure_ws(c, (2 * S + 2) * sizeof(uint64_t));
  if (rc) return rc;
  uint64_t* ws = static_cast<uint64_t*>(c.ws);
  PCK(cudaMemcpyAsync(ws, starts.data(), 2 * S * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  XoroFill a{ws, ws + 2 * S, d_out, (int64_t)count, L, S};
  PCK(xoro_fill(a, p, fp, st));
  ++*launches;
  uint64_t e[2];
  PCK(cudaMemcpyAsync(e, ws + 2 * S, sizeof(e), cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  x.s0 = e[0];
  x.s1 = e[1];
  return MODLIN_OK;
}

}  // namespace

int prng_fill_device(PrngCache& c, int num_sms, modlin_prng* g, uint64_t p, const FieldParams& fp, uint64_t* d_out,
                     uint64_t count, cudaStream_t st, uint64_t* launches) {
  if (!count) return MODLIN_OK;
  if (g->xo) return xoro_fill_host(c, num_sms, *g->xo, p, fp, d_out, count, st, launches);
  if (g->mm) return mix_fill(c, num_sms, *g->mm, p, fp, d_out, count, st, launches);
  return MODLIN_EINVAL_ARG;
}

}  // namespace modlin
