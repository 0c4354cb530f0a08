// Synthetic-workload generation on the device.
//
// Uniform residues: output k is the k-th accepted draw of the SplitMix64
// stream (src/prng.rs:61-67) whose state starts at `seed`; a draw x is
// accepted when x >> (64 - bitlen(p-1)) < p. Draw i only depends on
// seed + (i+1) * golden, so draws are generated in parallel and the accepted
// ones compacted in order (per-block counts, one scan, ordered scatter) —
// bit-identical to the sequential host stream.
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"
#include "gen_kernels.cuh"

namespace modlin {

constexpr int kGenThreads = 256;
constexpr int kGenPerThread = 16;
constexpr int kGenPerBlock = kGenThreads * kGenPerThread;

__device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i) {
  uint64_t w = seed + (i + 1) * 0x9e3779b97f4a7c15ULL;
  w = (w ^ (w >> 30)) * 0xbf58476d1ce4e5b9ULL;
  w = (w ^ (w >> 27)) * 0x94d049bb133111ebULL;
  return w ^ (w >> 31);
}

__global__ void gen_count_kernel(uint64_t p, int bits, uint64_t seed, uint64_t draw0, uint64_t ndraw,
                                 uint32_t* counts) {
  __shared__ uint32_t wsum[kGenThreads / 32];
  const uint64_t base = draw0 + (uint64_t)blockIdx.x * kGenPerBlock + (uint64_t)threadIdx.x * kGenPerThread;
  uint32_t cnt = 0;
  for (int q = 0; q < kGenPerThread; ++q) {
    const uint64_t i = base + q;
    if (i < draw0 + ndraw) cnt += (splitmix_at(seed, i) >> (64 - bits)) < p;
  }
  for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kGenThreads / 32; ++w) t += wsum[w];
    counts[blockIdx.x] = t;
  }
}

// Exclusive scan of `nb` block counts (one CTA); total in offs[nb].
__global__ void gen_scan_kernel(const uint32_t* counts, uint64_t* offs, int64_t nb) {
  __shared__ uint64_t part[1024];
  const int tid = threadIdx.x;
  const int64_t per = (nb + blockDim.x - 1) / blockDim.x;
  const int64_t b0 = tid * per, b1 = b0 + per < nb ? b0 + per : nb;
  uint64_t s = 0;
  for (int64_t b = b0; b < b1; ++b) s += counts[b];
  part[tid] = s;
  __syncthreads();
  if (tid == 0) {
    uint64_t run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const uint64_t v = part[t];
      part[t] = run;
      run += v;
    }
    offs[nb] = run;
  }
  __syncthreads();
  uint64_t run = part[tid];
  for (int64_t b = b0; b < b1; ++b) {
    offs[b] = run;
    run += counts[b];
  }
}

__global__ void gen_scatter_kernel(uint64_t p, int bits, uint64_t seed, uint64_t draw0, uint64_t ndraw,
                                   const uint64_t* offs, uint64_t out0, uint64_t* out, uint64_t count) {
  __shared__ uint32_t wpre[kGenThreads / 32 + 1];
  const uint64_t base = draw0 + (uint64_t)blockIdx.x * kGenPerBlock + (uint64_t)threadIdx.x * kGenPerThread;
  uint64_t vals[kGenPerThread];
  uint32_t acc_mask = 0, cnt = 0;
  for (int q = 0; q < kGenPerThread; ++q) {
    const uint64_t i = base + q;
    const uint64_t x = splitmix_at(seed, i) >> (64 - bits);
    vals[q] = x;
    if (i < draw0 + ndraw && x < p) {
      acc_mask |= 1u << q;
      ++cnt;
    }
  }
  // Exclusive prefix of cnt over the block, in thread order.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = cnt;
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) wpre[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int w = 0; w < kGenThreads / 32; ++w) {
      const uint32_t v = wpre[w];
      wpre[w] = run;
      run += v;
    }
  }
  __syncthreads();
  uint64_t pos = offs[blockIdx.x] + wpre[warp] + (incl - cnt);
  for (int q = 0; q < kGenPerThread; ++q) {
    if (acc_mask & (1u << q)) {
      const uint64_t k = out0 + pos;
      if (k < count) out[k] = vals[q];
      ++pos;
    }
  }
}

template <class F>
__global__ void reduce_kernel(F f, uint64_t* x, uint64_t count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    x[i] = f.reduce((u128)x[i]);
}

// Host driver: returns the number of draws consumed (for continuation), or
// 0 on a CUDA error. Scratch: counts (u32) and offs (u64) for one chunk.
cudaError_t gen_uniform_device(uint64_t p, uint64_t seed, uint64_t* d_out, uint64_t count, cudaStream_t st,
                               uint64_t* launches) {
  const int bits = 64 - __builtin_clzll(p - 1);
  const double accept = (double)p / (bits == 64 ? 18446744073709551616.0 : (double)(1ULL << bits));
  const uint64_t chunk_blocks = 1 << 16;  // 2^28 draws per chunk
  uint32_t* counts = nullptr;
  uint64_t* offs = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&counts, chunk_blocks * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  e = cudaMallocAsync((void**)&offs, (chunk_blocks + 1) * sizeof(uint64_t), st);
  if (e != cudaSuccess) {
    cudaFreeAsync(counts, st);
    return e;
  }
  uint64_t produced = 0, draw0 = 0;
  while (produced < count) {
    const uint64_t need = count - produced;
    uint64_t ndraw = (uint64_t)((double)need / accept * 1.001) + 4096;
    const uint64_t maxd = chunk_blocks * (uint64_t)kGenPerBlock;
    if (ndraw > maxd) ndraw = maxd;
    const uint64_t nb = (ndraw + kGenPerBlock - 1) / kGenPerBlock;
    gen_count_kernel<<<(unsigned)nb, kGenThreads, 0, st>>>(p, bits, seed, draw0, ndraw, counts);
    gen_scan_kernel<<<1, 1024, 0, st>>>(counts, offs, (int64_t)nb);
    gen_scatter_kernel<<<(unsigned)nb, kGenThreads, 0, st>>>(p, bits, seed, draw0, ndraw, offs, produced, d_out,
                                                             count);
    if (launches) *launches += 3;
    uint64_t total = 0;
    e = cudaMemcpyAsync(&total, offs + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) break;
    produced += total;
    draw0 += ndraw;
  }
  cudaFreeAsync(counts, st);
  cudaFreeAsync(offs, st);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

cudaError_t reduce_device(const FieldParams& fp, uint64_t* d_x, uint64_t count, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  unsigned blocks = (unsigned)((count + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (fp.p == kM61)
    reduce_kernel<<<blocks, 256, 0, st>>>(FpM61(fp), d_x, count);
  else
    reduce_kernel<<<blocks, 256, 0, st>>>(FpBarrett(fp), d_x, count);
  return cudaGetLastError();
}

}  // namespace modlin

namespace modlin {

// ---------------------------------------------------------------------------
// Planted recurrences on the device: each job extends s[0..L) to s[0..n) by
// s[i] = sum_{j=1..L} a_j s[i-j] mod p (coefficients a[0..L) = a_1..a_L).
// One CTA per job (persistent over a job counter); every output is a
// CTA-wide dot product with u128 lazy accumulation, reduced mod p. Exact,
// so the stream equals the host generator's bit for bit.
// ---------------------------------------------------------------------------
template <class F>
__device__ void plant_extend(const F& f, const uint64_t* __restrict__ a, uint64_t* s, int64_t L, int64_t n,
                             uint64_t (*ws)[32]) {
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = T >> 5;
  const uint64_t sb = f.safe_batch();
  for (int64_t i = L; i < n; ++i) {
    u128 acc = 0;
    uint64_t tot = 0, cnt = 0;
    for (int64_t j = tid; j < L; j += T) {
      acc += (u128)a[j] * s[i - 1 - j];
      if (++cnt == sb) {
        tot = f.add(tot, f.reduce(acc));
        acc = 0;
        cnt = 0;
      }
    }
    uint64_t part = f.add(tot, f.reduce(acc));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part = f.add(part, __shfl_down_sync(0xffffffffu, part, off));
    if (lane == 0) ws[i & 1][warp] = part;
    __syncthreads();
    if (tid == 0) {
      uint64_t v = 0;
      for (int w = 0; w < nw; ++w) v = f.add(v, ws[i & 1][w]);
      s[i] = v;
    }
    __syncthreads();
  }
}

__global__ void plant_kernel(const PlantJob* __restrict__ jobs, int64_t count, unsigned long long* next) {
  __shared__ uint64_t ws[2][32];
  __shared__ long long q;
  for (;;) {
    if (threadIdx.x == 0) q = (long long)atomicAdd(next, 1ULL);
    __syncthreads();
    const long long k = q;
    __syncthreads();
    if (k >= count) break;
    const PlantJob J = jobs[k];
    const FieldParams fp{J.p, J.mu_lo, J.mu_hi, J.safe_batch};
    if (J.p == kM61)
      plant_extend(FpM61(fp), J.a, J.s, J.L, J.n, ws);
    else
      plant_extend(FpBarrett(fp), J.a, J.s, J.L, J.n, ws);
    __syncthreads();
  }
}

cudaError_t plant_device(const PlantJob* d_jobs, int64_t count, unsigned long long* d_next, int blocks, int threads,
                         cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  plant_kernel<<<blocks, threads, 0, st>>>(d_jobs, count, d_next);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Jump-ahead for long planted streams. With f(x) = x^L - sum_j a_j x^(L-j)
// and the functional phi(x^i) = s[i] (well defined: phi kills multiples of f),
// s[t + i] = phi(x^t x^i) = sum_j r_j s[j + i] for r = x^t mod f. The stream
// is cut into K segments; segment k starts from the state computed with
// r_k = x^(kT) mod f and is then extended by the recurrence, so every value
// equals the sequential stream's. Polynomial products and remainders mod f
// run a warp per output coefficient; the remainder uses the reversed-inverse
// quotient rev(q) = rev(c) * g mod x^(L-1), g = 1 / (1 - sum_j a_j x^j).
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ uint64_t warp_dot_sum(const F& f, u128 acc, uint64_t tot) {
  uint64_t v = f.add(tot, f.reduce(acc));
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = f.add(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

// c[m] = sum_{i+j=m} a[i] b[j], m < 2L-1.
template <class F>
__global__ void poly_mul_kernel(F f, const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                                uint64_t* __restrict__ c, int L) {
  const int m = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (m >= 2 * L - 1) return;
  const int lo = m - (L - 1) > 0 ? m - (L - 1) : 0, hi = m < L - 1 ? m : L - 1;
  const uint64_t sb = f.safe_batch();
  u128 acc = 0;
  uint64_t tot = 0, cnt = 0;
  for (int i = lo + lane; i <= hi; i += 32) {
    acc += f.prod(a[i], b[m - i]);
    if (++cnt == sb) {
      tot = f.add(tot, f.reduce(acc));
      acc = 0;
      cnt = 0;
    }
  }
  const uint64_t v = warp_dot_sum(f, acc, tot);
  if (lane == 0) c[m] = v;
}

// q[L-2-i] = sum_{k<=i} c[2L-2-k] g[i-k], i < L-1 (the quotient c div f).
template <class F>
__global__ void poly_quot_kernel(F f, const uint64_t* __restrict__ c, const uint64_t* __restrict__ g,
                                 uint64_t* __restrict__ q, int L) {
  const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= L - 1) return;
  const uint64_t sb = f.safe_batch();
  u128 acc = 0;
  uint64_t tot = 0, cnt = 0;
  for (int k = lane; k <= i; k += 32) {
    acc += f.prod(c[2 * L - 2 - k], g[i - k]);
    if (++cnt == sb) {
      tot = f.add(tot, f.reduce(acc));
      acc = 0;
      cnt = 0;
    }
  }
  const uint64_t v = warp_dot_sum(f, acc, tot);
  if (lane == 0) q[L - 2 - i] = v;
}

// r[m] = c[m] - (q f)[m] = c[m] + sum_{i<=min(m,L-2)} q[i] a_(L-m+i), m < L
// (a[] holds a_1..a_L at indices 0..L-1).
template <class F>
__global__ void poly_rem_kernel(F f, const uint64_t* __restrict__ c, const uint64_t* __restrict__ q,
                                const uint64_t* __restrict__ a, uint64_t* __restrict__ r, int L) {
  const int m = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (m >= L) return;
  const int hi = m < L - 2 ? m : L - 2;
  const uint64_t sb = f.safe_batch();
  u128 acc = 0;
  uint64_t tot = 0, cnt = 0;
  for (int i = lane; i <= hi; i += 32) {
    acc += f.prod(q[i], a[L - 1 - m + i]);
    if (++cnt == sb) {
      tot = f.add(tot, f.reduce(acc));
      acc = 0;
      cnt = 0;
    }
  }
  const uint64_t v = warp_dot_sum(f, acc, tot);
  if (lane == 0) r[m] = f.add(c[m], v);
}

// Segment states: out[k T + i] = sum_{j<L} R[k][j] s[j + i] for i < min(L,
// count - k T); 64 x 64 output tiles, 4 x 4 per thread, u128 accumulators.
template <class F>
__global__ void __launch_bounds__(256) jump_states_kernel(F f, const uint64_t* __restrict__ R,
                                                          const uint64_t* __restrict__ s, int L, int K, int64_t T,
                                                          int64_t count, uint64_t* __restrict__ out) {
  __shared__ uint64_t Rs[32][64 + 1];
  __shared__ uint64_t Ss[96];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int i0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  const uint64_t sb = f.safe_batch();
  u128 acc[4][4];
  uint64_t tot[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b] = 0;
      tot[a][b] = 0;
    }
  uint64_t cnt = 0;
  for (int j0 = 0; j0 < L; j0 += 32) {
    for (int idx = tid; idx < 32 * 64; idx += 256) {
      const int kk = idx >> 5, jj = idx & 31;
      const int k = k0 + kk, j = j0 + jj;
      Rs[jj][kk] = (k < K && j < L) ? R[(int64_t)k * L + j] : 0;
    }
    for (int t = tid; t < 96; t += 256) {
      const int idx = j0 + i0 + t;
      Ss[t] = idx < 2 * L - 1 ? s[idx] : 0;
    }
    __syncthreads();
    const int jn = L - j0 < 32 ? L - j0 : 32;
    for (int jj = 0; jj < jn; ++jj) {
      uint64_t rv[4], sv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) rv[a] = Rs[jj][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) sv[b] = Ss[jj + tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += f.prod(rv[a], sv[b]);
      if (++cnt == sb) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            tot[a][b] = f.add(tot[a][b], f.reduce(acc[a][b]));
            acc[a][b] = 0;
          }
        cnt = 0;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int k = k0 + ty + 16 * a;
    if (k >= K) continue;
    const int64_t base = (int64_t)k * T;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + tx + 16 * b;
      if (i < L && base + i < count) out[base + i] = f.add(tot[a][b], f.reduce(acc[a][b]));
    }
  }
}

template <class F>
static cudaError_t jump_mulmod(const F& f, const uint64_t* x, const uint64_t* y, uint64_t* r, const uint64_t* a,
                               const uint64_t* g, uint64_t* cbuf, uint64_t* qbuf, int L, cudaStream_t st) {
  poly_mul_kernel<F><<<(2 * L - 1 + 7) / 8, 256, 0, st>>>(f, x, y, cbuf, L);
  poly_quot_kernel<F><<<(L - 1 + 7) / 8, 256, 0, st>>>(f, cbuf, g, qbuf, L);
  poly_rem_kernel<F><<<(L + 7) / 8, 256, 0, st>>>(f, cbuf, qbuf, a, r, L);
  return cudaGetLastError();
}

template <class F>
static cudaError_t jump_states_t(const F& f, const JumpPlan& P, cudaStream_t st) {
  const int L = P.L;
  // R[0] = 1, xT = x^T mod f by square-and-multiply from x mod f, then
  // R[k] = R[k-1] * xT mod f.
  cudaError_t e = cudaMemsetAsync(P.R, 0, (size_t)P.K * L * 8, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(P.xpow, 0, (size_t)2 * L * 8, st);
  if (e != cudaSuccess) return e;
  const uint64_t one = 1;
  e = cudaMemcpyAsync(P.R, &one, 8, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(P.xpow + L + 1, &one, 8, cudaMemcpyHostToDevice, st);  // x (L >= 2)
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(P.xpow, &one, 8, cudaMemcpyHostToDevice, st);  // accumulator = 1
  if (e != cudaSuccess) return e;
  uint64_t* acc = P.xpow;
  uint64_t* base = P.xpow + L;
  int top = 63;
  while (top > 0 && !((P.T >> top) & 1)) --top;
  for (int b = top; b >= 0; --b) {
    e = jump_mulmod(f, acc, acc, P.tmp, P.a, P.g, P.cbuf, P.qbuf, L, st);
    if (e == cudaSuccess && ((P.T >> b) & 1)) e = jump_mulmod(f, P.tmp, base, acc, P.a, P.g, P.cbuf, P.qbuf, L, st);
    else if (e == cudaSuccess) e = cudaMemcpyAsync(acc, P.tmp, (size_t)L * 8, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  for (int k = 1; k < P.K; ++k) {
    e = jump_mulmod(f, P.R + (int64_t)(k - 1) * L, acc, P.R + (int64_t)k * L, P.a, P.g, P.cbuf, P.qbuf, L, st);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((L + 63) / 64, (P.K + 63) / 64);
  jump_states_kernel<F><<<grid, 256, 0, st>>>(f, P.R, P.head, L, P.K, P.T, P.count, P.out);
  return cudaGetLastError();
}

cudaError_t jump_states(const FieldParams& fp, const JumpPlan& P, cudaStream_t st) {
  if (P.L < 2 || P.K < 1) return cudaErrorInvalidValue;
  if (fp.p == kM61) return jump_states_t(FpM61(fp), P, st);
  return jump_states_t(FpBarrett(fp), P, st);
}

}  // namespace modlin
