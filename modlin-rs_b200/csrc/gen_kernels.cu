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

}  // namespace modlin
