// Berlekamp-Massey with no allocation on the call path.
//
// Some callers cannot allocate device memory when they call in: a host that
// hands every byte of device memory to its own pool allocator, or a loop that
// must not pay the implicit device synchronisation of cudaMalloc/cudaFree.
// modlin_linear_complexity_device_noalloc serves them: it runs the
// one-CTA-per-sequence Berlekamp-Massey kernel (bm_block_kernel) with its
// scratch — the c, b and t polynomials — in dynamic shared memory when they
// fit (3n words within 200 KiB, n <= 8533), else in a fixed file-scope
// device array, never in a workspace from cudaMalloc. The caller passes the
// sequence and the result slot, both in device memory.
//
// Limits and sharing:
//  * at most kNoAllocMaxN residues per call (the array holds 3 * kNoAllocMaxN
//    words = 6 MiB, which every GPU that loads the library keeps until exit);
//  * every call uses the same array, so calls that overlap on the GPU race:
//    issue them on one stream (or otherwise order them);
//  * the array keeps the previous call's contents; the kernel initialises c
//    and b itself, and t is written before it is read, so nothing needs
//    clearing between calls;
//  * the first call on a device is the set-up: with that device current it
//    looks up the array's device address (cudaGetSymbolAddress) and caches
//    it, and it loads the modules of the array and of the kernel, which the
//    CUDA runtime otherwise loads lazily at first use. Loading a module
//    allocates device memory, so make that first call (n = 0 is enough)
//    before the caller's pool takes the device memory, and before any stream
//    capture. The cached address belongs to the device's primary context:
//    after cudaDeviceReset on that device this entry point must not be used
//    again in the process.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/modlin.h"
#include "bm_kernels.cuh"
#include "field.cuh"

namespace modlin {

constexpr int64_t kNoAllocMaxN = int64_t(1) << 18;
constexpr int64_t kNoAllocSmemWords = (200 * 1024) / 8;  // shared memory used when 3n words fit

static __device__ __align__(256) uint64_t g_noalloc_scratch[3 * kNoAllocMaxN];

static std::mutex g_noalloc_mu;
static uint64_t* g_noalloc_addr[64];  // device address of the array, per device

static int noalloc_scratch(uint64_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return MODLIN_ENODEV;
  }
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e == cudaSuccess) e = bm_block_prepare();
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return MODLIN_ECUDA;
    }
    g_noalloc_addr[dev] = static_cast<uint64_t*>(p);
  }
  *out = g_noalloc_addr[dev];
  return MODLIN_OK;
}

}  // namespace modlin

extern "C" int modlin_linear_complexity_device_noalloc(uint64_t p, const uint64_t* d_s, size_t n,
                                                       int64_t* d_lc_out, void* stream) {
  using namespace modlin;
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (n > (size_t)kNoAllocMaxN) return MODLIN_EINVAL_N;
  if (!d_lc_out || (!d_s && n)) return MODLIN_EINVAL_ARG;
  uint64_t* scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc != MODLIN_OK) return rc;
  const BmJob job{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_s, (int64_t)n, 0};
  const cudaError_t e = launch_bm_block(job, scratch, kNoAllocSmemWords, n >= 4096 ? 1024 : 256, d_lc_out,
                                        static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? MODLIN_OK : MODLIN_ECUDA;
}
