// Kernel launches with programmatic dependent launch (PDL).
//
// The rank's block steps are chains of short dependent kernels (block
// inverses, 64 x 64 products, limb splits, narrow updates); at the end of the
// elimination each link lasts a few microseconds, and the gap between two
// dependent launches in one stream (~3 us on B200) is a large share of the
// step. Launched with cudaLaunchAttributeProgrammaticStreamSerialization,
// the next kernel's CTAs are scheduled by the GPU as soon as the previous
// grid's CTAs have exited, instead of after a full launch round trip
// (measured: ~1.8 us saved per boundary). Every kernel launched this way
// calls pdl_wait() before its first global-memory access (read or write),
// which returns once the previous grid has completed and its writes are
// visible, so the data dependencies are exactly those of a plain launch.
// Without the attribute pdl_wait() returns at once.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <utility>

namespace modlin {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Predication of a speculatively queued block step. The rank driver queues
// step t of its block pipeline before it knows whether step t's diagonal
// block is invertible; the look-ahead chain that inverts it records the
// first failed step in a device word (*bad = min(*bad, t)), and every kernel
// of step t is launched with Guard{bad, t} and does nothing when
// *bad <= step. The word only changes between launches that depend on each
// other (a chain and the kernels of its own or a later step), so every
// thread of a launch reads the same value. A default Guard never skips.
struct Guard {
  int* bad = nullptr;
  int step = 0;
};

__device__ __forceinline__ bool guard_skip(const Guard& g) { return g.bad && __ldcg(g.bad) <= g.step; }

// PDL is on unless the environment sets MODLIN_PDL=0 (read once).
inline bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("MODLIN_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

// kernel<<<grid, block, smem, st>>>(args...), with the PDL attribute when
// enabled (and, when cluster_x > 1, a cluster of cluster_x CTAs).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            int cluster_x, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[2];
  int na = 0;
  if (pdl_enabled()) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (cluster_x > 1) {
    at[na].id = cudaLaunchAttributeClusterDimension;
    at[na].val.clusterDim.x = cluster_x;
    at[na].val.clusterDim.y = 1;
    at[na].val.clusterDim.z = 1;
    ++na;
  }
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = na ? at : nullptr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace modlin
