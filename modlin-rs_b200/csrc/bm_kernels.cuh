// Berlekamp-Massey launchers (host side).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "field.cuh"

namespace modlin {

// One sequence of a batch: field constants inline so a launch mixes primes.
struct BmJob {
  uint64_t p, mu_lo, mu_hi, safe_batch;
  const uint64_t* s;  // device pointer, n residues
  int64_t n;
  int64_t slot;       // output index
};

cudaError_t launch_bm_block(const BmJob& job, uint64_t* gws, int64_t smem_words, int threads, int64_t* d_out,
                            cudaStream_t st);
cudaError_t launch_bm_batch(const BmJob* d_jobs, int64_t count, unsigned long long* d_next, uint64_t* gws,
                            int64_t gws_words, int64_t smem_words, int blocks, int threads, int64_t* d_out,
                            cudaStream_t st);
int bm_batch_max_blocks_per_sm(int threads, int64_t smem_words);
// Loads the module of bm_block_kernel on the current device now (a lazily
// loaded module would otherwise be loaded, and its memory allocated, at the
// first launch).
cudaError_t bm_block_prepare();
// spin: cycles a CTA waits at a grid barrier before it gives up and sets the
// error word; skip_cta (>= 0, tests only): that CTA skips its arrival at the
// first step barrier, so the waits expire.
cudaError_t launch_bm_grid(const FieldParams& fp, const uint64_t* s, int64_t n, int ctas, int threads, uint64_t* b0,
                           uint64_t* b1, void* gs, long long spin, int skip_cta, int64_t* d_out, cudaStream_t st,
                           int* ctas_used);
// One long sequence on one thread-block cluster of R = 16 CTAs (8 where 16
// cannot be launched and the slices fit); b0, b1: n-word global workspaces.
// bm_cluster_size gives R for n (0: too long for the cluster's shared memory).
constexpr int64_t kBmClusterSliceBytes = 200 * 1024;
int bm_cluster_size(int64_t n);
cudaError_t launch_bm_cluster(const FieldParams& fp, const uint64_t* s, int64_t n, int R, uint64_t* b0, uint64_t* b1,
                              int64_t* d_out, cudaStream_t st);
size_t grid_sync_bytes();
int grid_sync_err_offset();

}  // namespace modlin
