// Batched rank launcher (host side).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace modlin {

// One matrix of a batch: n x n row-major residues at device pointer m
// (clobbered), field constants inline so one launch mixes primes.
struct RankJob {
  uint64_t p, mu_lo, mu_hi, safe_batch;
  uint64_t* m;
  int64_t n;
  int64_t slot;  // output index
};

constexpr int kRankBatchThreads = 256;
// Largest side the batched kernel takes (its row permutation lives in shared
// memory); larger matrices go through the single-matrix engine.
constexpr int64_t kRankBatchMaxN = 8192;

// The tensor-core variant of the batched rank (one CTA per matrix, trailing
// updates as INT8-limb GEMMs on its SM); used for the sides the autotuner
// finds it faster on.
size_t rank_batch_tc_smem_bytes(int64_t max_n);
int rank_batch_tc_blocks_per_sm(int64_t max_n);
// d_err: two device ints, zeroed by the caller; d_err[0] != 0 afterwards means
// a bounded wait expired.
cudaError_t launch_rank_batch_tc(const RankJob* d_jobs, int64_t count, unsigned long long* d_next, int64_t max_n,
                                 int blocks, int64_t* d_out, int* d_err, cudaStream_t st);
size_t rank_batch_smem_bytes(int64_t max_n);
int rank_batch_blocks_per_sm(int64_t max_n);
cudaError_t launch_rank_batch(const RankJob* d_jobs, int64_t count, unsigned long long* d_next, int64_t max_n,
                              int blocks, int64_t* d_out, cudaStream_t st);

}  // namespace modlin
