// Device-side workload generation (host side declarations).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"

namespace modlin {

cudaError_t gen_uniform_device(uint64_t p, uint64_t seed, uint64_t* d_out, uint64_t count, cudaStream_t st,
                               uint64_t* launches);
cudaError_t reduce_device(const FieldParams& fp, uint64_t* d_x, uint64_t count, cudaStream_t st);

// One planted-recurrence extension job (device pointers): s[0..L) given,
// s[L..n) produced; a[0..L) = a_1..a_L.
struct PlantJob {
  uint64_t p, mu_lo, mu_hi, safe_batch;
  const uint64_t* a;
  uint64_t* s;
  int64_t L, n;
};
cudaError_t plant_device(const PlantJob* d_jobs, int64_t count, unsigned long long* d_next, int blocks, int threads,
                         cudaStream_t st);

// Segment states of a long planted stream (jump-ahead): with head =
// s[0 .. 2L-1), writes out[k T .. k T + L) = s[k T .. k T + L) for k < K (cut
// at count). a = a_1..a_L, g = 1 / (1 - sum_j a_j x^j) mod x^(L-1); R (K x L),
// xpow (2L), tmp (L), cbuf (2L), qbuf (L) are device scratch. L >= 2.
struct JumpPlan {
  const uint64_t* a;
  const uint64_t* g;
  const uint64_t* head;
  uint64_t* out;
  uint64_t *R, *xpow, *tmp, *cbuf, *qbuf;
  int L, K;
  int64_t T, count;
};
cudaError_t jump_states(const FieldParams& fp, const JumpPlan& P, cudaStream_t st);

}  // namespace modlin
