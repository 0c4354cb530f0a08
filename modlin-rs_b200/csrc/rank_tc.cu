// Tensor-core trailing update — placeholder until the tcgen05 kernel lands:
// MODLIN_RANK_TC reports "not supported" instead of silently running the
// plain kernel.
#include "rank_tc.cuh"

#include <climits>

namespace modlin {

int tc_crossover_n(uint64_t) { return INT_MAX; }
size_t tc_a_bytes(int) { return 16; }
size_t tc_b_bytes(int) { return 16; }

cudaError_t launch_trailing_tc(const FieldParams&, uint64_t*, int64_t, int, int, int, const uint64_t*, int,
                               const uint64_t*, int64_t, int, uint8_t*, uint8_t*, int, cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace modlin
