// Tensor-core (tcgen05 kind::i8) trailing update of the blocked rank.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "field.cuh"
#include "launch.cuh"

namespace modlin {

// Extra output of a tensor-core update over 2^61 - 1: the result rows from
// row0 on are also written as limb planes in the A-operand layout of a
// K = kk update (the layout tc_split_a writes for rows row0 ..), so the next
// product needs no split kernel. With c_zero the update computes 0 - A * B:
// C is neither read nor written (only the limb planes are).
struct LimbOut {
  uint8_t* Aw = nullptr;
  int32_t row0 = 0;
  int32_t kk = 64;
  int32_t c_zero = 0;
};

// Smallest side for which MODLIN_RANK_AUTO uses the tensor-core update.
int tc_crossover_n(uint64_t p);
// Workspace bytes for the limb planes of L (rows x K) and U (K x cols), K <= 128.
size_t tc_a_bytes(int rows);
size_t tc_b_bytes(int cols);
// A[rbeg..rend, jend..cend] -= L * U mod p, K <= 128, via exact INT8-limb GEMMs (L row
// r at Lbuf[(r - r0) * lda], U row k at Ubuf[k * ldU], absolute columns). `err` points
// at two device ints (zeroed by the caller); err[0] != 0 afterwards means a
// bounded wait inside the kernel expired.
cudaError_t launch_trailing_tc(const FieldParams& fp, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend,
                               const uint64_t* Lbuf, int64_t lda, int r0, const uint64_t* Ubuf, int64_t ldU, int K,
                               uint8_t* Aw, uint8_t* Bw, int num_sms, int* err, cudaStream_t st,
                               const Guard& g = Guard());

// The three steps of launch_trailing_tc, for callers that reuse one operand's
// limb planes across launches: limb planes of A rows [rbeg, rend) (row r at
// A[(r - r0) * lda]), of B columns [jend, cend) (row k at B[k * ldb]), and the
// update A[rbeg..rend, jend..cend] -= A * B on at most max_ctas SMs. The same
// K (<= 64 or <= 128: two plane layouts) must be given to all three.
cudaError_t tc_split_a(const FieldParams& fp, const uint64_t* A, int64_t lda, int r0, int rbeg, int rend, int K,
                       uint8_t* Aw, cudaStream_t st, const Guard& g = Guard());
cudaError_t tc_split_b(const FieldParams& fp, const uint64_t* B, int64_t ldb, int jend, int cend, int K, uint8_t* Bw,
                       cudaStream_t st, const Guard& g = Guard());
cudaError_t tc_update(const FieldParams& fp, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend, int K,
                      const uint8_t* Aw, const uint8_t* Bw, int max_ctas, int* err, cudaStream_t st,
                      const Guard& g = Guard(), const LimbOut& lo = LimbOut());
// Whether tc_update takes a LimbOut for this prime (2^61 - 1 only).
inline bool tc_limb_out_supported(uint64_t p) { return p == kM61; }

// Each launch takes an optional Guard (launch.cuh): a predicated block step
// whose kernels do nothing once the step is known to have failed.

// Updates over 2^61 - 1 on CTA pairs or (default) on single CTAs.
extern bool g_tc_pairs;

}  // namespace modlin
