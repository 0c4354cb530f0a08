// Launch wrappers of the rank kernels (host side).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"
#include "launch.cuh"
#include "rank_plain.cuh"

namespace modlin {

// Inverse of the 64 x 64 diagonal block (negated, row = panel column) or,
// when it is singular, *status = 1 (status may be null) and, with a guard,
// *g.bad = min(*g.bad, g.step + 1): the inverse belongs to the look-ahead
// chain of step g.step + 1 and does nothing once step g.step has failed.
// With reset_status the kernel first sets *status = 0 (no separate memset).
template <class F>
void launch_block_inverse(const F& f, const uint64_t* m, int64_t ld, int r0, int col, uint64_t* Vneg, int* status,
                          cudaStream_t st, bool reset_status = false, const Guard& g = Guard());
// C = D - A * B (negate) or D + A * B on 64 x 64 blocks (D may be null).
template <class F>
void launch_small_gemm64(const F& f, const uint64_t* A, int64_t lda, const uint64_t* B, int64_t ldb, const uint64_t* D,
                         int64_t ldd, uint64_t* C, int64_t ldc, bool negate, cudaStream_t st,
                         const Guard& g = Guard());
// Up to kSgMaxProbs independent 64 x 64 products in one launch: problem i is
// C = D - A * B (negate) or D + A * B (D may be null) with inner dimension k
// (64 or 128; 0 means 64), or, with A null, the copy C = D.
struct SgProb {
  const uint64_t* A;
  const uint64_t* B;
  const uint64_t* D;
  uint64_t* C;
  int64_t lda, ldb, ldd, ldc;
  int negate;
  int k;
};
constexpr int kSgMaxProbs = 4;
template <class F>
void launch_small_gemm64_batch(const F& f, const SgProb* probs, int count, cudaStream_t st,
                               const Guard& g = Guard());
// n words at p set to zero (a kernel, so that it chains with programmatic
// dependent launches).
void launch_zero(uint64_t* p, int64_t n, cudaStream_t st, const Guard& g = Guard());
template <class F>
void launch_window(const F& f, const uint64_t* m, int64_t ld, int n, int r0, int col, int W, int round,
                   PanelState* ps, uint64_t* Upanel, uint64_t* G, const uint64_t* Lbuf, uint8_t* is_pivot,
                   cudaStream_t st);
template <class F>
void launch_bulk(const F& f, uint64_t* m, int64_t ld, int n, int r0, int col, int W, int pb_lo, PanelState* ps,
                 const uint64_t* Upanel, uint64_t* Lbuf, const uint8_t* is_pivot, int num_sms, cudaStream_t st);
template <class F>
void launch_couple(const F& f, const uint64_t* m, int64_t ld, int n, int jend, const PanelState* ps,
                   const uint64_t* G, uint64_t* Ubuf, int64_t ldU, cudaStream_t st);
void launch_moves(uint64_t* m, int64_t ld, int n, int jend, const int2* moves, int nmoves, uint64_t* Lbuf, int r0,
                  int pb, cudaStream_t st);
void launch_clear_flags(const PanelState* ps, uint8_t* is_pivot, cudaStream_t st);
// err: device error words (err[0] = 1 when a bounded wait expired).
template <class F>
void launch_trailing_plain(const F& f, uint64_t* m, int64_t ld, int rbeg, int rend, int jend, int cend,
                           const uint64_t* Lbuf, int r0, const uint64_t* Ubuf, int64_t ldU, int K, int* err,
                           cudaStream_t st);
// The plain trailing update's arithmetic alone (its inner loop on operands
// resident in shared memory, `iters` passes of depth 64 per thread): blocks x
// 256 x 16 x 64 x iters modular multiply-adds. The CTAs per SM that
// trailing_plain_kernel reaches are given by plain_blocks_per_sm.
template <class F>
cudaError_t launch_plain_mac_peak(const F& f, int blocks, int iters, uint64_t* out, cudaStream_t st);
template <class F>
int plain_blocks_per_sm();

}  // namespace modlin
