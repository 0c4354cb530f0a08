// Blocked Gaussian elimination over F_p on the GPU — panel kernels and the
// plain (integer-pipe) trailing update.
//
// Mirrors the reference's blocked rank (src/fp.rs:125-255): columns are
// processed in panels of PANEL = 64; inside a panel every column gets the
// first nonzero row as pivot (src/fp.rs:150-157), the pivot rows are coupled
// among themselves (src/fp.rs:181-200) and the far rows receive one rank-pb
// update with u128 lazy accumulation (src/fp.rs:202-248).
//
// GPU restructuring (rank is invariant under the choice of pivot rows, so the
// result is bit-exact):
//  * window_kernel: one CTA eliminates a window of <= 64 candidate rows of the
//    panel in shared memory, column by column, with first-nonzero pivoting
//    (a ballot over the window). It eliminates fraction-free (row <- e*row -
//    h*pivot), so no modular inverse sits on the sequential path; it records
//    each pivot row's transformation (alpha, G) and inverts the pivot values
//    afterwards in parallel.
//  * bulk_kernel: every other active row is reduced against the window's
//    pivots (a warp per row, reference-style multipliers f = e * inv). Rows
//    left with a nonzero residual in the panel become the next window's
//    candidates; the panel is finished when no residual remains, which is
//    exactly the reference's "no nonzero entry below" condition.
//  * couple_kernel: the pivot rows' trailing parts are reduced among
//    themselves with (alpha, G), giving U (src/fp.rs:184-200).
//  * move_rows_kernel: pivot rows leave the active block [rank, n) so that
//    the trailing block stays contiguous (the reference's row swaps).
//  * trailing_plain_kernel: C -= L * U mod p on the integer pipes, u128
//    accumulation, one Barrett reduction per safe_batch products.
#pragma once
#include <cstdint>

#include "field.cuh"

namespace modlin {

constexpr int kPanel = 64;         // panel width (src/fp.rs:29)
constexpr int kWindow = 64;        // candidate rows per window round
constexpr int kWindowThreads = 512;
constexpr int kInvThreads = 1024;   // block_inverse_kernel: 16 threads per block row

// Device-resident panel state (one per rank job).
struct PanelState {
  int32_t prow[kPanel];    // physical row of pivot k
  int32_t pcol[kPanel];    // absolute column of pivot k
  uint64_t inv[kPanel];    // inverse of pivot value (Upanel[k][pcol[k]-col])
  uint64_t alpha[kPanel];  // fraction-free scale of pivot row k
  int32_t cand[kWindow];   // residual rows found by the last bulk pass
  int32_t pb;              // pivots so far in this panel
  int32_t ncand;           // number of residual rows (may exceed kWindow)
  uint64_t colmask;        // panel columns (relative) that have a pivot
  int32_t err;
  int32_t pad;
};

}  // namespace modlin
