// The C ABI (include/modlin.h): device context, the rank driver (panel loop),
// the linear-complexity drivers, batches and the workload generators.
#include <cuda_runtime.h>

#include <cmath>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/modlin.h"
#include "bm_kernels.cuh"
#include "field.cuh"
#include "gen_kernels.cuh"
#include "prng_kernels.cuh"
#include "rank_batch.cuh"
#include "rank_kernels.cuh"
#include "rank_tc.cuh"

namespace modlin {

std::atomic<uint64_t> g_launches{0};
// Failure-detection test (modlin_testing_grid_timeout_once): the next grid
// Berlekamp-Massey launch waits at most g_fault_spin cycles per barrier and
// CTA g_fault_skip_cta skips its first step arrival; consumed by that launch.
static std::atomic<long long> g_fault_spin{0};
static std::atomic<int> g_fault_skip_cta{-1};
static double g_last_trailing_ms = 0.0;
static double g_last_trailing_macs = 0.0;

// ---------------------------------------------------------------------------
// Per-device context: one stream, cached workspaces, pinned staging.
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Choices the autotuner measures (defaults until modlin_autotune runs on the
// device): plain/tensor-core crossover per limb count, smallest side for
// two-panel block steps, BM threads per CTA by length, BM block/cluster
// crossover, BM batch threads by the longest sequence.
struct Tune {
  bool measured = false;
  int tc_cross[4] = {512, 512, 512, 512};           // 1, 2, 4, 8 limbs
  int two_panel_min = 256;
  int bm_threads[4] = {256, 256, 1024, 1024};       // n < 1024, < 4096, < 16384, longer
  int bm_cluster_min = 16384;
  int bm_batch_threads[3] = {128, 256, 512};        // longest < 512, < 2048, longer
  // Shared memory per batch CTA (KiB), by the same classes: a sequence whose
  // c, b, t (24 bytes per entry) do not fit runs from the CTA's global
  // workspace; smaller caps put more CTAs on an SM.
  int bm_batch_smem_kib[3] = {200, 200, 200};
  int batch_tc_min = 1 << 30;  // batched rank: sides on the tensor-core kernel (off until measured faster)
};

static int limb_class(uint64_t p) {
  const int bits = 64 - __builtin_clzll(p - 1);
  return bits <= 8 ? 0 : bits <= 16 ? 1 : bits <= 32 ? 2 : 3;
}
static int bm_len_class(size_t n) { return n < 1024 ? 0 : n < 4096 ? 1 : n < 16384 ? 2 : 3; }
static int bm_batch_class(int64_t maxn) { return maxn < 512 ? 0 : maxn < 2048 ? 1 : 2; }

struct Ctx {
  int device = -1;
  Tune tune;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  // rank workspaces
  DevBuf mat, lbuf, ubuf, upanel, gmat, pstate, ispiv, moves;
  DevBuf repsbuf;  // matrices of a batched -R run
  DevBuf tcA, tcB;  // limb planes for the tensor-core trailing update
  DevBuf tcerr;     // bounded-wait error words of the tensor-core kernel
  DevBuf binv;      // block-step status words and the negated block inverse
  DevBuf tcBn;      // limb planes of the narrow update's B operand (W = P^-1 U_next)
  DevBuf tcBp[2];   // limb planes of -P^-1 (B operand of the multipliers H = X P^-1), alternating steps
  DevBuf tcX[2];    // limb planes of the block steps' X panels (alternating steps)
  cudaStream_t aux = nullptr;  // look-ahead stream: the next block's inverse
  cudaEvent_t ev_narrow = nullptr, ev_inv[2] = {nullptr, nullptr};
  PanelState* h_ps = nullptr;
  int2* h_moves = nullptr;
  // linear-complexity workspaces
  DevBuf seq, bmws, bmout, bmsync, bmjobs, bmnext;
  DevBuf gena, genjobs;  // planted-generator coefficients and jobs
  DevBuf jump;           // jump-ahead scratch of the long planted generator
  DevBuf batchm, rbjobs, rbout;  // batched rank: matrix arena, jobs, ranks
  DevBuf tunebuf;                // autotuner inputs
  PrngCache prng;                // generator fills: jump matrices, workspace
  DevBuf invst;                  // status word of modlin_block_inverse_device
  int64_t* h_out = nullptr;
  std::vector<cudaEvent_t> ev;
};

static std::mutex g_ctx_mu;
static Ctx* g_ctx[64];

static int get_ctx(Ctx** out) {
  // A failed earlier call may have left a (non-sticky) error in the runtime's
  // last-error slot; it must not be reported by this call.
  cudaGetLastError();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MODLIN_ENODEV;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MODLIN_ENODEV;
  if (dev < 0 || dev >= 64) return MODLIN_ENODEV;
  std::lock_guard<std::mutex> g(g_ctx_mu);
  if (!g_ctx[dev]) {
    Ctx* c = new Ctx();
    c->device = dev;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return MODLIN_ECUDA;
    }
    if (cudaMallocHost((void**)&c->h_ps, sizeof(PanelState)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_moves, sizeof(int2) * kPanel) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_out, sizeof(int64_t) * 4) != cudaSuccess) {
      delete c;
      return MODLIN_ENOMEM;
    }
    g_ctx[dev] = c;
  }
  *out = g_ctx[dev];
  return MODLIN_OK;
}

static int cuda_rc(cudaError_t e) {
  if (e == cudaSuccess) return MODLIN_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return MODLIN_ENOMEM;
  }
  return MODLIN_ECUDA;
}

// Device-memory entry points run on the caller's stream; NULL is the legacy
// default stream, so work the caller queued there (e.g. a copy that fills the
// input) is ordered before the call.
static cudaStream_t user_stream(void* s) { return s ? (cudaStream_t)s : cudaStreamLegacy; }

#define CK(expr)                          \
  do {                                    \
    cudaError_t _e = (expr);              \
    if (_e != cudaSuccess) return cuda_rc(_e); \
  } while (0)

// ---------------------------------------------------------------------------
// Rank driver.
// ---------------------------------------------------------------------------
struct RankRun {
  const FieldParams* fp;
  uint64_t* m;
  int n;
  int kernel;
  cudaStream_t st;
  Ctx* ctx;
  std::vector<int>* pcols;
  modlin_progress_fn cb;
  void* cb_ctx;
  int two_panel_min;  // smallest remaining block (rows) for two-panel steps (tensor-core path)
};

static bool use_tc(const RankRun& R) {
  if (R.kernel == MODLIN_RANK_PLAIN) return false;
  if (R.kernel == MODLIN_RANK_TC) return true;
  return R.n >= R.ctx->tune.tc_cross[limb_class(R.fp->p)];
}

// Whatever path leaves rank_impl (an error included), the look-ahead work on
// the second stream has finished before the workspaces it uses are reused.
struct AuxDrain {
  Ctx* C;
  ~AuxDrain() {
    if (C->aux) cudaStreamSynchronize(C->aux);
  }
};

template <class F>
static int rank_impl(const RankRun& R, size_t* rank_out) {
  const F f(*R.fp);
  Ctx* C = R.ctx;
  AuxDrain drain{C};
  const int n = R.n;
  const int64_t ld = n;
  cudaStream_t st = R.st;
  CK(C->lbuf.ensure((size_t)n * kPanel * 8));
  CK(C->ubuf.ensure((size_t)kPanel * n * 8));
  CK(C->upanel.ensure((size_t)kPanel * kPanel * 8));
  CK(C->gmat.ensure((size_t)kPanel * kPanel * 8));
  CK(C->pstate.ensure(sizeof(PanelState)));
  CK(C->ispiv.ensure((size_t)n));
  CK(C->moves.ensure(sizeof(int2) * kPanel));
  const bool tc = use_tc(R);
  if (tc) {
    CK(C->tcA.ensure(tc_a_bytes(n)));
    CK(C->tcB.ensure(tc_b_bytes(n)));
  }
  CK(C->tcerr.ensure(2 * sizeof(int)));
  CK(cudaMemsetAsync(C->tcerr.p, 0, 2 * sizeof(int), st));
  uint64_t* Lbuf = C->lbuf.as<uint64_t>();
  uint64_t* Ubuf = C->ubuf.as<uint64_t>();
  uint64_t* Upanel = C->upanel.as<uint64_t>();
  uint64_t* G = C->gmat.as<uint64_t>();
  PanelState* ps = C->pstate.as<PanelState>();
  uint8_t* ispiv = C->ispiv.as<uint8_t>();
  int2* d_moves = C->moves.as<int2>();
  CK(cudaMemsetAsync(ispiv, 0, (size_t)n, st));
  g_launches++;

  // Trailing-update timing with events on the launching stream.
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tev;
  size_t ev_used = 0;
  auto take_events = [&]() -> std::pair<cudaEvent_t, cudaEvent_t> {
    while (C->ev.size() < 2 * (ev_used + 1)) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      C->ev.push_back(e);
    }
    auto pr = std::make_pair(C->ev[2 * ev_used], C->ev[2 * ev_used + 1]);
    ++ev_used;
    return pr;
  };

  // ---- Block pipeline (tensor-core path) -------------------------------
  // A block step t takes w = 64 or 128 columns at (r0, c0): P = A[r0 ..
  // r0+w, c0 .. c0+w) is the pivot block, X = A[r0+w .., c0 .. c0+w) the
  // panel below it, U = A[r0 .. r0+w, c0+w ..) the pivot rows' trailing part.
  // When P is invertible its rows and columns are this step's pivots (every
  // panel column is independent of the earlier ones) and the trailing block
  // becomes the Schur complement A - X P^-1 U, whose rank is the rank of what
  // remains: the reference's panel elimination (src/fp.rs:146-248) in block
  // form. Per step, on the main stream:
  //   W = P^-1 U_next (the next step's wn columns; w x wn, 64 x 64 products),
  //   narrow update A[r0+w .., next columns] -= X W (K = w),
  //   H = X P^-1 (one n x w x w product), wide update A[.., rest] -= H U.
  // On the second stream, after the narrow update, the chain of step t+1
  // computes -P^-1 of the next block (one block inverse, or for w = 128 two
  // inverses and six 64 x 64 products) while the wide update runs. The
  // critical path per step is chain -> W -> narrow -> next chain; the
  // multipliers H and the wide update are off it.
  // The host queues step t before it knows whether step t's block is
  // invertible: every kernel of step t carries Guard{gbad, t} and does
  // nothing once a chain has recorded a failure at or before t. The host then
  // reads step t's chain result (the GPU works on step t meanwhile); on a
  // failure it waits for the skipped work, and the panel takes the general
  // path below.
  uint64_t* Hb = Lbuf;  // multipliers H, row stride w
  const size_t blk = (size_t)kPanel * kPanel;
  uint64_t *V11n = nullptr, *Yb = nullptr, *Sb = nullptr, *VSn = nullptr, *Zb = nullptr;
  uint64_t* Pn[2] = {nullptr, nullptr};  // -P^-1 of alternating steps (row stride w)
  uint64_t* Wbuf = Ubuf;                 // W = P^-1 U_next: w rows, row stride n, absolute columns
  int* gbad = nullptr;                   // first failed step of the pipeline (0x7f7f7f7f: none)
  int* h_bad = reinterpret_cast<int*>(C->h_out) + 4;  // its value after each step's chain
  uint8_t *tA = nullptr, *tB = nullptr, *tBn = nullptr, *tBp[2] = {nullptr, nullptr}, *tX[2] = {nullptr, nullptr};
  int* terr = C->tcerr.as<int>();
  if (tc) {
    CK(C->binv.ensure(256 + 14 * blk * 8));
    CK(C->lbuf.ensure((size_t)n * 2 * kPanel * 8));
    CK(C->ubuf.ensure((size_t)2 * kPanel * n * 8));
    CK(C->tcBn.ensure(tc_b_bytes(2 * kPanel)));
    CK(C->tcBp[0].ensure(tc_b_bytes(2 * kPanel)));
    CK(C->tcBp[1].ensure(tc_b_bytes(2 * kPanel)));
    CK(C->tcX[0].ensure(tc_a_bytes(n)));
    CK(C->tcX[1].ensure(tc_a_bytes(n)));
    Lbuf = Hb = C->lbuf.as<uint64_t>();
    Ubuf = Wbuf = C->ubuf.as<uint64_t>();
    gbad = C->binv.as<int>() + 16;
    V11n = reinterpret_cast<uint64_t*>(C->binv.as<char>() + 256);
    Yb = V11n + blk;
    Sb = Yb + blk;
    VSn = Sb + blk;
    Zb = VSn + blk;
    Pn[0] = Zb + blk;   // 128 x 128
    Pn[1] = Pn[0] + 4 * blk;
    tA = C->tcA.as<uint8_t>();
    tB = C->tcB.as<uint8_t>();
    tBn = C->tcBn.as<uint8_t>();
    tBp[0] = C->tcBp[0].as<uint8_t>();
    tBp[1] = C->tcBp[1].as<uint8_t>();
    tX[0] = C->tcX[0].as<uint8_t>();
    tX[1] = C->tcX[1].as<uint8_t>();
    if (!C->aux) {
      CK(cudaStreamCreateWithFlags(&C->aux, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&C->ev_narrow, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&C->ev_inv[0], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&C->ev_inv[1], cudaEventDisableTiming));
    }
  }

  // -P^-1 of the 128 x 128 block at (rr, cc) into Pout (row stride 128) on
  // `s`: P = [[P11, P12], [P21, P22]] in 64 x 64 blocks, V11 = P11^-1,
  // S = P22 - P21 V11 P12, and
  // -P^-1 = [[-V11 - Z S^-1 Y, Z S^-1], [S^-1 Y, -S^-1]] with Y = P21 V11,
  // Z = V11 P12: six kernels (programmatic dependent launches chain them).
  auto prep128 = [&](int rr, int cc, cudaStream_t s, uint64_t* Pout, const Guard& g) -> cudaError_t {
    const uint64_t* P11 = R.m + (int64_t)rr * ld + cc;
    const uint64_t* P12 = P11 + kPanel;
    const uint64_t* P21 = P11 + (int64_t)kPanel * ld;
    const uint64_t* P22 = P21 + kPanel;
    uint64_t* const TL = Pout;
    uint64_t* const TR = Pout + kPanel;
    uint64_t* const BL = Pout + 2 * blk;
    uint64_t* const BR = BL + kPanel;
    launch_block_inverse<F>(f, R.m, ld, rr, cc, V11n, nullptr, s, false, g);
    const SgProb yz[2] = {{P21, V11n, nullptr, Yb, ld, kPanel, 0, kPanel, 1, kPanel},    // Y = P21 V11
                          {V11n, P12, nullptr, Zb, kPanel, ld, 0, kPanel, 1, kPanel}};  // Z = V11 P12
    launch_small_gemm64_batch<F>(f, yz, 2, s, g);
    launch_small_gemm64<F>(f, Yb, kPanel, P12, ld, P22, ld, Sb, kPanel, true, s, g);  // S = P22 - Y P12
    launch_block_inverse<F>(f, Sb, kPanel, 0, 0, VSn, nullptr, s, false, g);
    const SgProb tb[3] = {{Zb, VSn, nullptr, TR, kPanel, kPanel, 0, 2 * kPanel, 1, kPanel},     // Z S^-1
                          {VSn, Yb, nullptr, BL, kPanel, kPanel, 0, 2 * kPanel, 1, kPanel},     // S^-1 Y
                          {nullptr, nullptr, VSn, BR, 0, 0, kPanel, 2 * kPanel, 0, kPanel}};   // -S^-1
    launch_small_gemm64_batch<F>(f, tb, 3, s, g);
    launch_small_gemm64<F>(f, TR, 2 * kPanel, Yb, kPanel, V11n, kPanel, TL, 2 * kPanel, true, s, g);
    g_launches += 6;
    return cudaGetLastError();
  };

  // Chain of step t on the second stream: -P^-1 of the w x w block at (r, c)
  // into Pn[t & 1] and its limb planes into tBp[t & 1]; a singular block
  // records t in gbad. Its kernels are skipped once an earlier step has
  // failed (Guard step t - 1). The host learns the result from h_bad[t & 1]
  // after ev_inv[t & 1].
  auto chain = [&](int t, int r, int c, int w) -> int {
    const Guard gc{gbad, t - 1};
    if (w == 2 * kPanel) {
      CK(prep128(r, c, C->aux, Pn[t & 1], gc));
    } else {
      launch_block_inverse<F>(f, R.m, ld, r, c, Pn[t & 1], nullptr, C->aux, false, gc);
      g_launches++;
      CK(cudaGetLastError());
    }
    CK(tc_split_b(*R.fp, Pn[t & 1], w, 0, w, w, tBp[t & 1], C->aux, gc));
    g_launches++;
    CK(cudaMemcpyAsync(h_bad + (t & 1), gbad, sizeof(int), cudaMemcpyDeviceToHost, C->aux));
    CK(cudaEventRecord(C->ev_inv[t & 1], C->aux));
    return MODLIN_OK;
  };

  // W = P^-1 U[.., c1 .. c1+wn) = -(Pn U) into Wbuf (w rows, row stride n,
  // columns c1 .. c1+wn): one launch of (w / 64) x (wn / 64) products with
  // inner dimension w.
  auto make_w = [&](const uint64_t* Pt, int r0, int w, int c1, int wn, const Guard& g) -> int {
    SgProb pr[4];
    int np = 0;
    for (int i = 0; i < w / kPanel; ++i)
      for (int j = 0; j < wn / kPanel; ++j)
        pr[np++] = {Pt + (int64_t)i * kPanel * w, R.m + (int64_t)r0 * ld + c1 + j * kPanel, nullptr,
                    Wbuf + (int64_t)i * kPanel * n + c1 + j * kPanel, w, ld, 0, n, 1, w};
    launch_small_gemm64_batch<F>(f, pr, np, st, g);
    g_launches++;
    return cuda_rc(cudaGetLastError());
  };

  const bool fused = tc && tc_limb_out_supported(R.fp->p);  // limb planes from the epilogues
  auto width = [&](int r, int c) -> int {
    if (!tc) return 0;
    if (n - r >= R.two_panel_min && n - c >= 2 * kPanel && n - r >= 2 * kPanel) return 2 * kPanel;
    if (n - c >= kPanel && n - r >= kPanel) return kPanel;
    return 0;
  };

  double trailing_macs = 0;
  // Block steps from (rank_io, col_io) while width() allows; returns with
  // rank_io/col_io at the first panel they did not take and `failed` set
  // when that panel's block was singular (it then takes the general path).
  auto run_pipeline = [&](int& rank_io, int& col_io, bool& failed) -> int {
    failed = false;
    CK(cudaMemsetAsync(gbad, 0x7f, sizeof(int), st));  // no step has failed
    CK(cudaEventRecord(C->ev_narrow, st));
    CK(cudaStreamWaitEvent(C->aux, C->ev_narrow, 0));
    int t = 0, r0 = rank_io, c0 = col_io, w = width(r0, c0);
    if (int rc = chain(0, r0, c0, w)) return rc;
    CK(tc_split_a(*R.fp, R.m + c0, ld, 0, r0 + w, n, w, tX[0], st));
    g_launches++;
    for (;;) {
      const int r1 = r0 + w, c1 = c0 + w;
      const int wn = r1 < n ? width(r1, c1) : 0;  // the next step's width (0: none)
      const int cw = c1 + wn;                      // first column of the wide update
      const Guard g{gbad, t};
      const uint64_t* Pt = Pn[t & 1];
      CK(cudaStreamWaitEvent(st, C->ev_inv[t & 1], 0));
      if (wn > 0) {
        if (int rc = make_w(Pt, r0, w, c1, wn, g)) return rc;
        CK(tc_split_b(*R.fp, Wbuf, n, c1, cw, w, tBn, st, g));
        // Over 2^61 - 1 the narrow update also writes the next step's X
        // (its rows from r1 + wn) as limb planes.
        LimbOut lx;
        if (fused) lx = LimbOut{tX[(t + 1) & 1], r1 + wn, wn > kPanel ? 2 * kPanel : kPanel, 0};
        CK(tc_update(*R.fp, R.m, ld, r1, n, c1, cw, w, tX[t & 1], tBn, C->num_sms, terr, st, g, lx));
        CK(cudaEventRecord(C->ev_narrow, st));
        CK(cudaStreamWaitEvent(C->aux, C->ev_narrow, 0));
        if (int rc = chain(t + 1, r1, c1, wn)) return rc;
        if (!fused) {
          CK(tc_split_a(*R.fp, R.m + c1, ld, 0, r1 + wn, n, wn, tX[(t + 1) & 1], st, g));
          g_launches++;
        }
        g_launches += 2;
      }
      if (r1 < n && cw < n) {
        // H = X P^-1 = 0 - X (-P^-1) for the rows r1 .. n (relative rows
        // w .. n - r0), as the wide update's A operand. Over 2^61 - 1 the
        // product writes H's limb planes directly; otherwise H goes through
        // Hb and a split.
        // With a chain running, one SM stays free for it (a CTA waiting for
        // that SM would hold up the whole product).
        const int ctas = wn > 0 ? C->num_sms - 1 : C->num_sms;
        if (fused) {
          const LimbOut lh{tA, w, w > kPanel ? 2 * kPanel : kPanel, 1};
          CK(tc_update(*R.fp, Hb, w, w, n - r0, 0, w, w, tX[t & 1], tBp[t & 1], ctas, terr, st, g, lh));
        } else {
          launch_zero(Hb + (size_t)w * w, (int64_t)(n - r1) * w, st, g);
          CK(tc_update(*R.fp, Hb, w, w, n - r0, 0, w, w, tX[t & 1], tBp[t & 1], ctas, terr, st, g));
          CK(tc_split_a(*R.fp, Hb, w, 0, w, n - r0, w, tA, st, g));
          g_launches += 2;
        }
        auto evp = take_events();
        cudaEventRecord(evp.first, st);
        CK(tc_split_b(*R.fp, R.m + (int64_t)r0 * ld, ld, cw, n, w, tB, st, g));
        CK(tc_update(*R.fp, R.m, ld, r1, n, cw, n, w, tA, tB, ctas, terr, st, g));
        cudaEventRecord(evp.second, st);
        g_launches += 3;
      }
      // Step t's chain result (the GPU has step t queued meanwhile).
      CK(cudaEventSynchronize(C->ev_inv[t & 1]));
      if (h_bad[t & 1] <= t) {
        // P_t is singular: nothing of step t (nor chain t + 1) took effect.
        failed = true;
        if (wn > 0) CK(cudaStreamWaitEvent(st, C->ev_inv[(t + 1) & 1], 0));
        rank_io = r0;
        col_io = c0;
        return MODLIN_OK;
      }
      if (R.pcols)
        for (int k = 0; k < w; ++k) R.pcols->push_back(c0 + k);
      if (r1 < n && cw < n) trailing_macs += (double)(n - r1) * (n - cw) * w;
      if (R.cb) R.cb(R.cb_ctx, (size_t)c1, (size_t)n);
      if (wn == 0) {
        rank_io = r1;
        col_io = c1;
        return MODLIN_OK;
      }
      r0 = r1;
      c0 = c1;
      w = wn;
      ++t;
    }
  };

  int rank = 0, col = 0;
  bool general_next = false;  // the panel at col had a singular block
  while (col < n && rank < n) {
    if (!general_next && width(rank, col) > 0) {
      if (int rc = run_pipeline(rank, col, general_next)) return rc;
      continue;
    }
    general_next = false;
    const int jend = std::min(col + kPanel, n);
    const int W = jend - col;
    const int r0 = rank;
    CK(cudaMemsetAsync(ps, 0, sizeof(PanelState), st));
    g_launches++;
    int round = 0, pb_lo = 0;
    PanelState* h = C->h_ps;
    for (;;) {
      launch_window<F>(f, R.m, ld, n, r0, col, W, round, ps, Upanel, G, Lbuf, ispiv, st);
      launch_bulk<F>(f, R.m, ld, n, r0, col, W, pb_lo, ps, Upanel, Lbuf, ispiv, C->num_sms, st);
      g_launches += 2;
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h, ps, sizeof(PanelState), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (h->ncand == 0) break;
      if (h->pb >= W || ++round > kPanel + 1) {
        // A residual with every panel column pivoted is impossible; report
        // it instead of looping.
        return MODLIN_ECUDA;
      }
      pb_lo = h->pb;
    }
    const int pb = h->pb;
    for (int k = 0; k < pb; ++k)
      if (R.pcols) R.pcols->push_back(h->pcol[k]);
    if (pb > 0 && jend < n) {
      launch_couple<F>(f, R.m, ld, n, jend, ps, G, Ubuf, n, st);
      g_launches++;
      // Compaction: pivot rows leave [r0 + pb, n).
      std::vector<char> piv_in_top(pb, 0);
      std::vector<int> holes;
      for (int k = 0; k < pb; ++k) {
        const int r = h->prow[k];
        if (r >= r0 + pb)
          holes.push_back(r);
        else
          piv_in_top[r - r0] = 1;
      }
      int nm = 0;
      for (int t = 0, hi = 0; t < pb; ++t)
        if (!piv_in_top[t]) C->h_moves[nm++] = make_int2(r0 + t, holes[hi++]);
      if (nm > 0) {
        CK(cudaMemcpyAsync(d_moves, C->h_moves, sizeof(int2) * nm, cudaMemcpyHostToDevice, st));
        launch_moves(R.m, ld, n, jend, d_moves, nm, Lbuf, r0, pb, st);
        g_launches++;
      }
      auto evp = take_events();
      cudaEventRecord(evp.first, st);
      trailing_macs += (double)(n - r0 - pb) * (n - jend) * pb;
      if (tc) {
        CK(launch_trailing_tc(*R.fp, R.m, ld, r0 + pb, n, jend, n, Lbuf, kPanel, r0, Ubuf, n, pb, C->tcA.as<uint8_t>(),
                              C->tcB.as<uint8_t>(), C->num_sms, C->tcerr.as<int>(), st));
        g_launches += 3;
      } else {
        launch_trailing_plain<F>(f, R.m, ld, r0 + pb, n, jend, n, Lbuf, r0, Ubuf, n, pb, C->tcerr.as<int>(), st);
        g_launches++;
      }
      cudaEventRecord(evp.second, st);
      CK(cudaGetLastError());
    }
    if (pb > 0) {
      launch_clear_flags(ps, ispiv, st);
      g_launches++;
    }
    rank += pb;
    col = jend;
    if (R.cb) R.cb(R.cb_ctx, (size_t)col, (size_t)n);
  }
  CK(cudaStreamSynchronize(st));
  {
    int err = 0;
    CK(cudaMemcpy(&err, C->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return MODLIN_ETIMEOUT;
  }
  double tms = 0;
  for (size_t i = 0; i < ev_used; ++i) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, C->ev[2 * i], C->ev[2 * i + 1]) == cudaSuccess) tms += ms;
  }
  g_last_trailing_ms = tms;
  g_last_trailing_macs = trailing_macs;
  *rank_out = (size_t)rank;
  return MODLIN_OK;
}

static int rank_device_locked(Ctx* C, uint64_t p, uint64_t* d_m, size_t n, const modlin_rank_opts* opts,
                              size_t* rank_out, size_t* pivot_cols_out, cudaStream_t st, modlin_progress_fn cb,
                              void* cb_ctx) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (n == 0 || n > 0x7fffffff / 2) return MODLIN_EINVAL_N;
  if (!rank_out) return MODLIN_EINVAL_ARG;
  std::vector<int> pc;
  RankRun R{&fp, d_m, (int)n, opts ? opts->kernel : MODLIN_RANK_AUTO, st, C, pivot_cols_out ? &pc : nullptr,
            cb, cb_ctx, C->tune.two_panel_min};
  const int rc = p == kM61 ? rank_impl<FpM61>(R, rank_out) : rank_impl<FpBarrett>(R, rank_out);
  if (rc != MODLIN_OK) return rc;
  if (pivot_cols_out) {
    std::sort(pc.begin(), pc.end());
    for (size_t i = 0; i < pc.size(); ++i) pivot_cols_out[i] = (size_t)pc[i];
  }
  return MODLIN_OK;
}

static bool check_residues(uint64_t p, const uint64_t* x, size_t count) {
  for (size_t i = 0; i < count; ++i)
    if (x[i] >= p) return false;
  return true;
}

// ---------------------------------------------------------------------------
// Linear-complexity drivers.
// ---------------------------------------------------------------------------
static int lc_device_locked(Ctx* C, uint64_t p, const uint64_t* d_s, size_t n, const modlin_lc_opts* opts,
                            size_t* lc_out, cudaStream_t st) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!lc_out) return MODLIN_EINVAL_ARG;
  if (n == 0) {
    *lc_out = 0;
    return MODLIN_OK;
  }
  int kernel = opts ? opts->kernel : MODLIN_LC_AUTO;
  if (kernel == MODLIN_LC_AUTO)
    kernel = (int64_t)n < C->tune.bm_cluster_min ? MODLIN_LC_BLOCK
             : (bm_cluster_size((int64_t)n) ? MODLIN_LC_CLUSTER : MODLIN_LC_GRID);
  if (kernel == MODLIN_LC_CLUSTER) {
    const int R = bm_cluster_size((int64_t)n);
    if (!R) return MODLIN_EINVAL_N;
    CK(C->bmout.ensure(sizeof(int64_t) * 4));
    CK(C->bmws.ensure((size_t)2 * n * 8));
    uint64_t* b0 = C->bmws.as<uint64_t>();
    CK(launch_bm_cluster(fp, d_s, (int64_t)n, R, b0, b0 + n, C->bmout.as<int64_t>(), st));
    g_launches++;
    CK(cudaMemcpyAsync(C->h_out, C->bmout.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *lc_out = (size_t)C->h_out[0];
    return MODLIN_OK;
  }
  CK(C->bmout.ensure(sizeof(int64_t) * 4));
  int64_t* d_out = C->bmout.as<int64_t>();
  if (kernel == MODLIN_LC_BLOCK) {
    const int64_t smem_words = (200 * 1024) / 8;
    if (3 * (int64_t)n > smem_words) CK(C->bmws.ensure((size_t)3 * n * 8));
    BmJob job{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_s, (int64_t)n, 0};
    CK(launch_bm_block(job, C->bmws.as<uint64_t>(), smem_words, C->tune.bm_threads[bm_len_class(n)], d_out, st));
    g_launches++;
  } else {
    int ctas = opts && opts->grid_ctas > 0 ? opts->grid_ctas : C->num_sms;
    // Each CTA keeps its slice of c in shared memory (<= 200 KiB).
    const int64_t min_ctas = ((int64_t)n * 8 + 200 * 1024 - 1) / (200 * 1024);
    if (ctas < min_ctas) ctas = (int)min_ctas;
    if ((int64_t)ctas > (int64_t)n) ctas = (int)n;
    CK(C->bmws.ensure((size_t)2 * n * 8));
    CK(C->bmsync.ensure(grid_sync_bytes()));
    CK(cudaMemsetAsync(C->bmsync.p, 0, grid_sync_bytes(), st));
    uint64_t* b0 = C->bmws.as<uint64_t>();
    int used = 0;
    // About one second of spinning at ~2 GHz before a wait is declared stuck.
    long long spin = 2000000000LL;
    const int skip_cta = g_fault_skip_cta.exchange(-1);
    if (skip_cta >= 0) spin = g_fault_spin.load();
    CK(launch_bm_grid(fp, d_s, (int64_t)n, ctas, 256, b0, b0 + n, C->bmsync.p, spin, skip_cta, d_out, st, &used));
    g_launches += 2;
    int err = 0;
    CK(cudaMemcpyAsync(&err, C->bmsync.as<char>() + grid_sync_err_offset(), sizeof(int), cudaMemcpyDeviceToHost,
                       st));
    CK(cudaStreamSynchronize(st));
    if (err) return MODLIN_ETIMEOUT;
  }
  CK(cudaMemcpyAsync(C->h_out, d_out, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *lc_out = (size_t)C->h_out[0];
  return MODLIN_OK;
}

// Batched rank: jobs up to kRankBatchMaxN go into one persistent launch
// (largest first), larger ones through the single-matrix engine afterwards.
static int rank_batch_locked(Ctx* C, const uint64_t* p, uint64_t* const* d_m, const size_t* n, size_t count,
                             size_t* ranks_out, cudaStream_t st, std::unique_lock<std::mutex>& g,
                             int kernel = MODLIN_RANK_AUTO) {
  if (count == 0) return MODLIN_OK;
  std::vector<RankJob> jobs;
  std::vector<size_t> big;
  int64_t maxn = 0;
  for (size_t i = 0; i < count; ++i) {
    if (n[i] == 0) {
      ranks_out[i] = 0;
      continue;
    }
    if ((int64_t)n[i] > kRankBatchMaxN) {
      big.push_back(i);
      continue;
    }
    FieldParams fp;
    make_field_params(p[i], &fp);
    jobs.push_back(RankJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_m[i], (int64_t)n[i], (int64_t)i});
    maxn = std::max<int64_t>(maxn, (int64_t)n[i]);
  }
  if (!jobs.empty()) {
    // Largest first (work ~ n^3): the persistent CTAs then finish together.
    // Sides from the tuned threshold on go to the tensor-core kernel, the rest to
    // the integer-pipe kernel, one launch each on the same stream.
    std::stable_sort(jobs.begin(), jobs.end(), [](const RankJob& a, const RankJob& b) { return a.n > b.n; });
    const int64_t tc_min = kernel == MODLIN_RANK_TC ? 0 : kernel == MODLIN_RANK_PLAIN ? INT64_MAX
                                                                                        : C->tune.batch_tc_min;
    size_t ntc = 0;
    while (ntc < jobs.size() && jobs[ntc].n >= tc_min) ++ntc;
    CK(C->rbjobs.ensure(sizeof(RankJob) * jobs.size()));
    CK(C->bmnext.ensure(2 * sizeof(unsigned long long)));
    CK(C->rbout.ensure(sizeof(int64_t) * count));
    CK(C->tcerr.ensure(2 * sizeof(int)));
    CK(cudaMemsetAsync(C->tcerr.p, 0, 2 * sizeof(int), st));
    CK(cudaMemcpyAsync(C->rbjobs.p, jobs.data(), sizeof(RankJob) * jobs.size(), cudaMemcpyHostToDevice, st));
    if (ntc > 0) {
      const int per_sm = rank_batch_tc_blocks_per_sm(jobs[0].n);
      if (per_sm < 1) return MODLIN_ECUDA;
      const int blocks = (int)std::min<int64_t>((int64_t)C->num_sms * per_sm, (int64_t)ntc);
      CK(launch_rank_batch_tc(C->rbjobs.as<RankJob>(), (int64_t)ntc, C->bmnext.as<unsigned long long>(), jobs[0].n,
                              blocks, C->rbout.as<int64_t>(), C->tcerr.as<int>(), st));
      g_launches += 2;
    }
    if (ntc < jobs.size()) {
      const int64_t mx = jobs[ntc].n;
      int per_sm = rank_batch_blocks_per_sm(mx);
      if (per_sm < 1) return MODLIN_ECUDA;
      int blocks = C->num_sms * per_sm;
      if ((size_t)blocks > jobs.size() - ntc) blocks = (int)(jobs.size() - ntc);
      CK(launch_rank_batch(C->rbjobs.as<RankJob>() + ntc, (int64_t)(jobs.size() - ntc),
                           C->bmnext.as<unsigned long long>() + 1, mx, blocks, C->rbout.as<int64_t>(), st));
      g_launches += 2;
    }
    std::vector<int64_t> out(count);
    CK(cudaMemcpyAsync(out.data(), C->rbout.p, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, st));
    int err = 0;
    CK(cudaMemcpyAsync(&err, C->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) return MODLIN_ETIMEOUT;
    for (const RankJob& j : jobs) ranks_out[j.slot] = (size_t)out[j.slot];
  }
  if (!big.empty()) {
    g.unlock();
    for (size_t i : big) {
      const int rc2 = modlin_rank_device(p[i], d_m[i], n[i], nullptr, &ranks_out[i], nullptr, st);
      if (rc2) return rc2;
    }
    g.lock();
  }
  return MODLIN_OK;
}

static int lc_batch_locked(Ctx* C, const uint64_t* p, const uint64_t* const* d_data, const size_t* n,
                           size_t count, size_t* lcs_out, cudaStream_t st) {
  if (count == 0) return MODLIN_OK;
  std::vector<BmJob> jobs(count);
  int64_t maxn = 0;
  for (size_t i = 0; i < count; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    jobs[i] = BmJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_data[i], (int64_t)n[i], (int64_t)i};
    maxn = std::max<int64_t>(maxn, (int64_t)n[i]);
  }
  // Longest first: the persistent CTAs then finish close together (LPT).
  std::stable_sort(jobs.begin(), jobs.end(), [](const BmJob& a, const BmJob& b) { return a.n > b.n; });
  const int threads = C->tune.bm_batch_threads[bm_batch_class(maxn)];
  int64_t smem_words = std::min<int64_t>(3 * maxn, (int64_t)C->tune.bm_batch_smem_kib[bm_batch_class(maxn)] * 128);
  int per_sm = bm_batch_max_blocks_per_sm(threads, smem_words);
  if (per_sm < 1) per_sm = 1;
  int blocks = C->num_sms * per_sm;
  if ((size_t)blocks > count) blocks = (int)count;
  const int64_t gws_words = 3 * maxn > smem_words ? 3 * maxn : 0;
  if (gws_words) CK(C->bmws.ensure((size_t)blocks * gws_words * 8));
  CK(C->bmjobs.ensure(sizeof(BmJob) * count));
  CK(C->bmnext.ensure(sizeof(unsigned long long)));
  CK(C->bmout.ensure(sizeof(int64_t) * count));
  CK(cudaMemcpyAsync(C->bmjobs.p, jobs.data(), sizeof(BmJob) * count, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(C->bmnext.p, 0, sizeof(unsigned long long), st));
  CK(launch_bm_batch(C->bmjobs.as<BmJob>(), (int64_t)count, C->bmnext.as<unsigned long long>(),
                     C->bmws.as<uint64_t>(), gws_words, smem_words, blocks, threads, C->bmout.as<int64_t>(), st));
  g_launches += 2;
  std::vector<int64_t> out(count);
  CK(cudaMemcpyAsync(out.data(), C->bmout.p, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < count; ++i) lcs_out[i] = (size_t)out[i];
  return MODLIN_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: measures the AUTO choices on this device (CUDA events on the
// library stream, best of a few runs) and stores them in the context.
// ---------------------------------------------------------------------------
template <class Fn>
static float best_ms(Ctx* C, int reps, Fn&& fn, int* rc_out) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(a, C->stream);
    const int rc = fn();
    cudaEventRecord(b, C->stream);
    cudaEventSynchronize(b);
    if (rc != MODLIN_OK) {
      *rc_out = rc;
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

// Smallest candidate from which `faster` holds for it and every larger one
// (sizes ascending); `none` when it never does.
static int crossover(const std::vector<int>& sizes, const std::vector<bool>& faster, int none) {
  int cross = none;
  for (int i = (int)sizes.size() - 1; i >= 0 && faster[i]; --i) cross = sizes[i];
  return cross;
}

// A failed step leaves its name and the CUDA error in the report.
#define TK(expr)                                                                        \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) {                                                            \
      rep += std::string("\"error\": \"") + #expr + ": " + cudaGetErrorName(_e) + "\"}"; \
      return cuda_rc(_e);                                                               \
    }                                                                                   \
  } while (0)

// Timings in the tuner's JSON report: a non-finite value (a failed or
// unmeasurable timing) is written as -1 so that the report stays valid JSON.
static double finite_ms(double t) { return std::isfinite(t) ? t : -1.0; }

static int autotune_locked(Ctx* C, std::string& rep) {
  int rc = MODLIN_OK;
  cudaStream_t st = C->stream;
  Tune T = C->tune;
  char buf[256];
  rep = "{";
  // 1. Plain vs tensor-core rank per limb count (uniform matrices).
  const uint64_t primes[4] = {127, 65521, 2147483647ULL, kM61};
  const std::vector<int> sizes = {64, 96, 128, 192, 256, 384, 512, 768, 1024};
  const int nmax = 16384;  // largest side measured (two-panel steps)
  TK(C->tunebuf.ensure((size_t)nmax * nmax * 8));
  TK(C->mat.ensure((size_t)nmax * nmax * 8));
  uint64_t* pristine = C->tunebuf.as<uint64_t>();
  uint64_t* work = C->mat.as<uint64_t>();
  rep += "\"rank_ms\": {";
  for (int li = 0; li < 4; ++li) {
    const uint64_t p = primes[li];
    std::vector<bool> tc_wins;
    for (int n : sizes) {
      uint64_t nl = 0;
      TK(gen_uniform_device(p, 1234 + n, pristine, (uint64_t)n * n, st, &nl));
      float t[2];
      for (int k = 0; k < 2; ++k) {
        const modlin_rank_opts o{k == 0 ? MODLIN_RANK_PLAIN : MODLIN_RANK_TC, 0};
        size_t r = 0;
        t[k] = best_ms(C, 2, [&]() -> int {
          if (cudaMemcpyAsync(work, pristine, (size_t)n * n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return MODLIN_ECUDA;
          return rank_device_locked(C, p, work, n, &o, &r, nullptr, st, nullptr, nullptr);
        }, &rc);
        if (rc) return rc;
      }
      tc_wins.push_back(t[1] <= t[0]);
      std::snprintf(buf, sizeof buf, "%s\"%d-limb n=%d\": [%.3f, %.3f]", rep.back() == '{' ? "" : ", ",
                    1 << li, n, finite_ms(t[0]), finite_ms(t[1]));
      rep += buf;
    }
    T.tc_cross[li] = crossover(sizes, tc_wins, 1 << 30);
  }
  rep += "}";
  // 2. The remaining-block size below which one-panel steps replace
  //    two-panel steps, measured directly on the largest rank (tensor cores,
  //    2^61 - 1): the late steps' exposed block chain decides it.
  {
    const std::vector<int> thr = {0, 2048, 4096, 6144, 8192, 12288, 1 << 30};
    rep += ", \"two_panel_ms\": {";
    const int saved = C->tune.two_panel_min;
    const int n = nmax;
    uint64_t nl = 0;
    TK(gen_uniform_device(kM61, 99 + n, pristine, (uint64_t)n * n, st, &nl));
    float best = 0;
    int best_thr = saved;
    for (size_t q = 0; q < thr.size(); ++q) {
      C->tune.two_panel_min = thr[q];
      const modlin_rank_opts o{MODLIN_RANK_TC, 0};
      size_t r = 0;
      const float t = best_ms(C, 2, [&]() -> int {
        if (cudaMemcpyAsync(work, pristine, (size_t)n * n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
          return MODLIN_ECUDA;
        return rank_device_locked(C, kM61, work, n, &o, &r, nullptr, st, nullptr, nullptr);
      }, &rc);
      if (rc) {
        C->tune.two_panel_min = saved;
        return rc;
      }
      if (q == 0 || t < best) {
        best = t;
        best_thr = thr[q];
      }
      std::snprintf(buf, sizeof buf, "%s\"below %d\": %.3f", q == 0 ? "" : ", ", thr[q], finite_ms(t));
      rep += buf;
    }
    C->tune.two_panel_min = saved;
    rep += "}";
    T.two_panel_min = best_thr;
  }
  // 3. Batched rank: tensor-core kernel against the integer-pipe kernel, per
  //    side (a batch of two matrices per SM, 2^61 - 1).
  {
    const std::vector<int> bsz = {128, 256, 512, 1024};
    std::vector<bool> tc_wins;
    const int cnt = 2 * C->num_sms;
    rep += ", \"batch_tc_ms\": {";
    const int saved = C->tune.batch_tc_min;
    for (int n : bsz) {
      const size_t nn = (size_t)n * n;
      TK(C->tunebuf.ensure((size_t)cnt * nn * 8));
      TK(C->batchm.ensure((size_t)cnt * nn * 8));
      uint64_t nl = 0;
      TK(gen_uniform_device(kM61, 31337 + n, C->tunebuf.as<uint64_t>(), (uint64_t)cnt * nn, st, &nl));
      std::vector<uint64_t> ps(cnt, kM61);
      std::vector<uint64_t*> ptrs(cnt);
      std::vector<size_t> ns(cnt, (size_t)n), out(cnt);
      for (int i = 0; i < cnt; ++i) ptrs[i] = C->batchm.as<uint64_t>() + (size_t)i * nn;
      float t[2];
      for (int k = 0; k < 2; ++k) {
        C->tune.batch_tc_min = k == 0 ? (1 << 30) : 0;
        std::unique_lock<std::mutex> dummy;  // the context lock is already held by the caller
        t[k] = best_ms(C, 2, [&]() -> int {
          if (cudaMemcpyAsync(C->batchm.p, C->tunebuf.p, (size_t)cnt * nn * 8, cudaMemcpyDeviceToDevice, st) !=
              cudaSuccess)
            return MODLIN_ECUDA;
          return rank_batch_locked(C, ps.data(), ptrs.data(), ns.data(), cnt, out.data(), st, dummy);
        }, &rc);
        C->tune.batch_tc_min = saved;
        if (rc) return rc;
      }
      tc_wins.push_back(t[1] <= t[0]);
      std::snprintf(buf, sizeof buf, "%s\"n=%d\": [%.3f, %.3f]", n == bsz[0] ? "" : ", ", n, finite_ms(t[0]),
                    finite_ms(t[1]));
      rep += buf;
    }
    rep += "}";
    T.batch_tc_min = crossover(bsz, tc_wins, 1 << 30);
  }
  // 4. BM: threads per CTA of the block kernel by length class, then the
  //    block/cluster crossover.
  FieldParams fp;
  make_field_params(kM61, &fp);
  const int64_t bm_len[4] = {768, 3072, 12288, 32768};
  const int thr[4] = {128, 256, 512, 1024};
  TK(C->seq.ensure((size_t)65536 * 8));
  TK(C->bmout.ensure(sizeof(int64_t) * 4));
  TK(C->bmws.ensure((size_t)3 * 65536 * 8));
  uint64_t* seq = C->seq.as<uint64_t>();
  const int64_t smem_words = (200 * 1024) / 8;
  rep += ", \"bm_block_ms\": {";
  for (int c = 0; c < 4; ++c) {
    uint64_t nl = 0;
    TK(gen_uniform_device(kM61, 555 + c, seq, (uint64_t)bm_len[c], st, &nl));
    float best = 1e30f;
    for (int t : thr) {
      BmJob job{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, seq, bm_len[c], 0};
      const float ms = best_ms(C, 2, [&]() -> int {
        const cudaError_t e = launch_bm_block(job, C->bmws.as<uint64_t>(), smem_words, t, C->bmout.as<int64_t>(), st);
        if (e != cudaSuccess) rep += std::string("\"error\": \"bm block t=") + std::to_string(t) + ": " +
                                     cudaGetErrorName(e) + "\", ";
        return e == cudaSuccess ? MODLIN_OK : MODLIN_ECUDA;
      }, &rc);
      if (rc) return rc;
      std::snprintf(buf, sizeof buf, "%s\"n=%lld t=%d\": %.3f", rep.back() == '{' ? "" : ", ",
                    (long long)bm_len[c], t, finite_ms(ms));
      rep += buf;
      if (ms < best) {
        best = ms;
        T.bm_threads[c] = t;
      }
    }
  }
  rep += "}, \"bm_cluster_ms\": {";
  {
    const std::vector<int> csz = {4096, 8192, 16384, 32768, 65536};
    std::vector<bool> cl_wins;
    for (int n : csz) {
      uint64_t nl = 0;
      TK(gen_uniform_device(kM61, 777 + n, seq, (uint64_t)n, st, &nl));
      BmJob job{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, seq, n, 0};
      const int tb = T.bm_threads[bm_len_class(n)];
      const float tblk = best_ms(C, 1, [&]() -> int {
        return launch_bm_block(job, C->bmws.as<uint64_t>(), smem_words, tb, C->bmout.as<int64_t>(), st) ==
                       cudaSuccess
                   ? MODLIN_OK
                   : MODLIN_ECUDA;
      }, &rc);
      if (rc) return rc;
      const float tcl = best_ms(C, 1, [&]() -> int {
        uint64_t* b0 = C->bmws.as<uint64_t>();
        const cudaError_t e = launch_bm_cluster(fp, seq, n, bm_cluster_size(n), b0, b0 + n, C->bmout.as<int64_t>(), st);
        if (e != cudaSuccess) rep += std::string("\"error\": \"bm cluster n=") + std::to_string(n) + ": " +
                                     cudaGetErrorName(e) + "\", ";
        return e == cudaSuccess ? MODLIN_OK : MODLIN_ECUDA;
      }, &rc);
      if (rc) return rc;
      cl_wins.push_back(tcl <= tblk);
      std::snprintf(buf, sizeof buf, "%s\"n=%d\": [%.3f, %.3f]", n == csz[0] ? "" : ", ", n, finite_ms(tblk),
                    finite_ms(tcl));
      rep += buf;
    }
    T.bm_cluster_min = crossover(csz, cl_wins, 1 << 30);
  }
  rep += "}";
  // 5. BM batches: threads per CTA and the shared-memory cap per CTA by the
  //    longest sequence.
  {
    const int64_t lo[3] = {64, 512, 2048}, hi[3] = {512, 2048, 8192};
    const int bthr[3] = {128, 256, 512};
    const int count = C->num_sms * 6;
    std::vector<size_t> ns(count);
    std::vector<const uint64_t*> ptrs(count);
    std::vector<uint64_t> ps(count, kM61);
    std::vector<size_t> out(count);
    TK(C->tunebuf.ensure((size_t)count * 8192 * 8));
    uint64_t* arena = C->tunebuf.as<uint64_t>();
    uint64_t nl = 0;
    TK(gen_uniform_device(kM61, 4242, arena, (uint64_t)count * 8192, st, &nl));
    rep += ", \"bm_batch_ms\": {";
    for (int c = 0; c < 3; ++c) {
      uint64_t z = 0x1234 + c;
      for (int i = 0; i < count; ++i) {
        z = z * 6364136223846793005ULL + 1442695040888963407ULL;
        ns[i] = (size_t)(lo[c] + (int64_t)((z >> 33) % (uint64_t)(hi[c] - lo[c])));
        ptrs[i] = arena + (size_t)i * 8192;
      }
      float best = 1e30f;
      const int saved = C->tune.bm_batch_threads[c], saved_kib = C->tune.bm_batch_smem_kib[c];
      for (int kib : {200, 96, 48, 24}) {
        if (kib < 200 && (int64_t)kib * 1024 >= 24 * hi[c]) continue;  // the same as a larger cap
        for (int t : bthr) {
          C->tune.bm_batch_threads[c] = t;
          C->tune.bm_batch_smem_kib[c] = kib;
          const float ms = best_ms(C, 1, [&]() -> int {
            return lc_batch_locked(C, ps.data(), ptrs.data(), ns.data(), count, out.data(), st);
          }, &rc);
          if (rc) {
            C->tune.bm_batch_threads[c] = saved;
            C->tune.bm_batch_smem_kib[c] = saved_kib;
            return rc;
          }
          std::snprintf(buf, sizeof buf, "%s\"max<%lld t=%d smem=%dK\": %.3f", rep.back() == '{' ? "" : ", ",
                        (long long)hi[c], t, kib, finite_ms(ms));
          rep += buf;
          if (ms < best) {
            best = ms;
            T.bm_batch_threads[c] = t;
            T.bm_batch_smem_kib[c] = kib;
          }
        }
      }
      C->tune.bm_batch_threads[c] = saved;
      C->tune.bm_batch_smem_kib[c] = saved_kib;
    }
    rep += "}";
  }
  T.measured = true;
  C->tune = T;
  std::snprintf(buf, sizeof buf,
                ", \"choice\": {\"tc_crossover\": [%d, %d, %d, %d], \"two_panel_min\": %d, "
                "\"batch_tc_min\": %d, \"bm_threads\": [%d, %d, %d, %d], \"bm_cluster_min\": %d, "
                "\"bm_batch_threads\": [%d, %d, %d], \"bm_batch_smem_kib\": [%d, %d, %d]}}",
                T.tc_cross[0], T.tc_cross[1], T.tc_cross[2], T.tc_cross[3], T.two_panel_min, T.batch_tc_min,
                T.bm_threads[0], T.bm_threads[1], T.bm_threads[2], T.bm_threads[3], T.bm_cluster_min,
                T.bm_batch_threads[0], T.bm_batch_threads[1], T.bm_batch_threads[2], T.bm_batch_smem_kib[0],
                T.bm_batch_smem_kib[1], T.bm_batch_smem_kib[2]);
  rep += buf;
  return MODLIN_OK;
}

// Pivot structure of one panel (the reference's in-panel elimination,
// src/fp.rs:146-178): the window and bulk kernels of the general path run on
// a copy of the rows x W panel, in the panel's row order.
template <class F>
static int panel_pivots_locked(Ctx* C, const F& f, const uint64_t* d_panel, size_t ld, size_t rows, size_t W,
                               size_t* prow_out, size_t* pcol_out, size_t* pb_out, cudaStream_t st) {
  CK(C->mat.ensure(rows * kPanel * 8));
  CK(C->lbuf.ensure(std::max(C->lbuf.bytes, rows * kPanel * 8)));
  CK(C->upanel.ensure((size_t)kPanel * kPanel * 8));
  CK(C->gmat.ensure((size_t)kPanel * kPanel * 8));
  CK(C->pstate.ensure(sizeof(PanelState)));
  CK(C->ispiv.ensure(rows));
  uint64_t* m = C->mat.as<uint64_t>();
  CK(cudaMemcpy2DAsync(m, kPanel * 8, d_panel, ld * 8, W * 8, rows, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemsetAsync(C->ispiv.p, 0, rows, st));
  CK(cudaMemsetAsync(C->pstate.p, 0, sizeof(PanelState), st));
  PanelState* ps = C->pstate.as<PanelState>();
  PanelState* h = C->h_ps;
  const int n = (int)rows;
  int round = 0, pb_lo = 0;
  for (;;) {
    launch_window<F>(f, m, kPanel, n, 0, 0, (int)W, round, ps, C->upanel.as<uint64_t>(), C->gmat.as<uint64_t>(),
                     C->lbuf.as<uint64_t>(), C->ispiv.as<uint8_t>(), st);
    launch_bulk<F>(f, m, kPanel, n, 0, 0, (int)W, pb_lo, ps, C->upanel.as<uint64_t>(), C->lbuf.as<uint64_t>(),
                   C->ispiv.as<uint8_t>(), C->num_sms, st);
    g_launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h, ps, sizeof(PanelState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h->ncand == 0) break;
    if (h->pb >= (int)W || ++round > kPanel + 1) return MODLIN_ECUDA;
    pb_lo = h->pb;
  }
  *pb_out = (size_t)h->pb;
  for (int k = 0; k < h->pb; ++k) {
    prow_out[k] = (size_t)h->prow[k];
    pcol_out[k] = (size_t)h->pcol[k];
  }
  return MODLIN_OK;
}

}  // namespace modlin

using namespace modlin;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* modlin_strerror(int code) {
  switch (code) {
    case MODLIN_OK: return "ok";
    case MODLIN_EINVAL_P: return "modulus must satisfy 2 <= p < 2^63";
    case MODLIN_EINVAL_N: return "invalid size";
    case MODLIN_EINPUT: return "input entry not reduced modulo p";
    case MODLIN_ECUDA: return "CUDA error";
    case MODLIN_ENOMEM: return "out of memory";
    case MODLIN_ETIMEOUT: return "bounded device wait expired";
    case MODLIN_ENODEV: return "no CUDA device";
    case MODLIN_EINVAL_ARG: return "invalid argument";
    default: return "unknown error";
  }
}

int modlin_field_new(uint64_t p, modlin_field* f) {
  FieldParams fp;
  if (!f) return MODLIN_EINVAL_ARG;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  f->p = fp.p;
  f->mu_lo = fp.mu_lo;
  f->mu_hi = fp.mu_hi;
  f->safe_batch = fp.safe_batch;
  return MODLIN_OK;
}

uint64_t modlin_field_reduce_u128(const modlin_field* f, uint64_t hi, uint64_t lo) {
  FieldParams fp{f->p, f->mu_lo, f->mu_hi, f->safe_batch};
  return FpBarrett(fp).reduce(((u128)hi << 64) | lo);
}

uint64_t modlin_field_reduce(const modlin_field* f, uint64_t x) { return modlin_field_reduce_u128(f, 0, x); }

uint64_t modlin_field_mul(const modlin_field* f, uint64_t a, uint64_t b) {
  const u128 t = (u128)a * b;
  return modlin_field_reduce_u128(f, (uint64_t)(t >> 64), (uint64_t)t);
}

int modlin_rank_device(uint64_t p, uint64_t* d_m, size_t n, const modlin_rank_opts* opts, size_t* rank_out,
                       size_t* pivot_cols_out, void* stream) {
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  if (!d_m) return MODLIN_EINVAL_ARG;
  std::lock_guard<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  return rank_device_locked(C, p, d_m, n, opts, rank_out, pivot_cols_out, st, nullptr, nullptr);
}

int modlin_trailing_update_device(uint64_t p, uint64_t* d_C, size_t ldc, size_t M, size_t N, const uint64_t* d_L,
                                  const uint64_t* d_U, size_t ldu, size_t K, int kernel, void* stream) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  const size_t kmax = kernel == MODLIN_RANK_PLAIN ? (size_t)kPanel : (size_t)2 * kPanel;
  if (K > kmax || M > 0x3fffffff || N > 0x3fffffff || ldc < N || ldu < N) return MODLIN_EINVAL_N;
  if ((M && N && K) && (!d_C || !d_L || !d_U)) return MODLIN_EINVAL_ARG;
  if (!M || !N || !K) return MODLIN_OK;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  if (kernel == MODLIN_RANK_PLAIN) {
    CK(C->tcerr.ensure(2 * sizeof(int)));
    CK(cudaMemsetAsync(C->tcerr.p, 0, 2 * sizeof(int), st));
    if (p == kM61)
      launch_trailing_plain<FpM61>(FpM61(fp), d_C, (int64_t)ldc, 0, (int)M, 0, (int)N, d_L, 0, d_U, (int64_t)ldu,
                                   (int)K, C->tcerr.as<int>(), st);
    else
      launch_trailing_plain<FpBarrett>(FpBarrett(fp), d_C, (int64_t)ldc, 0, (int)M, 0, (int)N, d_L, 0, d_U,
                                       (int64_t)ldu, (int)K, C->tcerr.as<int>(), st);
    g_launches++;
    CK(cudaGetLastError());
    int err = 0;
    CK(cudaMemcpyAsync(&err, C->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) return MODLIN_ETIMEOUT;
  } else {
    CK(C->tcA.ensure(tc_a_bytes((int)M)));
    CK(C->tcB.ensure(tc_b_bytes((int)N)));
    CK(C->tcerr.ensure(2 * sizeof(int)));
    CK(cudaMemsetAsync(C->tcerr.p, 0, 2 * sizeof(int), st));
    const int64_t lda = K <= (size_t)kPanel ? kPanel : 2 * kPanel;
    CK(launch_trailing_tc(fp, d_C, (int64_t)ldc, 0, (int)M, 0, (int)N, d_L, lda, 0, d_U, (int64_t)ldu, (int)K,
                          C->tcA.as<uint8_t>(), C->tcB.as<uint8_t>(), C->num_sms, C->tcerr.as<int>(), st));
    g_launches += 3;
    int err = 0;
    CK(cudaMemcpyAsync(&err, C->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) return MODLIN_ETIMEOUT;
  }
  return cuda_rc(cudaStreamSynchronize(st));
}

int modlin_rank_ex(uint64_t p, uint64_t* m, size_t n, const modlin_rank_opts* opts, size_t* rank_out,
                   size_t* pivot_cols_out, modlin_progress_fn cb, void* cb_ctx) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (n == 0 || n > 0x7fffffff / 2 || n > SIZE_MAX / n / 8) return MODLIN_EINVAL_N;
  if (!m || !rank_out) return MODLIN_EINVAL_ARG;
  if (opts && opts->check_input && !check_residues(p, m, n * n)) return MODLIN_EINPUT;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  const size_t bytes = n * n * 8;
  CK(C->mat.ensure(bytes));
  CK(cudaMemcpyAsync(C->mat.p, m, bytes, cudaMemcpyHostToDevice, C->stream));
  return rank_device_locked(C, p, C->mat.as<uint64_t>(), n, opts, rank_out, pivot_cols_out, C->stream, cb, cb_ctx);
}

int modlin_rank(uint64_t p, uint64_t* m, size_t n, size_t* rank_out, modlin_progress_fn cb, void* cb_ctx) {
  return modlin_rank_ex(p, m, n, nullptr, rank_out, nullptr, cb, cb_ctx);
}

int modlin_linear_complexity_device(uint64_t p, const uint64_t* d_s, size_t n, const modlin_lc_opts* opts,
                                    size_t* lc_out, void* stream) {
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  if (!d_s && n) return MODLIN_EINVAL_ARG;
  std::lock_guard<std::mutex> g(C->mu);
  return lc_device_locked(C, p, d_s, n, opts, lc_out, user_stream(stream));
}

int modlin_linear_complexity_ex(uint64_t p, const uint64_t* s, size_t n, const modlin_lc_opts* opts,
                                size_t* lc_out) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!lc_out || (!s && n)) return MODLIN_EINVAL_ARG;
  if (opts && opts->check_input && !check_residues(p, s, n)) return MODLIN_EINPUT;
  if (n == 0) {
    *lc_out = 0;
    return MODLIN_OK;
  }
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  CK(C->seq.ensure(n * 8));
  CK(cudaMemcpyAsync(C->seq.p, s, n * 8, cudaMemcpyHostToDevice, C->stream));
  return lc_device_locked(C, p, C->seq.as<uint64_t>(), n, opts, lc_out, C->stream);
}

int modlin_linear_complexity(uint64_t p, const uint64_t* s, size_t n, size_t* lc_out, modlin_progress_fn cb,
                             void* cb_ctx) {
  const int rc = modlin_linear_complexity_ex(p, s, n, nullptr, lc_out);
  if (rc == MODLIN_OK && cb) cb(cb_ctx, n, n);
  return rc;
}

int modlin_lc_batch_device(const uint64_t* p, const uint64_t* const* d_data, const size_t* n, size_t count,
                           size_t* lcs_out, void* stream) {
  if (count && (!p || !d_data || !n || !lcs_out)) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  return lc_batch_locked(C, p, d_data, n, count, lcs_out, user_stream(stream));
}

int modlin_lc_batch(const modlin_job* jobs, size_t count, size_t* lcs_out) {
  if (count && (!jobs || !lcs_out)) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  size_t total = 0;
  for (size_t i = 0; i < count; ++i) {
    if (!jobs[i].data && jobs[i].n) return MODLIN_EINVAL_ARG;
    total += jobs[i].n;
  }
  CK(C->seq.ensure(std::max<size_t>(total, 1) * 8));
  std::vector<const uint64_t*> ptrs(count);
  std::vector<uint64_t> ps(count);
  std::vector<size_t> ns(count);
  size_t off = 0;
  for (size_t i = 0; i < count; ++i) {
    if (jobs[i].n) CK(cudaMemcpyAsync(C->seq.as<uint64_t>() + off, jobs[i].data, jobs[i].n * 8,
                                      cudaMemcpyHostToDevice, C->stream));
    ptrs[i] = C->seq.as<uint64_t>() + off;
    ps[i] = jobs[i].p;
    ns[i] = jobs[i].n;
    off += jobs[i].n;
  }
  return lc_batch_locked(C, ps.data(), ptrs.data(), ns.data(), count, lcs_out, C->stream);
}

int modlin_rank_batch_device_ex(const uint64_t* p, uint64_t* const* d_m, const size_t* n, size_t count,
                                const modlin_rank_opts* opts, size_t* ranks_out, void* stream) {
  if (count && (!p || !d_m || !n || !ranks_out)) return MODLIN_EINVAL_ARG;
  for (size_t i = 0; i < count; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    if (n[i] && !d_m[i]) return MODLIN_EINVAL_ARG;
    if (n[i] > (size_t)INT32_MAX / 2) return MODLIN_EINVAL_N;
  }
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::unique_lock<std::mutex> g(C->mu);
  return rank_batch_locked(C, p, d_m, n, count, ranks_out, user_stream(stream), g,
                           opts ? opts->kernel : MODLIN_RANK_AUTO);
}

int modlin_rank_batch_device(const uint64_t* p, uint64_t* const* d_m, const size_t* n, size_t count,
                             size_t* ranks_out, void* stream) {
  if (count && (!p || !d_m || !n || !ranks_out)) return MODLIN_EINVAL_ARG;
  for (size_t i = 0; i < count; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    if (n[i] && !d_m[i]) return MODLIN_EINVAL_ARG;
    if (n[i] > (size_t)INT32_MAX / 2) return MODLIN_EINVAL_N;
  }
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::unique_lock<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  return rank_batch_locked(C, p, d_m, n, count, ranks_out, st, g);
}

int modlin_rank_batch(const modlin_job* jobs, size_t count, size_t* ranks_out) {
  if (count && (!jobs || !ranks_out)) return MODLIN_EINVAL_ARG;
  size_t total = 0;
  for (size_t i = 0; i < count; ++i) {
    if (!jobs[i].data && jobs[i].n) return MODLIN_EINVAL_ARG;
    if (jobs[i].n > (size_t)INT32_MAX / 2) return MODLIN_EINVAL_N;
    total += jobs[i].n * jobs[i].n;
  }
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::unique_lock<std::mutex> g(C->mu);
  // All matrices copied into one device arena (the inputs stay untouched).
  CK(C->batchm.ensure(std::max<size_t>(total, 1) * 8));
  std::vector<uint64_t*> ptrs(count);
  std::vector<uint64_t> ps(count);
  std::vector<size_t> ns(count);
  size_t off = 0;
  for (size_t i = 0; i < count; ++i) {
    const size_t nn = jobs[i].n * jobs[i].n;
    ptrs[i] = C->batchm.as<uint64_t>() + off;
    if (nn) CK(cudaMemcpyAsync(ptrs[i], jobs[i].data, nn * 8, cudaMemcpyHostToDevice, C->stream));
    ps[i] = jobs[i].p;
    ns[i] = jobs[i].n;
    off += nn;
  }
  return rank_batch_locked(C, ps.data(), ptrs.data(), ns.data(), count, ranks_out, C->stream, g);
}

int modlin_gen_uniform(uint64_t p, uint64_t seed, uint64_t* out, size_t count) {
  if (p < 2) return MODLIN_EINVAL_P;
  if (!out && count) return MODLIN_EINVAL_ARG;
  const int bits = 64 - __builtin_clzll(p - 1);
  uint64_t z = seed;
  for (size_t i = 0; i < count;) {
    z += 0x9e3779b97f4a7c15ULL;
    uint64_t w = z;
    w = (w ^ (w >> 30)) * 0xbf58476d1ce4e5b9ULL;
    w = (w ^ (w >> 27)) * 0x94d049bb133111ebULL;
    w ^= w >> 31;
    const uint64_t x = w >> (64 - bits);
    if (x < p) out[i++] = x;
  }
  return MODLIN_OK;
}

}  // extern "C"

// Planted recurrence parameters from SplitMix64(seed): a_1..a_L (a_L redrawn
// while 0), then the initial values s_0..s_{L-1}, all uniform residues.
static void draw_planted(uint64_t p, size_t L, uint64_t seed, std::vector<uint64_t>& a, std::vector<uint64_t>& init) {
  a.assign(L + 1, 0);
  init.assign(L, 0);
  uint64_t z = seed;
  const int bits = 64 - __builtin_clzll(p - 1);
  auto uni = [&]() {
    for (;;) {
      z += 0x9e3779b97f4a7c15ULL;
      uint64_t w = z;
      w = (w ^ (w >> 30)) * 0xbf58476d1ce4e5b9ULL;
      w = (w ^ (w >> 27)) * 0x94d049bb133111ebULL;
      w ^= w >> 31;
      const uint64_t x = w >> (64 - bits);
      if (x < p) return x;
    }
  };
  for (size_t j = 1; j <= L; ++j) a[j] = uni();
  while (L > 0 && a[L] == 0) a[L] = uni();
  for (size_t i = 0; i < L; ++i) init[i] = uni();
}

extern "C" {

int modlin_gen_planted(uint64_t p, size_t L, uint64_t seed, uint64_t* out, size_t count) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!out && count) return MODLIN_EINVAL_ARG;
  std::vector<uint64_t> a, init;
  draw_planted(p, L, seed, a, init);
  const FpBarrett f(fp);
  const uint64_t sb = fp.safe_batch;
  for (size_t i = 0; i < count; ++i) {
    if (i < L) {
      out[i] = init[i];
      continue;
    }
    u128 acc = 0;
    uint64_t tot = 0, cnt = 0;
    for (size_t j = 1; j <= L; ++j) {
      acc += (u128)a[j] * out[i - j];
      if (++cnt == sb) {
        tot = f.add(tot, f.reduce(acc));
        acc = 0;
        cnt = 0;
      }
    }
    out[i] = f.add(tot, f.reduce(acc));
  }
  return MODLIN_OK;
}

int modlin_gen_planted_batch_device(const uint64_t* p, const size_t* L, const uint64_t* seed, uint64_t* const* d_out,
                                    const size_t* count, size_t njobs, void* stream) {
  if (njobs && (!p || !L || !seed || !d_out || !count)) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  size_t total_a = 0;
  for (size_t i = 0; i < njobs; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    if (!d_out[i] && count[i]) return MODLIN_EINVAL_ARG;
    total_a += L[i];
  }
  std::vector<uint64_t> coeffs;
  coeffs.reserve(total_a);
  std::vector<PlantJob> jobs;
  std::vector<uint64_t> a, init;
  CK(C->gena.ensure(std::max<size_t>(total_a, 1) * 8));
  size_t off = 0;
  for (size_t i = 0; i < njobs; ++i) {
    draw_planted(p[i], L[i], seed[i], a, init);
    coeffs.insert(coeffs.end(), a.begin() + 1, a.end());
    const size_t ncopy = std::min(L[i], count[i]);
    if (ncopy) CK(cudaMemcpyAsync(d_out[i], init.data(), ncopy * 8, cudaMemcpyHostToDevice, st));
    // cudaMemcpyAsync from pageable memory returns after staging the data,
    // so `init` may be reused for the next job.
    FieldParams fp;
    make_field_params(p[i], &fp);
    if (count[i] > L[i])
      jobs.push_back(PlantJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, C->gena.as<uint64_t>() + off, d_out[i],
                              (int64_t)L[i], (int64_t)count[i]});
    off += L[i];
  }
  if (total_a) CK(cudaMemcpyAsync(C->gena.p, coeffs.data(), total_a * 8, cudaMemcpyHostToDevice, st));
  if (!jobs.empty()) {
    CK(C->genjobs.ensure(jobs.size() * sizeof(PlantJob)));
    CK(C->bmnext.ensure(sizeof(unsigned long long)));
    CK(cudaMemcpyAsync(C->genjobs.p, jobs.data(), jobs.size() * sizeof(PlantJob), cudaMemcpyHostToDevice, st));
    size_t maxL = 0;
    for (auto& j : jobs) maxL = std::max<size_t>(maxL, (size_t)j.L);
    const int threads = maxL >= 8192 ? 1024 : (maxL >= 1024 ? 512 : 128);
    int blocks = C->num_sms * (2048 / threads);
    if ((size_t)blocks > jobs.size()) blocks = (int)jobs.size();
    CK(plant_device(C->genjobs.as<PlantJob>(), (int64_t)jobs.size(), C->bmnext.as<unsigned long long>(), blocks,
                    threads, st));
    g_launches += 2;
  }
  return cuda_rc(cudaStreamSynchronize(st));
}

int modlin_gen_planted_device(uint64_t p, size_t L, uint64_t seed, uint64_t* d_out, size_t count, void* stream) {
  // Long streams of a high-order recurrence: jump-ahead segments extended in
  // parallel instead of one CTA walking the whole stream.
  const bool jump = L >= 64 && L <= (1u << 20) && count >= ((size_t)1 << 22) && count >= 256 * L;
  if (!jump) return modlin_gen_planted_batch_device(&p, &L, &seed, &d_out, &count, 1, stream);
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!d_out) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  const int Li = (int)L;
  int K = (int)std::min<size_t>(1024, count / (64 * L));
  const int64_t T = (int64_t)((count + K - 1) / K);
  K = (int)((count + T - 1) / T);
  std::vector<uint64_t> a, init;
  draw_planted(p, L, seed, a, init);
  // Scratch: a (L), head (2L), u (2L), R (K L), xpow (2L), tmp (L), cbuf (2L), qbuf (L).
  const size_t words = (size_t)L * (1 + 2 + 2 + 2 + 1 + 2 + 1) + (size_t)K * L;
  CK(C->jump.ensure(words * 8));
  uint64_t* w = C->jump.as<uint64_t>();
  uint64_t* d_a = w;
  uint64_t* head = d_a + L;
  uint64_t* u = head + 2 * L;
  uint64_t* xpow = u + 2 * L;
  uint64_t* tmp = xpow + 2 * L;
  uint64_t* cbuf = tmp + L;
  uint64_t* qbuf = cbuf + 2 * L;
  uint64_t* R = qbuf + L;
  CK(cudaMemcpyAsync(d_a, a.data() + 1, L * 8, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(head, init.data(), L * 8, cudaMemcpyHostToDevice, st));
  std::vector<uint64_t> impulse(L, 0);
  impulse[L - 1] = 1;
  CK(cudaMemcpyAsync(u, impulse.data(), L * 8, cudaMemcpyHostToDevice, st));
  // head = s[0 .. 2L-1); u[L-1 ..] = g, the power series 1 / (1 - sum a_j x^j).
  std::vector<PlantJob> jobs;
  jobs.push_back(PlantJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_a, head, (int64_t)L, (int64_t)(2 * L - 1)});
  jobs.push_back(PlantJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_a, u, (int64_t)L, (int64_t)(2 * L - 1)});
  CK(C->genjobs.ensure(std::max<size_t>(K, 2) * sizeof(PlantJob)));
  CK(C->bmnext.ensure(sizeof(unsigned long long)));
  CK(cudaMemcpyAsync(C->genjobs.p, jobs.data(), 2 * sizeof(PlantJob), cudaMemcpyHostToDevice, st));
  const int threads = L >= 8192 ? 1024 : 512;
  CK(plant_device(C->genjobs.as<PlantJob>(), 2, C->bmnext.as<unsigned long long>(), 2, threads, st));
  JumpPlan P{d_a, u + (L - 1), head, d_out, R, xpow, tmp, cbuf, qbuf, Li, K, T, (int64_t)count};
  CK(jump_states(fp, P, st));
  // Every segment extended from its state by the recurrence.
  jobs.clear();
  for (int k = 0; k < K; ++k) {
    const int64_t t0 = (int64_t)k * T;
    const int64_t len = std::min<int64_t>(T, (int64_t)count - t0);
    jobs.push_back(PlantJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_a, d_out + t0, (int64_t)L, len});
  }
  // The job table is read by the device after this host vector is reused:
  // wait for the first launch's copies before overwriting the table.
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpyAsync(C->genjobs.p, jobs.data(), jobs.size() * sizeof(PlantJob), cudaMemcpyHostToDevice, st));
  const int blocks = std::min<int>(K, C->num_sms * (2048 / threads));
  CK(plant_device(C->genjobs.as<PlantJob>(), (int64_t)K, C->bmnext.as<unsigned long long>(), blocks, threads, st));
  g_launches += 6 + 3 * (size_t)(K + 40);
  return cuda_rc(cudaStreamSynchronize(st));
}

int modlin_gen_uniform_device(uint64_t p, uint64_t seed, uint64_t* d_out, size_t count, void* stream) {
  if (p < 2) return MODLIN_EINVAL_P;
  if (!d_out && count) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  uint64_t nl = 0;
  cudaError_t e = gen_uniform_device(p, seed, d_out, count, user_stream(stream), &nl);
  g_launches += nl;
  return cuda_rc(e);
}

int modlin_reduce_device(uint64_t p, uint64_t* d_x, size_t count, void* stream) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  cudaStream_t st = user_stream(stream);
  CK(reduce_device(fp, d_x, count, st));
  g_launches++;
  return cuda_rc(cudaStreamSynchronize(st));
}

int modlin_panel_pivots_device(uint64_t p, const uint64_t* d_panel, size_t ld, size_t rows, size_t W,
                               size_t* prow_out, size_t* pcol_out, size_t* pb_out, void* stream) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!pb_out || !prow_out || !pcol_out) return MODLIN_EINVAL_ARG;
  if (W > (size_t)kPanel || ld < W || rows > 0x3fffffff) return MODLIN_EINVAL_N;
  *pb_out = 0;
  if (!rows || !W) return MODLIN_OK;
  if (!d_panel) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  cudaStream_t st = user_stream(stream);
  if (p == kM61) return panel_pivots_locked(C, FpM61(fp), d_panel, ld, rows, W, prow_out, pcol_out, pb_out, st);
  return panel_pivots_locked(C, FpBarrett(fp), d_panel, ld, rows, W, prow_out, pcol_out, pb_out, st);
}

int modlin_block_inverse_device(uint64_t p, const uint64_t* d_P, size_t ldp, uint64_t* d_out, int* singular,
                                 void* stream) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!d_P || !d_out || !singular || ldp < (size_t)kPanel) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g_(C->mu);
  cudaStream_t st = user_stream(stream);
  CK(C->invst.ensure(sizeof(int)));
  if (p == kM61)
    launch_block_inverse<FpM61>(FpM61(fp), d_P, (int64_t)ldp, 0, 0, d_out, C->invst.as<int>(), st, true);
  else
    launch_block_inverse<FpBarrett>(FpBarrett(fp), d_P, (int64_t)ldp, 0, 0, d_out, C->invst.as<int>(), st, true);
  g_launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(C->h_out, C->invst.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *singular = (int)*reinterpret_cast<int*>(C->h_out);
  return MODLIN_OK;
}

int modlin_prng_fill_device(modlin_prng* g, uint64_t p, uint64_t* d_out, size_t count, void* stream) {
  if (!g || (!d_out && count)) return MODLIN_EINVAL_ARG;
  FieldParams fp{};
  if (p && !make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!count) return MODLIN_OK;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g_(C->mu);
  uint64_t nl = 0;
  rc = prng_fill_device(C->prng, C->num_sms, g, p, fp, d_out, count, user_stream(stream), &nl);
  g_launches += nl;
  return rc;
}

int modlin_rank_prng(uint64_t p, modlin_prng* g, size_t n, const modlin_rank_opts* opts, size_t* rank_out,
                     modlin_progress_fn cb, void* cb_ctx) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (n == 0 || n > 0x7fffffff / 2 || n > SIZE_MAX / n / 8) return MODLIN_EINVAL_N;
  if (!g || !rank_out) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g_(C->mu);
  CK(C->mat.ensure(n * n * 8));
  uint64_t nl = 0;
  rc = prng_fill_device(C->prng, C->num_sms, g, p, fp, C->mat.as<uint64_t>(), (uint64_t)n * n, C->stream, &nl);
  g_launches += nl;
  if (rc) return rc;
  return rank_device_locked(C, p, C->mat.as<uint64_t>(), n, opts, rank_out, nullptr, C->stream, cb, cb_ctx);
}

int modlin_rank_prng_batch(uint64_t p, modlin_prng* g, size_t n, size_t reps, const modlin_rank_opts* opts,
                           size_t* ranks_out, modlin_progress_fn cb, void* cb_ctx) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (n == 0 || n > 0x7fffffff / 2 || n > SIZE_MAX / n / 8) return MODLIN_EINVAL_N;
  if (!g || (reps && !ranks_out)) return MODLIN_EINVAL_ARG;
  if (reps == 0) return MODLIN_OK;
  if (reps == 1 || (int64_t)n > kRankBatchMaxN) {
    for (size_t i = 0; i < reps; ++i) {
      const int rc = modlin_rank_prng(p, g, n, opts, ranks_out + i, nullptr, nullptr);
      if (rc) return rc;
      if (cb) cb(cb_ctx, i + 1, reps);
    }
    return MODLIN_OK;
  }
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::unique_lock<std::mutex> lk(C->mu);
  const size_t per = n * n;
  const size_t budget = (size_t)8 << 30;  // bytes of matrices in flight at once
  const size_t chunk = std::max<size_t>(1, std::min(reps, budget / (per * 8)));
  CK(C->repsbuf.ensure(chunk * per * 8));
  uint64_t* arena = C->repsbuf.as<uint64_t>();
  std::vector<uint64_t> ps(chunk, p);
  std::vector<size_t> ns(chunk, n);
  std::vector<uint64_t*> ptrs(chunk);
  for (size_t i = 0; i < chunk; ++i) ptrs[i] = arena + i * per;
  for (size_t done = 0; done < reps; done += chunk) {
    const size_t c = std::min(chunk, reps - done);
    uint64_t nl = 0;
    rc = prng_fill_device(C->prng, C->num_sms, g, p, fp, arena, (uint64_t)(c * per), C->stream, &nl);
    g_launches += nl;
    if (rc) return rc;
    rc = rank_batch_locked(C, ps.data(), ptrs.data(), ns.data(), c, ranks_out + done, C->stream, lk,
                           opts ? opts->kernel : MODLIN_RANK_AUTO);
    if (rc) return rc;
    if (cb) cb(cb_ctx, done + c, reps);
  }
  return MODLIN_OK;
}

uint64_t modlin_kernel_launches(void) { return g_launches.load(); }

int modlin_set_tc_pairs(int enable) {
  const int prev = g_tc_pairs ? 1 : 0;
  if (enable >= 0) g_tc_pairs = enable != 0;
  return prev;
}

int modlin_testing_grid_timeout_once(long long spin_cycles, int skip_cta) {
  if (spin_cycles < 1 || spin_cycles > 4000000000LL || skip_cta < 0) return MODLIN_EINVAL_ARG;
  g_fault_spin.store(spin_cycles);
  g_fault_skip_cta.store(skip_cta);
  return MODLIN_OK;
}

double modlin_last_trailing_ms(void) { return g_last_trailing_ms; }

double modlin_last_trailing_macs(void) { return g_last_trailing_macs; }

int modlin_plain_mac_peak(uint64_t p, double* modmac_per_s) {
  FieldParams fp;
  if (!make_field_params(p, &fp)) return MODLIN_EINVAL_P;
  if (!modmac_per_s) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  const bool m61 = p == kM61;
  const int per_sm = m61 ? plain_blocks_per_sm<FpM61>() : plain_blocks_per_sm<FpBarrett>();
  const int blocks = C->num_sms * (per_sm > 0 ? per_sm : 1);
  const int iters = 64;
  CK(C->bmout.ensure((size_t)blocks * 256 * 8));
  cudaStream_t st = C->stream;
  auto launch = [&]() {
    return m61 ? launch_plain_mac_peak(FpM61(fp), blocks, iters, C->bmout.as<uint64_t>(), st)
               : launch_plain_mac_peak(FpBarrett(fp), blocks, iters, C->bmout.as<uint64_t>(), st);
  };
  CK(launch());  // warm-up
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(e0, st);
    const cudaError_t e = launch();
    cudaEventRecord(e1, st);
    if (e != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return MODLIN_ECUDA;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  g_launches += 4;
  *modmac_per_s = (double)blocks * 256 * 16 * 64 * iters / (best * 1e-3);
  return MODLIN_OK;
}

// ---- Batch plans: device state built once, launches that can be captured.
}  // extern "C"

struct modlin_rank_batch_plan {
  int device;
  int64_t count, ntc;      // jobs, of which the first ntc (largest) on the tensor cores
  int64_t max_tc, max_small;
  int blocks_tc, blocks_small;
  int64_t* out;  // caller's device array
  modlin::DevBuf jobs, next, err;
};

struct modlin_lc_batch_plan {
  int device;
  int64_t count, smem_words, gws_words;
  int blocks, threads;
  int64_t* out;  // caller's device array
  modlin::DevBuf jobs, next, gws;
};

extern "C" {

int modlin_rank_batch_plan_new(const uint64_t* p, uint64_t* const* d_m, const size_t* n, size_t count,
                               int64_t* d_ranks_out, modlin_rank_batch_plan** plan_out) {
  if (!plan_out || (count && (!p || !d_m || !n || !d_ranks_out))) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::vector<RankJob> jobs;
  int64_t maxn = 1;
  for (size_t i = 0; i < count; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    if ((int64_t)n[i] > kRankBatchMaxN) return MODLIN_EINVAL_N;
    if (n[i] && !d_m[i]) return MODLIN_EINVAL_ARG;
    jobs.push_back(RankJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_m[i], (int64_t)n[i], (int64_t)i});
    maxn = std::max<int64_t>(maxn, (int64_t)n[i]);
  }
  (void)maxn;
  std::stable_sort(jobs.begin(), jobs.end(), [](const RankJob& a, const RankJob& b) { return a.n > b.n; });
  std::unique_ptr<modlin_rank_batch_plan> P(new modlin_rank_batch_plan());
  P->device = C->device;
  P->count = (int64_t)count;
  P->out = d_ranks_out;
  P->ntc = 0;
  while (P->ntc < (int64_t)jobs.size() && jobs[P->ntc].n >= C->tune.batch_tc_min) ++P->ntc;
  P->max_tc = P->ntc ? jobs[0].n : 1;
  P->max_small = P->ntc < (int64_t)jobs.size() ? jobs[P->ntc].n : 1;
  const int ptc = rank_batch_tc_blocks_per_sm(P->max_tc), psm = rank_batch_blocks_per_sm(P->max_small);
  if (ptc < 1 || psm < 1) return MODLIN_ECUDA;
  P->blocks_tc = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)C->num_sms * ptc, P->ntc));
  P->blocks_small =
      (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)C->num_sms * psm, (int64_t)count - P->ntc));
  CK(P->jobs.ensure(std::max<size_t>(jobs.size(), 1) * sizeof(RankJob)));
  CK(P->next.ensure(2 * sizeof(unsigned long long)));
  CK(P->err.ensure(2 * sizeof(int)));
  if (count) CK(cudaMemcpy(P->jobs.p, jobs.data(), jobs.size() * sizeof(RankJob), cudaMemcpyHostToDevice));
  *plan_out = P.release();
  return MODLIN_OK;
}

int modlin_rank_batch_plan_launch(modlin_rank_batch_plan* P, void* stream) {
  if (!P) return MODLIN_EINVAL_ARG;
  if (P->count == 0) return MODLIN_OK;
  cudaStream_t st = user_stream(stream);
  // -1 marks a job whose rank was not written (a bounded wait expired).
  CK(cudaMemsetAsync(P->out, 0xff, (size_t)P->count * sizeof(int64_t), st));
  CK(cudaMemsetAsync(P->err.p, 0, 2 * sizeof(int), st));
  if (P->ntc > 0)
    CK(launch_rank_batch_tc(P->jobs.as<RankJob>(), P->ntc, P->next.as<unsigned long long>(), P->max_tc, P->blocks_tc,
                            P->out, P->err.as<int>(), st));
  if (P->ntc < P->count)
    CK(launch_rank_batch(P->jobs.as<RankJob>() + P->ntc, P->count - P->ntc, P->next.as<unsigned long long>() + 1,
                         P->max_small, P->blocks_small, P->out, st));
  g_launches += 4;
  return MODLIN_OK;
}

void modlin_rank_batch_plan_free(modlin_rank_batch_plan* P) {
  if (!P) return;
  cudaFree(P->jobs.p);
  cudaFree(P->next.p);
  cudaFree(P->err.p);
  delete P;
}

int modlin_lc_batch_plan_new(const uint64_t* p, const uint64_t* const* d_s, const size_t* n, size_t count,
                             int64_t* d_lcs_out, modlin_lc_batch_plan** plan_out) {
  if (!plan_out || (count && (!p || !d_s || !n || !d_lcs_out))) return MODLIN_EINVAL_ARG;
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::vector<BmJob> jobs;
  int64_t maxn = 1;
  for (size_t i = 0; i < count; ++i) {
    FieldParams fp;
    if (!make_field_params(p[i], &fp)) return MODLIN_EINVAL_P;
    if (n[i] && !d_s[i]) return MODLIN_EINVAL_ARG;
    if (n[i] > (size_t)1 << 30) return MODLIN_EINVAL_N;
    jobs.push_back(BmJob{fp.p, fp.mu_lo, fp.mu_hi, fp.safe_batch, d_s[i], (int64_t)n[i], (int64_t)i});
    maxn = std::max<int64_t>(maxn, (int64_t)n[i]);
  }
  std::stable_sort(jobs.begin(), jobs.end(), [](const BmJob& a, const BmJob& b) { return a.n > b.n; });
  std::unique_ptr<modlin_lc_batch_plan> P(new modlin_lc_batch_plan());
  P->device = C->device;
  P->count = (int64_t)count;
  P->out = d_lcs_out;
  P->threads = C->tune.bm_batch_threads[bm_batch_class(maxn)];
  P->smem_words = std::min<int64_t>(3 * maxn, (int64_t)C->tune.bm_batch_smem_kib[bm_batch_class(maxn)] * 128);
  const int per_sm = std::max(1, bm_batch_max_blocks_per_sm(P->threads, P->smem_words));
  P->blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)C->num_sms * per_sm, (int64_t)count));
  P->gws_words = 3 * maxn > P->smem_words ? 3 * maxn : 0;
  CK(P->jobs.ensure(std::max<size_t>(jobs.size(), 1) * sizeof(BmJob)));
  CK(P->next.ensure(sizeof(unsigned long long)));
  if (P->gws_words) CK(P->gws.ensure((size_t)P->blocks * P->gws_words * 8));
  if (count) CK(cudaMemcpy(P->jobs.p, jobs.data(), jobs.size() * sizeof(BmJob), cudaMemcpyHostToDevice));
  *plan_out = P.release();
  return MODLIN_OK;
}

int modlin_lc_batch_plan_launch(modlin_lc_batch_plan* P, void* stream) {
  if (!P) return MODLIN_EINVAL_ARG;
  if (P->count == 0) return MODLIN_OK;
  cudaStream_t st = user_stream(stream);
  CK(cudaMemsetAsync(P->next.p, 0, sizeof(unsigned long long), st));
  CK(launch_bm_batch(P->jobs.as<BmJob>(), P->count, P->next.as<unsigned long long>(), P->gws.as<uint64_t>(),
                     P->gws_words, P->smem_words, P->blocks, P->threads, P->out, st));
  g_launches += 2;
  return MODLIN_OK;
}

void modlin_lc_batch_plan_free(modlin_lc_batch_plan* P) {
  if (!P) return;
  cudaFree(P->jobs.p);
  cudaFree(P->next.p);
  cudaFree(P->gws.p);
  delete P;
}

int modlin_autotune(char* report, size_t cap) {
  Ctx* C = nullptr;
  int rc = get_ctx(&C);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(C->mu);
  std::string rep;
  rc = autotune_locked(C, rep);
  if (report && cap) {
    const size_t k = std::min(cap - 1, rep.size());
    std::memcpy(report, rep.data(), k);
    report[k] = 0;
  }
  return rc;
}

}  // extern "C"
