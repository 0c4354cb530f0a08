// Device fill of the generators under test (host declarations): the stream
// of modlin_prng_fill, produced by many warps or threads at once from
// jump-ahead segment states, bit-identical to the sequential host stream.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/modlin.h"
#include "field.cuh"

namespace modlin {

// C[M x N] = A[M x K] * B[K x N] mod 2^61 - 1; row-major, entries in [0, p).
cudaError_t m61_gemm(const uint64_t* A, const uint64_t* B, uint64_t* C, int M, int K, int N, cudaStream_t st);

// One MIXMAX-N fill. State words: [sumtot, v[1], ..., v[N-1]] (v[0] only
// ever holds the previous sumtot and is never read or output). Block b >= 1
// is the state after (skip + 1) * b iterations from the starting state; it
// outputs v[1..N-1]. Block 0 is the starting state itself, whose outputs
// v[c0..N-1] (h0 of them) come first. Segment s covers blocks
// s*G+1 .. min((s+1)*G, nbk), starting from starts[s] = block s*G.
struct MixFill {
  int N;
  uint64_t special;        // MIXMAX-240's multiplier
  const uint64_t* starts;  // S x N
  uint64_t* ends;          // S x (N + 1): block min((s+1)*G, nbk), then v[0]
  int* flags;              // flags[s] = 1: segment s-1 ended on an entry 2^61 - 1
  int* any;                // count of flags set
  uint64_t* out;
  int64_t count, h0, nbk, G, S;
  int c0;
  int64_t seg_begin, seg_end;  // segments of this launch
};
// p == 0: raw outputs; else each output reduced mod p (fp = field of p).
cudaError_t mixmax_fill(const MixFill& a, uint64_t p, const FieldParams& fp, cudaStream_t st);
// Warps of one launch that run at once on this device (segments per wave).
int mixmax_resident_warps(int N, int num_sms);

// xoroshiro128++: thread t of S produces outputs [t*L, min((t+1)*L, count))
// from starts[2t], starts[2t+1] = (s0, s1); ends[0..2) = state after `count`.
struct XoroFill {
  const uint64_t* starts;
  uint64_t* ends;
  uint64_t* out;
  int64_t count, L, S;
};
cudaError_t xoro_fill(const XoroFill& a, uint64_t p, const FieldParams& fp, cudaStream_t st);

// Per-device state of the fills, guarded by the caller's lock: the cached
// MIXMAX jump matrices B^(2^k) (B = skip + 1 iterations, stored transposed so
// that a row of states times it is a row of states) and the workspace.
struct PrngCache {
  uint64_t* pow[3] = {nullptr, nullptr, nullptr};  // MIXMAX-17, -240, -256: kPowMax matrices N x N
  int have[3] = {0, 0, 0};
  void* ws = nullptr;
  size_t ws_bytes = 0;
};
// The next `count` outputs of g into d_out (reduced mod p unless p == 0),
// exactly modlin_prng_fill's; g advances past them. Synchronises `st`.
// Returns a MODLIN_* code; *launches counts kernel launches.
int prng_fill_device(PrngCache& c, int num_sms, modlin_prng* g, uint64_t p, const FieldParams& fp, uint64_t* d_out,
                     uint64_t count, cudaStream_t st, uint64_t* launches);

}  // namespace modlin
