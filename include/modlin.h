/*
 * modlin — B200-native modular rank and linear-complexity engine (C ABI).
 *
 * Drop-in boundary for the two hot paths of the modlin crate: the rank of an
 * n x n matrix over F_p by blocked Gaussian elimination and the linear
 * complexity of a sequence over F_p by Berlekamp-Massey, p prime, p < 2^63.
 * Every entry point takes plain pointers and sizes; all device memory is
 * owned by the library. Host matrices and sequences are owned by the caller.
 * Results are bit-exact: ranks and linear complexities are mathematical
 * invariants and every kernel computes exact residues.
 *
 * Entry points on device memory take `void *stream`, a cudaStream_t: the
 * work is queued there, and NULL means the legacy default stream, so work
 * the caller queued on it (a copy that fills the input, say) comes first.
 *
 * Return codes: MODLIN_OK (0) or a negative MODLIN_E* code; no entry point
 * aborts the process (the reference panics: src/fp.rs:50-51).
 * Reference citations are file:line inside the modlin crate.
 */
#ifndef MODLIN_H
#define MODLIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Exported symbols keep default visibility even in -fvisibility=hidden builds. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define MODLIN_OK 0
#define MODLIN_EINVAL_P (-1)   /* p < 2 or p >= 2^63 (src/fp.rs:50-51) */
#define MODLIN_EINVAL_N (-2)   /* rank of n == 0, n*n overflows, or n exceeds a limit */
#define MODLIN_EINPUT (-3)     /* an entry is >= p (checked only on request) */
#define MODLIN_ECUDA (-4)      /* CUDA runtime error */
#define MODLIN_ENOMEM (-5)     /* device or host allocation failed */
#define MODLIN_ETIMEOUT (-6)   /* a bounded device-side wait expired */
#define MODLIN_ENODEV (-7)     /* no CUDA device */
#define MODLIN_EINVAL_ARG (-8) /* NULL pointer or invalid option */

/* Progress callback: `done` of `total` columns (rank) or steps (linear
 * complexity); replaces the reference's generic `pl: &mut impl ProgressLog`
 * (src/fp.rs:125, :260), which has no C form. May be NULL. */
typedef void (*modlin_progress_fn)(void *ctx, size_t done, size_t total);
/* A generator under test (src/prng.rs); see the generator section below. */
typedef struct modlin_prng modlin_prng;

/* Human-readable text for a return code. */
const char *modlin_strerror(int code);

/* ---- Field contract (src/fp.rs:34-114) ---------------------------------- */

typedef struct {
    uint64_t p;
    uint64_t mu_lo, mu_hi;  /* mu = floor((2^128 - 1) / p), src/fp.rs:52 */
    uint64_t safe_batch;    /* products of (p-1)^2 summable in a u128, src/fp.rs:53-59 */
} modlin_field;

/* Field::new (src/fp.rs:49-61); MODLIN_EINVAL_P unless 2 <= p < 2^63. */
int modlin_field_new(uint64_t p, modlin_field *f);
/* Field::reduce (src/fp.rs:65-67). */
uint64_t modlin_field_reduce(const modlin_field *f, uint64_t x);
/* Field::reduce_u128 (src/fp.rs:71-79) of hi * 2^64 + lo. */
uint64_t modlin_field_reduce_u128(const modlin_field *f, uint64_t hi, uint64_t lo);
/* Field::mul (src/fp.rs:93-95), canonical inputs. */
uint64_t modlin_field_mul(const modlin_field *f, uint64_t a, uint64_t b);

/* ---- Rank (src/fp.rs:116-255) ------------------------------------------- */

#define MODLIN_RANK_AUTO 0   /* tensor-core trailing update where it pays */
#define MODLIN_RANK_PLAIN 1  /* u64 Barrett trailing update on the integer pipes */
#define MODLIN_RANK_TC 2     /* INT8-limb tcgen05 trailing update */

typedef struct {
    int kernel;       /* MODLIN_RANK_* */
    int check_input;  /* nonzero: reject entries >= p with MODLIN_EINPUT */
} modlin_rank_opts;

/* fp::rank (src/fp.rs:125): rank over F_p of the n x n row-major matrix `m`
 * (host memory, entries in [0, p)). Like the reference, the contents of `m`
 * afterwards are unspecified (the GPU path leaves them untouched). */
int modlin_rank(uint64_t p, uint64_t *m, size_t n, size_t *rank_out,
                modlin_progress_fn cb, void *cb_ctx);

/* modlin_rank with options; `pivot_cols_out` (may be NULL, else room for n
 * entries) receives the pivot columns in increasing order — the column
 * profile, an invariant of the matrix. */
int modlin_rank_ex(uint64_t p, uint64_t *m, size_t n, const modlin_rank_opts *opts,
                   size_t *rank_out, size_t *pivot_cols_out,
                   modlin_progress_fn cb, void *cb_ctx);

/* Same on a device-resident matrix (clobbered); `stream` is a cudaStream_t
 * (NULL = legacy default stream). The call returns when the rank is known. */
int modlin_rank_device(uint64_t p, uint64_t *d_m, size_t n, const modlin_rank_opts *opts,
                       size_t *rank_out, size_t *pivot_cols_out, void *stream);
/* One matrix of the -R test (src/main.rs:94-112): the next n*n outputs of g,
 * reduced mod p, row by row, generated in device memory
 * (modlin_prng_fill_device) and ranked there; g advances past them. */
int modlin_rank_prng(uint64_t p, modlin_prng *g, size_t n, const modlin_rank_opts *opts, size_t *rank_out,
                     modlin_progress_fn cb, void *cb_ctx);

/* The CLI's -R loop over `reps` matrices (src/main.rs:82-125) in batched
 * launches: the next reps * n*n outputs of g, reduced mod p, fill reps
 * matrices in device memory (row-major, one after another: the same matrices
 * as reps calls of modlin_rank_prng) and their ranks go to ranks_out[0..reps)
 * from one persistent launch per group of matrices that fits 8 GiB. Sides
 * above 8192 (and reps == 1) run one matrix at a time. cb (may be NULL)
 * receives matrices done / reps. */
int modlin_rank_prng_batch(uint64_t p, modlin_prng *g, size_t n, size_t reps, const modlin_rank_opts *opts,
                           size_t *ranks_out, modlin_progress_fn cb, void *cb_ctx);

/* The trailing update of one panel (src/fp.rs:202-248) as a standalone
 * device operation: C[M x N] -= L[M x K] * U[K x N] (mod p), all entries in
 * [0, p). K <= 64 (L row stride 64), or with the tensor-core kernel also
 * K <= 128 (two panels at once; L row stride 128). U has row stride ldu, C
 * row stride ldc. kernel: MODLIN_RANK_PLAIN or MODLIN_RANK_TC
 * (MODLIN_RANK_AUTO = TC). */
int modlin_trailing_update_device(uint64_t p, uint64_t *d_C, size_t ldc, size_t M, size_t N,
                                  const uint64_t *d_L, const uint64_t *d_U, size_t ldu, size_t K,
                                  int kernel, void *stream);
/* The pivots of one panel as the reference's in-panel elimination finds
 * them (src/fp.rs:146-178: per column the first row, in row order, that is
 * nonzero after the previous pivots' elimination): d_panel is rows x W
 * (W <= 64, row stride ld >= W) residues in device memory, left unchanged;
 * *pb_out receives the number of pivots, prow_out[k] / pcol_out[k] (room for
 * 64 each) the row and the column (0-based, within the panel) of pivot k.
 * Used by the column-sharded rank for panels whose diagonal block is
 * singular. Returns when the result is on the host. */
int modlin_panel_pivots_device(uint64_t p, const uint64_t *d_panel, size_t ld, size_t rows, size_t W,
                               size_t *prow_out, size_t *pcol_out, size_t *pb_out, void *stream);
/* The multiplier block of one block step of the rank (the pivot block's
 * inverse; the reference's in-panel elimination, src/fp.rs:146-200, as one
 * device operation): P is 64 x 64 at d_P (row stride ldp >= 64), entries in
 * [0, p); d_out (64 x 64, row stride 64) receives -P^-1, row c belonging to
 * column c of P; *singular = 1 (d_out unspecified) when P is singular. */
int modlin_block_inverse_device(uint64_t p, const uint64_t *d_P, size_t ldp, uint64_t *d_out, int *singular,
                                void *stream);

/* ---- Linear complexity (src/fp.rs:257-308) ------------------------------ */

#define MODLIN_LC_AUTO 0      /* block kernel for short, cluster for long, grid beyond the cluster */
#define MODLIN_LC_BLOCK 1     /* one CTA runs the whole sequence (plain form) */
#define MODLIN_LC_GRID 2      /* persistent cooperative kernel, one grid barrier per step */
#define MODLIN_LC_CLUSTER 3   /* one 16-CTA thread-block cluster, one cluster barrier per step
                                 (n <= 409600; MODLIN_EINVAL_N beyond) */

typedef struct {
    int kernel;       /* MODLIN_LC_* */
    int check_input;
    int grid_ctas;    /* MODLIN_LC_GRID: CTAs to use (0 = one per SM) */
} modlin_lc_opts;

/* fp::linear_complexity (src/fp.rs:260): length of the shortest LFSR that
 * generates s[0..n) (host memory, entries in [0, p)). */
int modlin_linear_complexity(uint64_t p, const uint64_t *s, size_t n, size_t *lc_out,
                             modlin_progress_fn cb, void *cb_ctx);
int modlin_linear_complexity_ex(uint64_t p, const uint64_t *s, size_t n, const modlin_lc_opts *opts,
                                size_t *lc_out);
int modlin_linear_complexity_device(uint64_t p, const uint64_t *d_s, size_t n,
                                    const modlin_lc_opts *opts, size_t *lc_out, void *stream);

/* No counterpart in the reference. For callers that cannot allocate device
 * memory on the call path (a host whose pool allocator owns all device
 * memory, or a loop that must not pay cudaMalloc's implicit synchronisation):
 * the linear complexity of the device sequence d_s[0..n) is written to the
 * device slot *d_lc_out, asynchronously on `stream`, without any allocation
 * (n = 0 writes 0). The Berlekamp-Massey scratch lives in shared memory when
 * it fits (n <= 8533), else in a fixed 6 MiB device array, so n <= 262144
 * (MODLIN_EINVAL_N beyond). All calls share that array: calls that overlap on
 * the GPU race, so order them (e.g. one stream). The first call on a device
 * is a set-up that loads the library's device code for this entry point and
 * the array (the CUDA driver allocates device memory for them) and looks up
 * the array's address: make it (n = 0 is enough) before the caller's pool
 * reserves the device memory and before any stream capture. Not usable on a
 * device after cudaDeviceReset of that device. */
int modlin_linear_complexity_device_noalloc(uint64_t p, const uint64_t *d_s, size_t n,
                                            int64_t *d_lc_out, void *stream);

/* ---- Batched jobs (the CLI's `reps`, src/main.rs:82 and :152) ----------- */

typedef struct {
    uint64_t p;
    const uint64_t *data; /* host, n*n row-major (rank) or n (linear complexity) */
    size_t n;
} modlin_job;

/* Ranks of `count` matrices of any sides and primes in one persistent
 * launch (matrices are copied; the inputs are not modified). */
int modlin_rank_batch(const modlin_job *jobs, size_t count, size_t *ranks_out);
/* Device-resident batch: d_m[i] is an n[i] x n[i] row-major matrix mod p[i]
 * in device memory, clobbered like modlin_rank_device. Sides up to 8192 go
 * into one persistent launch; larger ones run one after another. */
int modlin_rank_batch_device(const uint64_t *p, uint64_t *const *d_m, const size_t *n, size_t count,
                             size_t *ranks_out, void *stream);
/* modlin_rank_batch_device with options: kernel MODLIN_RANK_TC puts every job
 * of side up to 8192 on the tensor-core batch kernel, MODLIN_RANK_PLAIN on the
 * integer-pipe one, MODLIN_RANK_AUTO splits them at the tuned side. */
int modlin_rank_batch_device_ex(const uint64_t *p, uint64_t *const *d_m, const size_t *n, size_t count,
                                const modlin_rank_opts *opts, size_t *ranks_out, void *stream);
/* Linear complexities of `count` sequences in one persistent launch. */
int modlin_lc_batch(const modlin_job *jobs, size_t count, size_t *lcs_out);

/* Device-resident batch: data[i] are device pointers. */
int modlin_lc_batch_device(const uint64_t *p, const uint64_t *const *d_data, const size_t *n,
                           size_t count, size_t *lcs_out, void *stream);

/* Batch plans: the device job table of a batch of device-resident matrices
 * (sides up to 8192) or sequences is built once; each launch then queues one
 * counter reset and one persistent kernel on `stream`, with no allocation and
 * no host synchronisation, so it can be captured in a CUDA graph and replayed
 * (each launch clobbers the matrices, like modlin_rank_device: restore them
 * between replays). Result i (rank or linear complexity of job i) is written
 * to the caller's device array d_*_out[i] by each launch. Inputs and outputs
 * must stay at the same addresses for the plan's life. No reference
 * counterpart: the reference runs `reps` one after another (src/main.rs:82,
 * :152). */
typedef struct modlin_rank_batch_plan modlin_rank_batch_plan;
typedef struct modlin_lc_batch_plan modlin_lc_batch_plan;
int modlin_rank_batch_plan_new(const uint64_t *p, uint64_t *const *d_m, const size_t *n, size_t count,
                               int64_t *d_ranks_out, modlin_rank_batch_plan **plan_out);
int modlin_rank_batch_plan_launch(modlin_rank_batch_plan *plan, void *stream);
void modlin_rank_batch_plan_free(modlin_rank_batch_plan *plan);
int modlin_lc_batch_plan_new(const uint64_t *p, const uint64_t *const *d_s, const size_t *n, size_t count,
                             int64_t *d_lcs_out, modlin_lc_batch_plan **plan_out);
int modlin_lc_batch_plan_launch(modlin_lc_batch_plan *plan, void *stream);
void modlin_lc_batch_plan_free(modlin_lc_batch_plan *plan);

/* ---- p-values (src/stats.rs) -------------------------------------------- */

double modlin_corank_prob(uint64_t p, size_t n, size_t d);          /* src/stats.rs:52-62 */
double modlin_corank_tail_pvalue(uint64_t p, size_t n, size_t c);   /* src/stats.rs:69-84 */
double modlin_lc_left_tail_pvalue(uint64_t p, size_t n, size_t ell);/* src/stats.rs:101-126 */
/* src/stats.rs:129-137: "0", "1" or Rust's `{:?}` rendering; returns the
 * length written (excluding the NUL). */
int modlin_pretty_p_value(double p, char *buf, size_t cap);

/* ---- Generators (src/prng.rs) ------------------------------------------- */

#define MODLIN_PRNG_XOROSHIRO128PP 0
#define MODLIN_PRNG_MIXMAX17 17
#define MODLIN_PRNG_MIXMAX240 240
#define MODLIN_PRNG_MIXMAX256 256

/* Prng::try_new (src/prng.rs:58, :152): NULL + *err = MODLIN_EINVAL_ARG for
 * a rejected seed (MIXMAX forbids 0) or an unknown kind. */
modlin_prng *modlin_prng_new(int kind, uint64_t seed, int *err);
/* Prng::NAME (src/prng.rs:56, :288, :309, :330). */
const char *modlin_prng_name(int kind);
/* count successive next_u64() outputs. */
void modlin_prng_fill(modlin_prng *g, uint64_t *out, size_t count);
void modlin_prng_free(modlin_prng *g);
/* The same `count` outputs, written to device memory by many warps at once
 * from jump-ahead states (no reference counterpart: the reference fills its
 * matrix one next_u64() at a time, src/main.rs:94-104). Bit-identical to
 * modlin_prng_fill; each output is reduced mod p (Field::reduce) unless p is
 * 0. g advances past the outputs, so host and device fills interleave.
 * Returns after the fill is complete. */
int modlin_prng_fill_device(modlin_prng *g, uint64_t p, uint64_t *d_out, size_t count, void *stream);
/* A generator's position as 64-bit words, to save and restore it:
 * xoroshiro128++ 2 words (s0, s1); MIXMAX-N N + 2 words (v[0..N), sumtot,
 * counter). set_state rejects (MODLIN_EINVAL_ARG) a wrong word count, a
 * MIXMAX entry above 2^61 - 1 (no step produces one) or a counter outside
 * [1, N]. */
size_t modlin_prng_state_words(int kind);
int modlin_prng_get_state(const modlin_prng *g, uint64_t *words, size_t n);
int modlin_prng_set_state(modlin_prng *g, const uint64_t *words, size_t n);

/* ---- Synthetic workloads ------------------------------------------------ */

/* Uniform residues in [0, p): the top bitlen(p-1) bits of successive
 * SplitMix64 outputs (state initialised to `seed`), rejected while >= p. */
int modlin_gen_uniform(uint64_t p, uint64_t seed, uint64_t *out, size_t count);
/* Same, generated on the device (bit-identical to the host stream). */
int modlin_gen_uniform_device(uint64_t p, uint64_t seed, uint64_t *d_out, size_t count, void *stream);
/* Planted order-L recurrence: a_1..a_L (a_L redrawn while 0) then
 * s_0..s_{L-1} uniform residues from SplitMix64(seed);
 * s[i] = sum_{j=1..L} a_j s[i-j] mod p. */
int modlin_gen_planted(uint64_t p, size_t L, uint64_t seed, uint64_t *out, size_t count);
/* Same streams as modlin_gen_planted, produced on the device: the 2L seeded
 * draws (coefficients, initial state) on the host, the recurrence extended
 * by one CTA per sequence. Bit-identical to the host generator. */
int modlin_gen_planted_device(uint64_t p, size_t L, uint64_t seed, uint64_t *d_out, size_t count, void *stream);
/* A batch of planted sequences, job i: prime p[i], order L[i], seed seed[i],
 * count[i] outputs at device pointer d_out[i]; all in one launch. */
int modlin_gen_planted_batch_device(const uint64_t *p, const size_t *L, const uint64_t *seed,
                                    uint64_t *const *d_out, const size_t *count, size_t njobs, void *stream);
/* Field::reduce on the device, in place (src/main.rs:94-104 fill). */
int modlin_reduce_device(uint64_t p, uint64_t *d_x, size_t count, void *stream);

/* ---- Autotuning ----------------------------------------------------------- */

/* Measures, on the current device, the choices MODLIN_RANK_AUTO and
 * MODLIN_LC_AUTO make (no reference counterpart: the reference has one CPU
 * path): the side from which the tensor-core trailing update beats the plain
 * one, per limb count (1, 2, 4 or 8 limbs for p below 2^8, 2^16, 2^32, 2^63;
 * the limb count itself is the smallest exact one); the remaining-block size
 * below which one-panel block steps replace two-panel ones (timed on a
 * 16384 x 16384 rank); Berlekamp-Massey threads per CTA by length, the
 * block/cluster crossover, and batch threads per CTA by the longest sequence.
 * Takes a few seconds; the choices hold for this process and device. `report`
 * (may be NULL) receives them and the timings as JSON, truncated to cap - 1
 * characters. Before any call, fixed defaults apply. */
int modlin_autotune(char *report, size_t cap);

/* ---- Diagnostics --------------------------------------------------------- */

/* Number of this library's kernel launches since load (for launch-count
 * claims in measurements). */
uint64_t modlin_kernel_launches(void);
/* The roofline of the plain trailing update (MODLIN_RANK_PLAIN) for modulus
 * p: its inner loop alone (u64 x u64 -> u128 products, lazy accumulation,
 * one reduction per safe_batch products, operands from shared memory, no
 * global traffic) on every SM at the kernel's occupancy, in modular
 * multiply-adds per second (best of three timed launches). No reference
 * counterpart: it is the denominator of the plain kernel's pipe fraction. */
int modlin_plain_mac_peak(uint64_t p, double *modmac_per_s);
/* Tensor-core updates over 2^61 - 1 run on CTA pairs (thread-block clusters
 * of two CTAs sharing each B tile, M = 256 MMAs) when enable = 1 or on single
 * CTAs when enable = 0 (the default); enable < 0 only queries.
 * Returns the previous setting. Both kernels give the same, exact results;
 * no reference counterpart (a kernel choice, like MODLIN_RANK_TC). */
int modlin_set_tc_pairs(int enable);
/* Failure-detection test hook (no reference counterpart; the reference has
 * no device waits): the next MODLIN_LC_GRID launch in this process bounds
 * each grid-barrier wait by spin_cycles (1 .. 4e9) instead of ~1 s, and its
 * CTA skip_cta (a CTA the launch has: 0 always is) does not arrive at the
 * first step's barrier, so every wait expires, the kernel returns early and
 * the call reports MODLIN_ETIMEOUT. Nothing faults or hangs. */
int modlin_testing_grid_timeout_once(long long spin_cycles, int skip_cta);
/* Milliseconds spent in the trailing-update kernels of the last rank call,
 * measured with CUDA events on the launching stream (0 if unavailable). */
double modlin_last_trailing_ms(void);
/* Modular multiply-adds done by those timed trailing updates (rows x columns
 * x depth of each), so that their rate is this / the time above. */
double modlin_last_trailing_macs(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
