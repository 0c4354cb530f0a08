/*
 * CPU oracle for the modular rank / Berlekamp-Massey engine.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * crate (vigna/modlin-rs, Rust) used as the checker: only tests/, the smoke
 * entry point and the CPU-baseline leg of bench.py may load it. The product
 * library never links or calls it.
 *
 * Parity pin: the restatement is checked against every golden vector and
 * known-answer test the reference ships for this path (tests/test_prng.rs
 * MIXMAX/xoroshiro vectors, tests/test_stats.rs exact values, the README's
 * end-to-end runs: corank 432 for MIXMAX-17 -R 500, linear complexity 272
 * for MIXMAX-17 -L 1000, ...) and against the naive oracles of
 * tests/test_rank.rs and tests/test_linear_complexity.rs.
 *
 * Every function cites the reference file:line it restates (paths are
 * relative to the reference crate root).
 */
#ifndef MODLIN_ORACLE_H
#define MODLIN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned __int128 u128;

/* src/fp.rs:34-46 — Field { p, mu, safe_batch } */
typedef struct {
    uint64_t p;
    u128 mu;
    uint64_t safe_batch;
} oracle_field;

/* src/fp.rs:49-61 */
int oracle_field_new(uint64_t p, oracle_field *f);
/* src/fp.rs:65-67, 71-79 */
uint64_t oracle_reduce(const oracle_field *f, uint64_t x);
uint64_t oracle_reduce_u128_parts(const oracle_field *f, uint64_t hi, uint64_t lo);
/* src/fp.rs:93-95 */
uint64_t oracle_mul(const oracle_field *f, uint64_t a, uint64_t b);
/* src/fp.rs:110-113 */
uint64_t oracle_inv(const oracle_field *f, uint64_t a);

/* src/fp.rs:125-255 — blocked rank. `m` (n*n, row-major, entries < p) is
 * clobbered. If pcols != NULL it receives the pivot columns in discovery
 * order (at most n entries). threads <= 0 means all OpenMP threads. */
size_t oracle_rank(uint64_t p, uint64_t *m, size_t n, size_t *pcols, int threads);

/* tests/test_rank.rs:44-72 — naive unblocked elimination with `%`. */
size_t oracle_rank_naive(uint64_t p, uint64_t *m, size_t n);

/* src/fp.rs:260-308 — Berlekamp-Massey. If dot_macs/axpy_macs are not NULL
 * they receive the number of multiply-adds of the discrepancy dots and of the
 * connection-polynomial updates (the algorithmic work of the run). */
size_t oracle_linear_complexity(uint64_t p, const uint64_t *s, size_t n,
                                uint64_t *dot_macs, uint64_t *axpy_macs);

/* tests/test_linear_complexity.rs:37-70 — naive BM with `%`. */
size_t oracle_lc_naive(uint64_t p, const uint64_t *s, size_t n);

/* src/stats.rs */
double oracle_corank_prob(uint64_t p, size_t n, size_t d);          /* :52-62 */
double oracle_corank_tail_pvalue(uint64_t p, size_t n, size_t c);   /* :69-84 */
double oracle_lc_left_tail_pvalue(uint64_t p, size_t n, size_t ell);/* :101-126 */
/* :129-137 — writes the Rust `{:?}` rendering (or "0"/"1"); returns length */
int oracle_pretty_p_value(double p, char *buf, size_t cap);

/* src/prng.rs — generators. kind: 0 = xoroshiro128++, 17 = MIXMAX N=17,
 * 240 = MIXMAX N=240, 256 = MIXMAX N=256. Returns 0 on success, -1 on a
 * rejected seed (MIXMAX seed 0, prng.rs:153-155), -2 on unknown kind. */
int oracle_prng_fill(int kind, uint64_t seed, uint64_t *out, size_t count);

/* src/prng.rs:61-67 — SplitMix64 step. */
uint64_t oracle_splitmix64(uint64_t *state);

/* miller-rabin primality (primal::is_prime, used by src/cli.rs:178) */
int oracle_is_prime(uint64_t n);

/* Input generators of the reference's own tests (running counter `seed`,
 * pre-incremented): tests/test_rank.rs:104-138 (one case of
 * blocked_matches_reference), tests/test_linear_complexity.rs:110 and
 * :119-127. */
uint64_t oracle_mix_rank(uint64_t x);
uint64_t oracle_mix_lc(uint64_t x);
void oracle_test_rank_case(uint64_t p, size_t n, size_t target, uint64_t *seed, uint64_t *a);
void oracle_test_lc_random(uint64_t p, size_t n, uint64_t *seed, uint64_t *s);
void oracle_test_lc_lfsr(uint64_t p, size_t k, size_t len, uint64_t *seed, uint64_t *s);

/* Workload generators (uniform residues by SplitMix64 + rejection; planted
 * order-L recurrences), used to cross-check the product's generators. */
void oracle_gen_uniform(uint64_t p, uint64_t *state, uint64_t *out, size_t count);
void oracle_gen_planted(uint64_t p, size_t L, uint64_t *state, uint64_t *out, size_t count);
/* n x n uniform matrix with ncols columns and the last nrows rows replaced by
 * combinations of earlier ones (checker input for full-size parity tests). */
void oracle_gen_dependent(uint64_t p, size_t n, uint64_t *state, size_t ncols, size_t nrows, uint64_t *out,
                          size_t *dep_cols);

#ifdef __cplusplus
}
#endif
#endif
