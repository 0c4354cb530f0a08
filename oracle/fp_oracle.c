/*
 * TEST INFRASTRUCTURE ONLY — CPU restatement of src/fp.rs of the reference
 * crate (Field / Barrett arithmetic, blocked rank, Berlekamp-Massey) plus the
 * naive oracles of its integration tests. Used as the checker by tests/, the
 * smoke entry point and the CPU-baseline leg of bench.py; never by the
 * product library.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/fp.rs:26-32 */
#define PANEL 64
#define TILE 256

/* src/fp.rs:13-24 — high 128 bits of the 256-bit product a*b. */
static inline u128 mul_hi_128(u128 a, u128 b) {
    u128 a1 = (uint64_t)(a >> 64), a0 = (uint64_t)a;
    u128 b1 = (uint64_t)(b >> 64), b0 = (uint64_t)b;
    u128 lo = a0 * b0, mid1 = a1 * b0, mid2 = a0 * b1, hi = a1 * b1;
    u128 m64 = (u128)UINT64_MAX;
    u128 carry = (lo >> 64) + (mid1 & m64) + (mid2 & m64);
    return hi + (mid1 >> 64) + (mid2 >> 64) + (carry >> 64);
}

/* src/fp.rs:49-61 */
int oracle_field_new(uint64_t p, oracle_field *f) {
    if (p < 2 || p >= (1ULL << 63)) return -1;
    u128 umax = ~(u128)0;
    f->p = p;
    f->mu = umax / p;
    u128 max_prod = (u128)(p - 1) * (u128)(p - 1);
    u128 sb = umax / max_prod; /* p >= 2 so max_prod >= 1 */
    if (sb > (u128)SIZE_MAX) sb = SIZE_MAX;
    f->safe_batch = sb ? (uint64_t)sb : 1;
    return 0;
}

/* src/fp.rs:71-79 — Barrett: q = hi(t*mu) <= floor(t/p), r < 3p. */
static inline uint64_t reduce_u128(const oracle_field *f, u128 t) {
    u128 q = mul_hi_128(t, f->mu);
    u128 p = f->p;
    u128 r = t - q * p;
    while (r >= p) r -= p;
    return (uint64_t)r;
}

uint64_t oracle_reduce_u128_parts(const oracle_field *f, uint64_t hi, uint64_t lo) {
    return reduce_u128(f, ((u128)hi << 64) | lo);
}

/* src/fp.rs:65-67 */
uint64_t oracle_reduce(const oracle_field *f, uint64_t x) { return reduce_u128(f, x); }

/* src/fp.rs:82-95 */
static inline uint64_t f_add(const oracle_field *f, uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= f->p ? s - f->p : s;
}
static inline uint64_t f_sub(const oracle_field *f, uint64_t a, uint64_t b) {
    return a >= b ? a - b : a + f->p - b;
}
static inline uint64_t f_mul(const oracle_field *f, uint64_t a, uint64_t b) {
    return reduce_u128(f, (u128)a * b);
}
uint64_t oracle_mul(const oracle_field *f, uint64_t a, uint64_t b) { return f_mul(f, a, b); }

/* src/fp.rs:97-113 — Fermat inverse a^(p-2). */
static uint64_t f_pow(const oracle_field *f, uint64_t a, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = f_mul(f, r, a);
        a = f_mul(f, a, a);
        e >>= 1;
    }
    return r;
}
uint64_t oracle_inv(const oracle_field *f, uint64_t a) { return f_pow(f, a, f->p - 2); }

/* src/fp.rs:125-255 — blocked right-looking elimination: PANEL-wide panel
 * factorisation with first-nonzero pivoting and whole-row swaps, U-block
 * coupling among the panel's pivot rows, then the tiled rank-pb trailing
 * update with u128 lazy accumulation (one reduction per safe_batch
 * products). rayon's par_chunks_mut over rows becomes an OpenMP loop. */
size_t oracle_rank(uint64_t p, uint64_t *m, size_t n, size_t *pcols_out, int threads) {
    oracle_field F;
    if (oracle_field_new(p, &F) != 0 || n == 0) return 0;
    const oracle_field *f = &F;
#ifdef _OPENMP
    int nthr = threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
#endif
    uint64_t *u = (uint64_t *)calloc((size_t)PANEL * n, sizeof(uint64_t));
    uint64_t *utile = (uint64_t *)calloc((size_t)PANEL * TILE, sizeof(uint64_t));
    size_t pcols[PANEL];
    size_t npc_total = 0;
    size_t rank = 0, col = 0;
    while (col < n && rank < n) {
        size_t jend = col + PANEL < n ? col + PANEL : n;
        size_t p0 = rank;
        size_t pb = 0;
        for (size_t j = col; j < jend; j++) {
            if (rank == n) break;
            size_t pr = n;
            for (size_t r = rank; r < n; r++)
                if (m[r * n + j] != 0) { pr = r; break; }
            if (pr == n) continue;
            if (pr != rank) {
                uint64_t *a = m + rank * n, *b = m + pr * n;
                for (size_t c = 0; c < n; c++) { uint64_t t = a[c]; a[c] = b[c]; b[c] = t; }
            }
            uint64_t inv = f_pow(f, m[rank * n + j], p - 2);
            const uint64_t *prow = m + rank * n;
            size_t lo = rank + 1;
#pragma omp parallel for num_threads(nthr) schedule(static) if (n - lo > 64)
            for (size_t r = lo; r < n; r++) {
                uint64_t *rr = m + r * n;
                uint64_t e = rr[j];
                if (e != 0) {
                    uint64_t fm = f_mul(f, e, inv);
                    rr[j] = fm;
                    for (size_t c = j + 1; c < jend; c++) rr[c] = f_sub(f, rr[c], f_mul(f, fm, prow[c]));
                }
            }
            pcols[pb++] = j;
            if (pcols_out) pcols_out[npc_total] = j;
            npc_total++;
            rank++;
        }
        if (pb > 0 && jend < n) {
            /* src/fp.rs:184-200 — U block with triangular coupling. */
            for (size_t k = 0; k < pb; k++)
                memcpy(u + k * n + jend, m + (p0 + k) * n + jend, (n - jend) * sizeof(uint64_t));
            for (size_t k = 1; k < pb; k++)
                for (size_t k2 = 0; k2 < k; k2++) {
                    uint64_t fm = m[(p0 + k) * n + pcols[k2]];
                    if (fm != 0) {
                        uint64_t *uk = u + k * n;
                        const uint64_t *uk2 = u + k2 * n;
                        for (size_t c = jend; c < n; c++) uk[c] = f_sub(f, uk[c], f_mul(f, fm, uk2[c]));
                    }
                }
            /* src/fp.rs:208-248 — tiled trailing update. */
            uint64_t sb = f->safe_batch;
            for (size_t c0 = jend; c0 < n; c0 += TILE) {
                size_t c1 = c0 + TILE < n ? c0 + TILE : n;
                size_t w = c1 - c0;
                for (size_t k = 0; k < pb; k++)
                    for (size_t ci = 0; ci < w; ci++) utile[ci * pb + k] = u[k * n + c0 + ci];
#pragma omp parallel for num_threads(nthr) schedule(static) if (n - rank > 16)
                for (size_t r = rank; r < n; r++) {
                    uint64_t *rr = m + r * n;
                    uint64_t fs[PANEL];
                    for (size_t k = 0; k < pb; k++) fs[k] = rr[pcols[k]];
                    for (size_t ci = 0; ci < w; ci++) {
                        const uint64_t *ut = utile + ci * pb;
                        uint64_t total = 0, cnt = 0;
                        u128 acc = 0;
                        for (size_t k = 0; k < pb; k++) {
                            acc += (u128)fs[k] * ut[k];
                            if (++cnt == sb) {
                                total = f_add(f, total, reduce_u128(f, acc));
                                acc = 0;
                                cnt = 0;
                            }
                        }
                        if (cnt > 0) total = f_add(f, total, reduce_u128(f, acc));
                        rr[c0 + ci] = f_sub(f, rr[c0 + ci], total);
                    }
                }
            }
        }
        col = jend;
    }
    free(u);
    free(utile);
    return rank;
}

/* tests/test_rank.rs:11-42 helpers (u128 `%` arithmetic). */
static inline uint64_t n_mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
static inline uint64_t n_addmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a + b) % p); }
static inline uint64_t n_submod(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + p - b; }
static uint64_t n_powmod(uint64_t a, uint64_t e, uint64_t p) {
    u128 r = 1 % p, base = a % p;
    while (e) {
        if (e & 1) r = r * base % p;
        base = base * base % p;
        e >>= 1;
    }
    return (uint64_t)r;
}

/* tests/test_rank.rs:44-72 */
size_t oracle_rank_naive(uint64_t p, uint64_t *m, size_t n) {
    size_t rank = 0;
    for (size_t col = 0; col < n; col++) {
        if (rank == n) break;
        size_t pr = n;
        for (size_t r = rank; r < n; r++)
            if (m[r * n + col] != 0) { pr = r; break; }
        if (pr == n) continue;
        if (pr != rank)
            for (size_t c = col; c < n; c++) {
                uint64_t t = m[pr * n + c];
                m[pr * n + c] = m[rank * n + c];
                m[rank * n + c] = t;
            }
        uint64_t inv = n_powmod(m[rank * n + col], p - 2, p);
        for (size_t r = rank + 1; r < n; r++) {
            uint64_t head = m[r * n + col];
            if (head != 0) {
                uint64_t fm = n_mulmod(head, inv, p);
                for (size_t c = col; c < n; c++)
                    m[r * n + c] = n_submod(m[r * n + c], n_mulmod(fm, m[rank * n + c], p), p);
            }
        }
        rank++;
    }
    return rank;
}

/* src/fp.rs:260-308 — Berlekamp-Massey with the c[m..m+bl) update window. */
size_t oracle_linear_complexity(uint64_t p, const uint64_t *s, size_t n,
                                uint64_t *dot_macs, uint64_t *axpy_macs) {
    oracle_field F;
    if (oracle_field_new(p, &F) != 0) return 0;
    const oracle_field *f = &F;
    if (n == 0) {
        if (dot_macs) *dot_macs = 0;
        if (axpy_macs) *axpy_macs = 0;
        return 0;
    }
    uint64_t *c = (uint64_t *)calloc(n, sizeof(uint64_t));
    uint64_t *b = (uint64_t *)calloc(n, sizeof(uint64_t));
    uint64_t *t = (uint64_t *)calloc(n, sizeof(uint64_t));
    c[0] = 1;
    b[0] = 1;
    size_t l = 0, bl = 1, m = 1;
    uint64_t bb_inv = 1, nd = 0, na = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t d = s[i];
        for (size_t j = 1; j <= l; j++) d = f_add(f, d, f_mul(f, c[j], s[i - j]));
        nd += l;
        if (d == 0) { m++; continue; }
        uint64_t coef = f_mul(f, d, bb_inv);
        size_t jmax = bl < n - m ? bl : n - m;
        na += jmax;
        if (2 * l <= i) {
            size_t old_l = l;
            memcpy(t, c, (old_l + 1) * sizeof(uint64_t));
            for (size_t j = 0; j < jmax; j++) c[j + m] = f_sub(f, c[j + m], f_mul(f, coef, b[j]));
            uint64_t *tmp = b; b = t; t = tmp;
            bl = old_l + 1;
            bb_inv = f_pow(f, d, p - 2);
            l = i + 1 - old_l;
            m = 1;
        } else {
            for (size_t j = 0; j < jmax; j++) c[j + m] = f_sub(f, c[j + m], f_mul(f, coef, b[j]));
            m++;
        }
    }
    free(c); free(b); free(t);
    if (dot_macs) *dot_macs = nd;
    if (axpy_macs) *axpy_macs = na;
    return l;
}

/* tests/test_linear_complexity.rs:37-70 — full-length update, clone of c. */
size_t oracle_lc_naive(uint64_t p, const uint64_t *s, size_t n) {
    if (n == 0) return 0;
    uint64_t *c = (uint64_t *)calloc(n, sizeof(uint64_t));
    uint64_t *b = (uint64_t *)calloc(n, sizeof(uint64_t));
    uint64_t *t = (uint64_t *)calloc(n, sizeof(uint64_t));
    c[0] = 1; b[0] = 1;
    size_t l = 0, m = 1;
    uint64_t bb = 1;
    for (size_t i = 0; i < n; i++) {
        uint64_t d = s[i];
        for (size_t j = 1; j <= l; j++) d = n_addmod(d, n_mulmod(c[j], s[i - j], p), p);
        if (d == 0) { m++; continue; }
        uint64_t coef = n_mulmod(d, n_powmod(bb, p - 2, p), p);
        memcpy(t, c, n * sizeof(uint64_t));
        for (size_t j = 0; j < n - m; j++) c[j + m] = n_submod(c[j + m], n_mulmod(coef, b[j], p), p);
        if (2 * l <= i) {
            l = i + 1 - l;
            memcpy(b, t, n * sizeof(uint64_t));
            bb = d;
            m = 1;
        } else {
            m++;
        }
    }
    free(c); free(b); free(t);
    return l;
}

/* Deterministic Miller-Rabin for 64-bit n (the bases 2..37 are a proven
 * witness set below 3.3e24); restates the behaviour of primal::is_prime,
 * which src/cli.rs:178 uses to validate -p. */
int oracle_is_prime(uint64_t n) {
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (int i = 0; i < 12; i++) {
        uint64_t x = n_powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; r++) {
            x = n_mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}

/* ---- Input generators of the reference's own tests ------------------------ */

/* tests/test_rank.rs:11-16 — full SplitMix64 finalizer of x * golden. */
static inline uint64_t mix_rank(uint64_t x) {
    uint64_t z = x * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* src/fp.rs:318-322 and tests/test_linear_complexity.rs:95-99 — 2-round mixer. */
static inline uint64_t mix_lc(uint64_t x) {
    uint64_t z = x * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    return z ^ (z >> 31);
}

uint64_t oracle_mix_rank(uint64_t x) { return mix_rank(x); }
uint64_t oracle_mix_lc(uint64_t x) { return mix_lc(x); }

/* tests/test_rank.rs:104-138 — one case of blocked_matches_reference: `target`
 * random rows, the others random combinations of them, then a Fisher-Yates
 * row shuffle. `*seed` is the test's running counter (pre-incremented). */
void oracle_test_rank_case(uint64_t p, size_t n, size_t target, uint64_t *seed, uint64_t *a) {
    if (target > n) target = n;
    memset(a, 0, n * n * sizeof(uint64_t));
    for (size_t r = 0; r < target; r++)
        for (size_t c = 0; c < n; c++) a[r * n + c] = mix_rank(++*seed) % p;
    for (size_t r = target; r < n; r++)
        for (size_t k = 0; k < target; k++) {
            uint64_t coeff = mix_rank(++*seed) % p;
            if (coeff == 0) continue;
            for (size_t c = 0; c < n; c++)
                a[r * n + c] = n_addmod(a[r * n + c], n_mulmod(coeff, a[k * n + c], p), p);
        }
    for (size_t r = n; r-- > 1;) {
        size_t s = (size_t)(mix_rank(++*seed) % (uint64_t)(r + 1));
        if (s != r)
            for (size_t c = 0; c < n; c++) {
                uint64_t t = a[r * n + c];
                a[r * n + c] = a[s * n + c];
                a[s * n + c] = t;
            }
    }
}

/* tests/test_linear_complexity.rs:110 — n random residues. */
void oracle_test_lc_random(uint64_t p, size_t n, uint64_t *seed, uint64_t *s) {
    for (size_t i = 0; i < n; i++) s[i] = mix_lc(++*seed) % p;
}

/* tests/test_linear_complexity.rs:119-127 — order-k LFSR of length len:
 * s[i] = sum_j c_j s[i-1-j]. */
void oracle_test_lc_lfsr(uint64_t p, size_t k, size_t len, uint64_t *seed, uint64_t *s) {
    uint64_t *coeffs = (uint64_t *)malloc(k * sizeof(uint64_t));
    for (size_t j = 0; j < k; j++) coeffs[j] = mix_lc(++*seed) % p;
    for (size_t i = 0; i < k && i < len; i++) s[i] = mix_lc(++*seed) % p;
    for (size_t i = k; i < len; i++) {
        uint64_t v = 0;
        for (size_t j = 0; j < k; j++) v = n_addmod(v, n_mulmod(coeffs[j], s[i - 1 - j], p), p);
        s[i] = v;
    }
    free(coeffs);
}

/* ---- Workload generators (the benchmark conventions) ---------------------- */

/* Uniform residue in [0,p): the top bitlen(p-1) bits of a SplitMix64 draw,
 * rejected while >= p. */
static inline uint64_t uniform_residue(uint64_t p, uint64_t *state) {
    int bits = 64 - __builtin_clzll(p - 1);
    for (;;) {
        uint64_t x = oracle_splitmix64(state) >> (64 - bits);
        if (x < p) return x;
    }
}

void oracle_gen_uniform(uint64_t p, uint64_t *state, uint64_t *out, size_t count) {
    for (size_t i = 0; i < count; i++) out[i] = uniform_residue(p, state);
}

/* Planted order-L recurrence: coefficients a_1..a_L (a_L redrawn while 0),
 * then initial values s_0..s_{L-1}, all uniform residues from `state`;
 * s[i] = sum_{j=1..L} a_j s[i-j] mod p for i >= L. */
void oracle_gen_planted(uint64_t p, size_t L, uint64_t *state, uint64_t *out, size_t count) {
    oracle_field F;
    oracle_field_new(p, &F);
    uint64_t *a = (uint64_t *)malloc((L + 1) * sizeof(uint64_t));
    for (size_t j = 1; j <= L; j++) a[j] = uniform_residue(p, state);
    while (L > 0 && a[L] == 0) a[L] = uniform_residue(p, state);
    uint64_t *init = (uint64_t *)malloc((L + 1) * sizeof(uint64_t));
    for (size_t i = 0; i < L; i++) init[i] = uniform_residue(p, state);
    for (size_t i = 0; i < count; i++) {
        if (i < L) { out[i] = init[i]; continue; }
        u128 acc = 0;
        uint64_t total = 0, cnt = 0;
        for (size_t j = 1; j <= L; j++) {
            acc += (u128)a[j] * out[i - j];
            if (++cnt == F.safe_batch) { total = f_add(&F, total, reduce_u128(&F, acc)); acc = 0; cnt = 0; }
        }
        out[i] = f_add(&F, total, reduce_u128(&F, acc));
    }
    free(a);
    free(init);
}

/* Matrix with planted dependencies (checker input; no reference counterpart).
 * An n x n matrix of uniform residues from `state` (row-major), then:
 *  - ncols distinct columns j, drawn as splitmix64 % (n - 2) + 2 (redrawn when
 *    already taken) and processed in increasing order, each become
 *    a*col(j1) + b*col(j2) with j1 = splitmix64 % j, j2 = splitmix64 % j and
 *    a, b uniform residues (drawn in that order per column);
 *  - each of the last nrows rows becomes sum_{t<4} c_t * row(i_t) with
 *    i_t = splitmix64 % (n - nrows) and c_t a uniform residue (drawn i_t, c_t
 *    per term, rows in increasing order).
 * Generically rank = n - max(ncols, nrows), and the pivot columns are the
 * first `rank` columns outside the planted set. dep_cols (ncols entries)
 * receives the planted columns in increasing order. */
static int cmp_size(const void *x, const void *y) {
    size_t a = *(const size_t *)x, b = *(const size_t *)y;
    return a < b ? -1 : a > b;
}

void oracle_gen_dependent(uint64_t p, size_t n, uint64_t *state, size_t ncols, size_t nrows, uint64_t *out,
                          size_t *dep_cols) {
    oracle_field F;
    oracle_field_new(p, &F);
    oracle_gen_uniform(p, state, out, n * n);
    if (n < 3) ncols = 0;
    if (ncols > n - 2) ncols = n - 2;
    if (nrows >= n) nrows = n - 1;
    unsigned char *taken = (unsigned char *)calloc(n, 1);
    for (size_t t = 0; t < ncols; t++) {
        size_t j;
        do j = (size_t)(oracle_splitmix64(state) % (n - 2)) + 2; while (taken[j]);
        taken[j] = 1;
        dep_cols[t] = j;
    }
    qsort(dep_cols, ncols, sizeof(size_t), cmp_size);
    size_t *src = (size_t *)malloc((2 * ncols + 1) * sizeof(size_t));
    uint64_t *cf = (uint64_t *)malloc((2 * ncols + 1) * sizeof(uint64_t));
    for (size_t t = 0; t < ncols; t++) {
        const size_t j = dep_cols[t];
        src[2 * t] = (size_t)(oracle_splitmix64(state) % j);
        src[2 * t + 1] = (size_t)(oracle_splitmix64(state) % j);
        cf[2 * t] = uniform_residue(p, state);
        cf[2 * t + 1] = uniform_residue(p, state);
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
        uint64_t *r = out + i * n;
        for (size_t t = 0; t < ncols; t++)
            r[dep_cols[t]] = f_add(&F, f_mul(&F, cf[2 * t], r[src[2 * t]]), f_mul(&F, cf[2 * t + 1], r[src[2 * t + 1]]));
    }
    size_t *rs = (size_t *)malloc((4 * nrows + 1) * sizeof(size_t));
    uint64_t *rc = (uint64_t *)malloc((4 * nrows + 1) * sizeof(uint64_t));
    for (size_t t = 0; t < 4 * nrows; t++) {
        rs[t] = (size_t)(oracle_splitmix64(state) % (n - nrows));
        rc[t] = uniform_residue(p, state);
    }
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < nrows; q++) {
        uint64_t *r = out + (n - nrows + q) * n;
        for (size_t c = 0; c < n; c++) {
            uint64_t v = 0;
            for (int t = 0; t < 4; t++) v = f_add(&F, v, f_mul(&F, rc[4 * q + t], out[rs[4 * q + t] * n + c]));
            r[c] = v;
        }
    }
    free(taken);
    free(src);
    free(cf);
    free(rs);
    free(rc);
}
