/*
 * TEST INFRASTRUCTURE ONLY — CPU restatement of src/stats.rs of the reference
 * crate (f64 null distributions, one-sided p-values and p-value formatting).
 * Must be compiled with -ffp-contract=off and without -ffast-math: Rust never
 * contracts a*b+c, and the reference's exact p-values (1e-307, 1.0,
 * 0.9947916666666666) are pinned bit for bit.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* src/stats.rs:16 */
#define P_FLOOR 1e-307
static const double LN_2 = 0.693147180559945309417232121458176568;

/* f64::powi lowers to compiler-rt's __powidf2: square-and-multiply over the
 * exponent bits, reciprocal at the end for a negative exponent. */
static double powi(double a, int b) {
    int recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

/* src/stats.rs:19-23 */
static double ln_u64(uint64_t p) {
    int e = 63 - __builtin_clzll(p);
    double mantissa = (double)p / (double)(1ULL << e);
    return fma((double)e, LN_2, log(mantissa));
}

/* src/stats.rs:26-41 */
static double sum_ln_1m(double p, size_t a, size_t b) {
    if (a > b) return 0.0;
    double inv = 1.0 / p;
    double pj = powi(inv, (int)a);
    double s = 0.0;
    for (size_t j = a; j <= b; j++) {
        if (pj < 1e-18) break;
        s += log1p(-pj);
        pj *= inv;
    }
    return s;
}

static double clamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

/* src/stats.rs:52-62 */
double oracle_corank_prob(uint64_t p, size_t n, size_t d) {
    if (d > n) return 0.0;
    double pf = (double)p;
    double t0 = -powi((double)d, 2) * ln_u64(p);
    double t1 = 2.0 * sum_ln_1m(pf, d + 1, n);
    double lp = t0 + t1;
    lp = lp - sum_ln_1m(pf, 1, n - d);
    return lp < -745.0 ? 0.0 : exp(lp);
}

/* src/stats.rs:69-84 */
double oracle_corank_tail_pvalue(uint64_t p, size_t n, size_t c) {
    if (c == 0) return 1.0;
    double s = 0.0;
    for (size_t d = c; d <= n; d++) {
        double pr = oracle_corank_prob(p, n, d);
        if (pr == 0.0) break;
        s += pr;
    }
    return clamp(s, P_FLOOR, 1.0);
}

/* src/stats.rs:101-126 */
double oracle_lc_left_tail_pvalue(uint64_t p, size_t n, size_t ell) {
    if (ell >= n) return 1.0;
    double lnp = ln_u64(p);
    double pr;
    if (2 * ell <= n) {
        double a = (double)(2 * ell + 1) * lnp;
        double ln_num = a > 0.0 ? a + log1p(exp(-a)) : log1p(exp(a));
        double ln_den = (double)n * lnp + log((double)p + 1.0);
        pr = exp(ln_num - ln_den);
    } else {
        double hi = exp(((double)n - 2.0 * (double)ell) * lnp);
        double lo = exp(-(double)n * lnp);
        pr = 1.0 - (hi - lo) / ((double)p + 1.0);
    }
    return clamp(pr, P_FLOOR, 1.0);
}

/* Shortest round-trip significant digits of a finite nonzero double:
 * the correctly rounded k-digit rendering for the smallest k that parses
 * back to the same value. */
static int shortest_digits(double x, char *digits, int *exp10) {
    char tmp[64];
    for (int k = 1; k <= 17; k++) {
        snprintf(tmp, sizeof tmp, "%.*e", k - 1, x);
        if (strtod(tmp, NULL) == x) {
            /* tmp = d[.ddd]e[+-]XX */
            int nd = 0;
            const char *q = tmp;
            if (*q == '-') q++;
            for (; *q && *q != 'e'; q++)
                if (*q >= '0' && *q <= '9') digits[nd++] = *q;
            while (nd > 1 && digits[nd - 1] == '0') nd--;
            digits[nd] = 0;
            *exp10 = atoi(q + 1);
            return nd;
        }
    }
    return 0;
}

/* src/stats.rs:129-137 — "0", "1", else Rust's `{:?}` for f64: shortest
 * round-trip digits, scientific notation (no '+', no exponent padding) when
 * |x| < 1e-4 or |x| >= 1e16, else plain decimal with at least one fractional
 * digit. */
int oracle_pretty_p_value(double p, char *buf, size_t cap) {
    if (p == 0.0) return snprintf(buf, cap, "0");
    if (p == 1.0) return snprintf(buf, cap, "1");
    if (isnan(p)) return snprintf(buf, cap, "NaN");
    if (isinf(p)) return snprintf(buf, cap, p > 0 ? "inf" : "-inf");
    char digits[32];
    int e = 0;
    int nd = shortest_digits(p, digits, &e);
    char out[400];
    size_t o = 0;
    if (p < 0) out[o++] = '-';
    double a = fabs(p);
    if (a < 1e-4 || a >= 1e16) {
        out[o++] = digits[0];
        if (nd > 1) {
            out[o++] = '.';
            for (int i = 1; i < nd; i++) out[o++] = digits[i];
        }
        o += (size_t)snprintf(out + o, sizeof out - o, "e%d", e);
    } else if (e < 0) {
        out[o++] = '0';
        out[o++] = '.';
        for (int i = 0; i < -e - 1; i++) out[o++] = '0';
        for (int i = 0; i < nd; i++) out[o++] = digits[i];
    } else {
        for (int i = 0; i <= e; i++) out[o++] = i < nd ? digits[i] : '0';
        out[o++] = '.';
        if (nd > e + 1)
            for (int i = e + 1; i < nd; i++) out[o++] = digits[i];
        else
            out[o++] = '0';
    }
    out[o] = 0;
    return snprintf(buf, cap, "%s", out);
}
