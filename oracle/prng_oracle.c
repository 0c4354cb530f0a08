/*
 * TEST INFRASTRUCTURE ONLY — CPU restatement of src/prng.rs of the reference
 * crate: xoroshiro128++ (SplitMix64-seeded) and the MIXMAX matrix generator
 * over 2^61-1 in its N=17, N=240 and N=256 instances. Pinned by the golden
 * vectors of tests/test_prng.rs.
 */
#include "oracle.h"

/* src/prng.rs:61-67 */
uint64_t oracle_splitmix64(uint64_t *z) {
    *z += 0x9e3779b97f4a7c15ULL;
    uint64_t w = *z;
    w = (w ^ (w >> 30)) * 0xbf58476d1ce4e5b9ULL;
    w = (w ^ (w >> 27)) * 0x94d049bb133111ebULL;
    return w ^ (w >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* src/prng.rs:58-83 */
static void xoroshiro_fill(uint64_t seed, uint64_t *out, size_t count) {
    uint64_t z = seed;
    uint64_t s0 = oracle_splitmix64(&z), s1 = oracle_splitmix64(&z);
    for (size_t i = 0; i < count; i++) {
        uint64_t a = s0, b = s1;
        out[i] = rotl(a + b, 17) + a;
        b ^= a;
        s0 = rotl(a, 49) ^ b ^ (b << 21);
        s1 = rotl(b, 28);
    }
}

/* src/prng.rs:99-127 */
#define MM_P 2305843009213693951ULL
#define MM_BITS 61
static inline uint64_t mod_mersenne(uint64_t k) { return (k & MM_P) + (k >> MM_BITS); }
static inline uint64_t modadd(uint64_t a, uint64_t b) { return mod_mersenne(a + b); }
static inline uint64_t fmodmul_m61(uint64_t cum, uint64_t a, uint64_t b) {
    u128 s = (u128)a * b + cum;
    uint64_t lo = (uint64_t)s, hi = (uint64_t)(s >> 64);
    uint64_t s1 = (lo & MM_P) + hi * 8 + (lo >> MM_BITS);
    return mod_mersenne(s1);
}

typedef struct {
    int n, specialmul, skip;
    uint64_t special; /* UINT64_MAX encodes the C value -1 */
    uint64_t v[256];
    uint64_t sumtot;
    int counter;
} mixmax;

/* src/prng.rs:152-176 — seed_spbox */
static int mixmax_seed(mixmax *g, uint64_t seed) {
    if (seed == 0) return -1;
    const uint64_t MULT64 = 6364136223846793005ULL;
    uint64_t l = seed, sumtot = 0, ovflow = 0;
    for (int i = 0; i < g->n; i++) {
        l *= MULT64;
        l = (l << 32) ^ (l >> 32);
        g->v[i] = l & MM_P;
        uint64_t s = sumtot + g->v[i];
        ovflow += s < sumtot;
        sumtot = s;
    }
    g->sumtot = mod_mersenne(mod_mersenne(sumtot) + (ovflow << 3));
    g->counter = g->n;
    return 0;
}

/* src/prng.rs:191-222 — iterate_raw_vec */
static void mixmax_iterate(mixmax *g) {
    uint64_t temp2 = g->v[1];
    uint64_t temp_v = g->sumtot;
    g->v[0] = temp_v;
    uint64_t sumtot = temp_v, ovflow = 0, temp_p = 0;
    for (int i = 1; i < g->n; i++) {
        if (g->specialmul) {
            uint64_t temp_po = ((temp_p << g->specialmul) & MM_P) | (temp_p >> (MM_BITS - g->specialmul));
            temp_p = modadd(temp_p, g->v[i]);
            temp_v = mod_mersenne(temp_v + temp_p + temp_po);
        } else {
            temp_p = modadd(temp_p, g->v[i]);
            temp_v = modadd(temp_v, temp_p);
        }
        g->v[i] = temp_v;
        uint64_t s = sumtot + temp_v;
        ovflow += s < sumtot;
        sumtot = s;
    }
    if (g->special) {
        uint64_t t2 = g->special == UINT64_MAX ? MM_P - temp2 : fmodmul_m61(0, g->special, temp2);
        g->v[2] = modadd(g->v[2], t2);
        uint64_t s = sumtot + t2;
        ovflow += s < sumtot;
        sumtot = s;
    }
    g->sumtot = mod_mersenne(mod_mersenne(sumtot) + (ovflow << 3));
}

/* src/prng.rs:227-269 — get_next / next_raw / output */
static uint64_t mixmax_output(mixmax *g) {
    int counter = g->counter;
    if (counter >= g->n)
        for (int k = 0; k < g->skip; k++) mixmax_iterate(g);
    g->counter = counter;
    uint64_t raw;
    if (g->counter < g->n) {
        raw = g->v[g->counter++];
    } else {
        mixmax_iterate(g);
        g->counter = 2;
        raw = g->v[1];
    }
    return raw << 3;
}

int oracle_prng_fill(int kind, uint64_t seed, uint64_t *out, size_t count) {
    if (kind == 0) {
        xoroshiro_fill(seed, out, count);
        return 0;
    }
    mixmax g;
    if (kind == 17) { g.n = 17; g.specialmul = 36; g.special = 0; g.skip = 0; }          /* prng.rs:305 */
    else if (kind == 240) { g.n = 240; g.specialmul = 51; g.special = 487013230256099140ULL; g.skip = 0; } /* :284 */
    else if (kind == 256) { g.n = 256; g.specialmul = 0; g.special = UINT64_MAX; g.skip = 2; }            /* :326 */
    else return -2;
    if (mixmax_seed(&g, seed) != 0) return -1;
    for (size_t i = 0; i < count; i++) out[i] = mixmax_output(&g);
    return 0;
}
