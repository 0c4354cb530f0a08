// Prime-field arithmetic over F_p, p < 2^63, for sm_100a device code and host.
//
// The contract is the reference's `Field` (src/fp.rs:34-114): canonical
// residues in [0, p), Barrett reciprocal mu = floor((2^128 - 1) / p) and exact
// reduction of any 128-bit value, add/sub/mul on canonical inputs, Fermat
// inverse. Three policies implement it:
//   * FpBarrett — any p in [2, 2^63): the reference's Barrett reduction
//     (src/fp.rs:71-79) on 64-bit integer pipes;
//   * FpM61 — p = 2^61 - 1 (MIXMAX's modulus and every large benchmark
//     workload): shift-and-add reduction, since 2^61 = 1 mod p;
//   * FpSmall — p < 2^32: 32-bit products and a 64-bit Barrett step.
// All return the exact residue, so every kernel built on them is bit-exact.
#pragma once
#include <cstdint>

#ifndef MODLIN_HD
#define MODLIN_HD __host__ __device__ __forceinline__
#endif

namespace modlin {

typedef unsigned __int128 u128;

// src/fp.rs:13-24: high 128 bits of the 256-bit product a*b.
MODLIN_HD u128 mul_hi_128(u128 a, u128 b) {
  const uint64_t a1 = (uint64_t)(a >> 64), a0 = (uint64_t)a;
  const uint64_t b1 = (uint64_t)(b >> 64), b0 = (uint64_t)b;
  const u128 lo = (u128)a0 * b0, mid1 = (u128)a1 * b0, mid2 = (u128)a0 * b1;
  const u128 hi = (u128)a1 * b1;
  const u128 carry = (lo >> 64) + (uint64_t)mid1 + (uint64_t)mid2;
  return hi + (mid1 >> 64) + (mid2 >> 64) + (carry >> 64);
}

// Host-side construction data for a field (src/fp.rs:49-61).
struct FieldParams {
  uint64_t p;
  uint64_t mu_lo, mu_hi;  // mu = floor((2^128 - 1) / p)
  uint64_t safe_batch;    // products of (p-1)^2 summable in a u128
};

inline bool make_field_params(uint64_t p, FieldParams* f) {
  if (p < 2 || p >= (1ULL << 63)) return false;
  const u128 umax = ~(u128)0;
  const u128 mu = umax / p;
  const u128 maxp = (u128)(p - 1) * (p - 1);
  u128 sb = umax / maxp;
  if (sb > (u128)UINT64_MAX) sb = UINT64_MAX;
  f->p = p;
  f->mu_lo = (uint64_t)mu;
  f->mu_hi = (uint64_t)(mu >> 64);
  f->safe_batch = sb ? (uint64_t)sb : 1;
  return true;
}

constexpr uint64_t kM61 = (1ULL << 61) - 1;

struct FpBarrett {
  uint64_t p, mu_lo, mu_hi, sb;
  FpBarrett() = default;
  MODLIN_HD explicit FpBarrett(const FieldParams& f) : p(f.p), mu_lo(f.mu_lo), mu_hi(f.mu_hi), sb(f.safe_batch) {}
  // src/fp.rs:71-79: q = hi(t*mu) <= floor(t/p), r = t - q*p < 3p.
  MODLIN_HD uint64_t reduce(u128 t) const {
    const u128 mu = ((u128)mu_hi << 64) | mu_lo;
    const u128 q = mul_hi_128(t, mu);
    u128 r = t - q * p;
    if (r >= p) r -= p;
    if (r >= p) r -= p;
    return (uint64_t)r;
  }
  MODLIN_HD uint64_t add(uint64_t a, uint64_t b) const {
    const uint64_t s = a + b;
    return s >= p ? s - p : s;
  }
  MODLIN_HD uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + p - b; }
  MODLIN_HD uint64_t mul(uint64_t a, uint64_t b) const { return reduce((u128)a * b); }
  // Full product of two residues, for lazy accumulation.
  MODLIN_HD u128 prod(uint64_t a, uint64_t b) const { return (u128)a * b; }
  // Exact residue of a sum of at most two products of residues.
  MODLIN_HD uint64_t reduce2(u128 t) const { return reduce(t); }
  // Number of (p-1)^2 products a u128 accumulator holds before it must be reduced.
  MODLIN_HD uint64_t safe_batch() const { return sb; }
  MODLIN_HD uint64_t modulus() const { return p; }
};

// p < 2^32: residues fit in 32 bits, so a product is one 32x32->64 multiply
// and a single product reduces with the 64-bit half of the Barrett
// reciprocal: q = hi64(x * mu_hi) is at most 2 below floor(x / p).
struct FpSmall {
  FpBarrett wide;  // reduction of u128 accumulators
  FpSmall() = default;
  MODLIN_HD explicit FpSmall(const FieldParams& f) : wide(f) {}
  MODLIN_HD uint64_t reduce(u128 t) const { return wide.reduce(t); }
  MODLIN_HD uint64_t reduce2(u128 t) const { return wide.reduce(t); }
  MODLIN_HD uint64_t reduce64(uint64_t x) const {
    const uint64_t q = (uint64_t)(((u128)x * wide.mu_hi) >> 64);
    uint64_t r = x - q * wide.p;
    if (r >= wide.p) r -= wide.p;
    if (r >= wide.p) r -= wide.p;
    return r;
  }
  MODLIN_HD uint64_t add(uint64_t a, uint64_t b) const { return wide.add(a, b); }
  MODLIN_HD uint64_t sub(uint64_t a, uint64_t b) const { return wide.sub(a, b); }
  MODLIN_HD uint64_t mul(uint64_t a, uint64_t b) const {
    return reduce64((uint64_t)(uint32_t)a * (uint32_t)b);
  }
  MODLIN_HD u128 prod(uint64_t a, uint64_t b) const { return (u128)((uint64_t)(uint32_t)a * (uint32_t)b); }
  MODLIN_HD uint64_t safe_batch() const { return wide.sb; }
  MODLIN_HD uint64_t modulus() const { return wide.p; }
};

struct FpM61 {
  FpM61() = default;
  MODLIN_HD explicit FpM61(const FieldParams&) {}
  MODLIN_HD static uint64_t fold(uint64_t x) { return (x & kM61) + (x >> 61); }
  // Exact t mod (2^61 - 1) for any 128-bit t: 2^64 = 8 (mod p).
  MODLIN_HD uint64_t reduce(u128 t) const {
    const uint64_t t0 = (uint64_t)t, t1 = (uint64_t)(t >> 64);
    uint64_t a = fold(t1);  // < 2^61 + 8
    if (a >= kM61) a -= kM61;
    const uint64_t a8 = ((a << 3) & kM61) + (a >> 58);  // 8a mod p, < 2^61 + 8
    uint64_t x = fold(t0) + a8;                          // < 2^62 + 16
    x = fold(x);
    if (x >= kM61) x -= kM61;
    return x;
  }
  MODLIN_HD uint64_t add(uint64_t a, uint64_t b) const {
    const uint64_t s = a + b;
    return s >= kM61 ? s - kM61 : s;
  }
  MODLIN_HD uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + kM61 - b; }
  MODLIN_HD uint64_t mul(uint64_t a, uint64_t b) const {
    const u128 t = (u128)a * b;  // < 2^122
    const uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
    uint64_t x = (lo & kM61) + ((lo >> 61) | (hi << 3));  // < 2^62
    x = fold(x);
    return x >= kM61 ? x - kM61 : x;
  }
  MODLIN_HD u128 prod(uint64_t a, uint64_t b) const { return (u128)a * b; }
  // t < 2^123 (a sum of at most two products of residues): t = hi 2^64 + lo
  // with hi < 2^59, and 2^64 = 8 (mod p), so (lo mod 2^61) + (lo >> 61) +
  // 8 hi < 2^63 needs one more fold.
  MODLIN_HD uint64_t reduce2(u128 t) const {
    const uint64_t lo = (uint64_t)t, hi = (uint64_t)(t >> 64);
    uint64_t x = (lo & kM61) + (lo >> 61) + (hi << 3);
    x = fold(x);
    return x >= kM61 ? x - kM61 : x;
  }
  MODLIN_HD uint64_t safe_batch() const { return 64; }
  MODLIN_HD uint64_t modulus() const { return kM61; }
};

// a^-1 mod 2^61 - 1 (a != 0) as a^(p-2), p - 2 = 2^61 - 3 = 4 (2^59 - 1) + 1.
// With x_k = a^(2^k - 1), x_(j+k) = x_j^(2^k) x_k builds x_59 from x_1 in 58
// squarings and 9 multiplications; then a^(p-2) = x_59^4 a. One dependent
// chain of 70 modular multiplications: about half the single-thread latency
// of the binary extended Euclid for this p.
MODLIN_HD uint64_t m61_sqn(uint64_t x, int n) {
  const FpM61 f;
  for (int i = 0; i < n; ++i) x = f.mul(x, x);
  return x;
}
MODLIN_HD uint64_t fp_inv_m61(uint64_t a) {
  const FpM61 f;
  const uint64_t x2 = f.mul(m61_sqn(a, 1), a);
  const uint64_t x4 = f.mul(m61_sqn(x2, 2), x2);
  const uint64_t x8 = f.mul(m61_sqn(x4, 4), x4);
  const uint64_t x16 = f.mul(m61_sqn(x8, 8), x8);
  const uint64_t x32 = f.mul(m61_sqn(x16, 16), x16);
  const uint64_t x48 = f.mul(m61_sqn(x32, 16), x16);
  const uint64_t x56 = f.mul(m61_sqn(x48, 8), x8);
  const uint64_t x58 = f.mul(m61_sqn(x56, 2), x2);
  const uint64_t x59 = f.mul(m61_sqn(x58, 1), a);
  return f.mul(m61_sqn(x59, 2), a);
}

// src/fp.rs:97-113: Fermat inverse a^(p-2), a != 0.
template <class F>
MODLIN_HD uint64_t fp_pow(const F& f, uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = f.mul(r, a);
    a = f.mul(a, a);
    e >>= 1;
  }
  return r;
}
template <class F>
MODLIN_HD uint64_t fp_inv(const F& f, uint64_t a) {
  return fp_pow(f, a, f.modulus() - 2);
}

// Inverse of a (0 < a < p, p prime) by the binary extended Euclidean
// algorithm: invariants x1 * a = u and x2 * a = v (mod p), halving u or v and
// subtracting the smaller from the larger until one reaches 1. About
// 2 log2(p) short steps, against ~2 log2(p) dependent multiplications for
// Fermat; used where one thread computes an inverse while the others wait.
MODLIN_HD uint64_t fp_inv_binary(uint64_t a, uint64_t p) {
  uint64_t u = a, v = p, x1 = 1, x2 = 0;
  while (u != 1 && v != 1) {
    while ((u & 1) == 0) {
      u >>= 1;
      x1 = (x1 & 1) ? (x1 + p) >> 1 : x1 >> 1;  // x1 + p < 2^64 for p < 2^63
    }
    while ((v & 1) == 0) {
      v >>= 1;
      x2 = (x2 & 1) ? (x2 + p) >> 1 : x2 >> 1;
    }
    if (u >= v) {
      u -= v;
      x1 = x1 >= x2 ? x1 - x2 : x1 + p - x2;
    } else {
      v -= u;
      x2 = x2 >= x1 ? x2 - x1 : x2 + p - x1;
    }
  }
  return u == 1 ? x1 : x2;
}

}  // namespace modlin
