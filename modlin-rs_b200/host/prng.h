// Generators under test (host state and sequential step): xoroshiro128++ and
// MIXMAX over 2^61 - 1. Shared by the host stream (prng.cpp) and the device
// fill (csrc/prng_kernels.cu), which must reproduce it bit for bit.
//
// Restates src/prng.rs of the modlin crate, which selects one generator per
// build through a Cargo feature; here the kind is a runtime argument so one
// library serves every -R/-L run. MIXMAX is ROOT's MixMaxEngine<N, skip>
// (seed_spbox seeding, iterate_raw_vec, 61-bit outputs shifted left by 3).
#pragma once
#include <cstdint>

namespace modlin_prng_impl {

constexpr uint64_t kMP = 2305843009213693951ULL;  // 2^61 - 1
constexpr int kMBits = 61;

inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
// ROOT's MOD_MERSENNE: one fold, not canonical. For arguments below 3 * 2^61
// (every sum MIXMAX folds) the result is at most 2^61 - 1, and it equals
// 2^61 - 1, the second representation of 0, only when the argument is = 0.
inline uint64_t mersenne_fold(uint64_t k) { return (k & kMP) + (k >> kMBits); }

struct Xoroshiro {
  uint64_t s0, s1;
  Xoroshiro() = default;
  explicit Xoroshiro(uint64_t seed) {  // src/prng.rs:58-72: SplitMix64 expansion
    uint64_t z = seed;
    auto sm = [&z]() {
      z += 0x9e3779b97f4a7c15ULL;
      uint64_t w = z;
      w = (w ^ (w >> 30)) * 0xbf58476d1ce4e5b9ULL;
      w = (w ^ (w >> 27)) * 0x94d049bb133111ebULL;
      return w ^ (w >> 31);
    };
    s0 = sm();
    s1 = sm();
  }
  // The state transition alone (GF(2)-linear in (s0, s1)).
  void step() {
    uint64_t b = s1 ^ s0;
    s0 = rotl(s0, 49) ^ b ^ (b << 21);
    s1 = rotl(b, 28);
  }
  uint64_t next() {  // src/prng.rs:75-83
    const uint64_t r = rotl(s0 + s1, 17) + s0;
    step();
    return r;
  }
};

// MixMax<N, SPECIALMUL, SPECIAL, SKIP> (src/prng.rs:133-270).
struct MixMax {
  int N, specialmul, skip;
  uint64_t special;  // UINT64_MAX stands for ROOT's -1 (N = 256)
  uint64_t v[256];
  uint64_t sumtot;
  int counter;

  static uint64_t fmodmul(uint64_t cum, uint64_t a, uint64_t b) {  // src/prng.rs:117-127
    const unsigned __int128 s = (unsigned __int128)a * b + cum;
    const uint64_t lo = (uint64_t)s, hi = (uint64_t)(s >> 64);
    return mersenne_fold((lo & kMP) + hi * 8 + (lo >> kMBits));
  }

  bool seed(uint64_t sd) {  // src/prng.rs:152-176, ROOT seed_spbox
    if (sd == 0) return false;
    uint64_t l = sd, acc = 0, ovf = 0;
    for (int i = 0; i < N; ++i) {
      l *= 6364136223846793005ULL;
      l = (l << 32) ^ (l >> 32);
      v[i] = l & kMP;
      const uint64_t t = acc + v[i];
      ovf += t < acc;
      acc = t;
    }
    sumtot = mersenne_fold(mersenne_fold(acc) + (ovf << 3));
    counter = N;
    return true;
  }

  void iterate() {  // src/prng.rs:191-222
    const uint64_t temp2 = v[1];
    uint64_t tv = sumtot, acc = tv, ovf = 0, tp = 0;
    v[0] = tv;
    for (int i = 1; i < N; ++i) {
      if (specialmul) {
        const uint64_t tpo = ((tp << specialmul) & kMP) | (tp >> (kMBits - specialmul));
        tp = mersenne_fold(tp + v[i]);
        tv = mersenne_fold(tv + tp + tpo);
      } else {
        tp = mersenne_fold(tp + v[i]);
        tv = mersenne_fold(tv + tp);
      }
      v[i] = tv;
      const uint64_t t = acc + tv;
      ovf += t < acc;
      acc = t;
    }
    if (special) {
      const uint64_t t2 = special == UINT64_MAX ? kMP - temp2 : fmodmul(0, special, temp2);
      v[2] = mersenne_fold(v[2] + t2);
      const uint64_t t = acc + t2;
      ovf += t < acc;
      acc = t;
    }
    sumtot = mersenne_fold(mersenne_fold(acc) + (ovf << 3));
  }

  uint64_t next() {  // src/prng.rs:243-269: next_raw() << 3
    const int c = counter;
    if (c >= N)
      for (int k = 0; k < skip; ++k) iterate();
    counter = c;
    uint64_t raw;
    if (counter < N) {
      raw = v[counter++];
    } else {
      iterate();
      counter = 2;
      raw = v[1];
    }
    return raw << 3;
  }
};

}  // namespace modlin_prng_impl

struct modlin_prng {
  int kind;
  modlin_prng_impl::Xoroshiro* xo;
  modlin_prng_impl::MixMax* mm;
};
