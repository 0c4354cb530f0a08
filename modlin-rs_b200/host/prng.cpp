// Generators under test (host): xoroshiro128++ and MIXMAX over 2^61 - 1.
//
// Restates src/prng.rs of the modlin crate, which selects one generator per
// build through a Cargo feature; here the kind is a runtime argument so one
// library serves every -R/-L run. MIXMAX is ROOT's MixMaxEngine<N, skip>
// (seed_spbox seeding, iterate_raw_vec, 61-bit outputs shifted left by 3).
#include <cstdint>
#include <cstring>
#include <new>

#include "../../include/modlin.h"

namespace {

constexpr uint64_t kMP = 2305843009213693951ULL;  // 2^61 - 1
constexpr int kMBits = 61;

inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
inline uint64_t mersenne_fold(uint64_t k) { return (k & kMP) + (k >> kMBits); }  // non-canonical, as ROOT

struct Xoroshiro {
  uint64_t s0, s1;
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
  uint64_t next() {  // src/prng.rs:75-83
    const uint64_t a = s0;
    uint64_t b = s1;
    const uint64_t r = rotl(a + b, 17) + a;
    b ^= a;
    s0 = rotl(a, 49) ^ b ^ (b << 21);
    s1 = rotl(b, 28);
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

}  // namespace

struct modlin_prng {
  int kind;
  Xoroshiro* xo;
  MixMax* mm;
};

extern "C" modlin_prng* modlin_prng_new(int kind, uint64_t seed, int* err) {
  auto* g = new (std::nothrow) modlin_prng{kind, nullptr, nullptr};
  if (!g) {
    if (err) *err = MODLIN_ENOMEM;
    return nullptr;
  }
  if (kind == MODLIN_PRNG_XOROSHIRO128PP) {
    g->xo = new Xoroshiro(seed);
  } else if (kind == MODLIN_PRNG_MIXMAX17 || kind == MODLIN_PRNG_MIXMAX240 || kind == MODLIN_PRNG_MIXMAX256) {
    g->mm = new MixMax();
    if (kind == MODLIN_PRNG_MIXMAX17) *g->mm = MixMax{17, 36, 0, 0, {}, 0, 0};                   // prng.rs:305
    if (kind == MODLIN_PRNG_MIXMAX240) *g->mm = MixMax{240, 51, 0, 487013230256099140ULL, {}, 0, 0};  // :284
    if (kind == MODLIN_PRNG_MIXMAX256) *g->mm = MixMax{256, 0, 2, UINT64_MAX, {}, 0, 0};          // :326
    if (!g->mm->seed(seed)) {
      modlin_prng_free(g);
      if (err) *err = MODLIN_EINVAL_ARG;
      return nullptr;
    }
  } else {
    delete g;
    if (err) *err = MODLIN_EINVAL_ARG;
    return nullptr;
  }
  if (err) *err = MODLIN_OK;
  return g;
}

extern "C" const char* modlin_prng_name(int kind) {
  switch (kind) {
    case MODLIN_PRNG_XOROSHIRO128PP: return "xoroshiro128++";                               // prng.rs:56
    case MODLIN_PRNG_MIXMAX240: return "MIXMAX (TRandomMixMax, N=240, s=487013230256099140)";  // :291
    case MODLIN_PRNG_MIXMAX17: return "MIXMAX (TRandomMixMax17, N=17)";                      // :312
    case MODLIN_PRNG_MIXMAX256: return "MIXMAX (TRandomMixMax256, N=256, skip=2)";           // :333
    default: return nullptr;
  }
}

extern "C" void modlin_prng_fill(modlin_prng* g, uint64_t* out, size_t count) {
  if (!g || !out) return;
  if (g->xo)
    for (size_t i = 0; i < count; ++i) out[i] = g->xo->next();
  else
    for (size_t i = 0; i < count; ++i) out[i] = g->mm->next();
}

extern "C" void modlin_prng_free(modlin_prng* g) {
  if (!g) return;
  delete g->xo;
  delete g->mm;
  delete g;
}
