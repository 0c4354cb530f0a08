// Generators under test, host side: construction, names and the sequential
// stream (src/prng.rs). The state and step live in prng.h.
#include <cstdint>
#include <cstring>
#include <new>

#include "../../include/modlin.h"
#include "prng.h"

using modlin_prng_impl::MixMax;
using modlin_prng_impl::Xoroshiro;

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

extern "C" size_t modlin_prng_state_words(int kind) {
  switch (kind) {
    case MODLIN_PRNG_XOROSHIRO128PP: return 2;
    case MODLIN_PRNG_MIXMAX17: return 17 + 2;
    case MODLIN_PRNG_MIXMAX240: return 240 + 2;
    case MODLIN_PRNG_MIXMAX256: return 256 + 2;
    default: return 0;
  }
}

extern "C" int modlin_prng_get_state(const modlin_prng* g, uint64_t* words, size_t n) {
  if (!g || !words || n != modlin_prng_state_words(g->kind)) return MODLIN_EINVAL_ARG;
  if (g->xo) {
    words[0] = g->xo->s0;
    words[1] = g->xo->s1;
  } else {
    const MixMax& m = *g->mm;
    for (int i = 0; i < m.N; ++i) words[i] = m.v[i];
    words[m.N] = m.sumtot;
    words[m.N + 1] = (uint64_t)m.counter;
  }
  return MODLIN_OK;
}

extern "C" int modlin_prng_set_state(modlin_prng* g, const uint64_t* words, size_t n) {
  if (!g || !words || n != modlin_prng_state_words(g->kind)) return MODLIN_EINVAL_ARG;
  if (g->xo) {
    g->xo->s0 = words[0];
    g->xo->s1 = words[1];
    return MODLIN_OK;
  }
  MixMax& m = *g->mm;
  for (int i = 0; i <= m.N; ++i)
    if (words[i] > modlin_prng_impl::kMP) return MODLIN_EINVAL_ARG;
  if (words[m.N + 1] < 1 || words[m.N + 1] > (uint64_t)m.N) return MODLIN_EINVAL_ARG;
  for (int i = 0; i < m.N; ++i) m.v[i] = words[i];
  m.sumtot = words[m.N];
  m.counter = (int)words[m.N + 1];
  return MODLIN_OK;
}
