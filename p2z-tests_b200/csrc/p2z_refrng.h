// p2z_refrng.h -- the reference's input random stream, restated: the C
// library's rand() after srand(seed) and the reference's polar-method randn
// (src/propagate-toz-test_OMP.cpp:127-145) that turns it into N(0,1)
// variates.  Host code (p2z_host.cpp) uses it to reproduce the reference's
// prepareTracks / prepareHits bit for bit.
//
// rand() of the GNU C library with its default state is an additive lagged
// Fibonacci generator (the published description of glibc's TYPE_3
// random()): with r[0] = seed (1 when seed is 0), r[i] = 16807 r[i-1] mod
// (2^31 - 1) for i = 1..30 (Schrage's method), r[i] = r[i-31] for i = 31..33,
// r[i] = r[i-31] + r[i-3] mod 2^32 for i >= 34, the k-th output of rand() is
// r[k + 344] >> 1.  The state a draw needs is the last 31 words, which is what
// p2z_ref_rng carries (a plain struct: it can be copied and resumed).
#pragma once

#include <math.h>
#include <stdint.h>

#include "p2z.h"

#if defined(__CUDACC__)
#define P2Z_RNG_HD __host__ __device__ __forceinline__
#else
#define P2Z_RNG_HD inline
#endif

namespace p2z_refrng {

constexpr int kLag = 31;      // long lag
constexpr int kShort = 3;     // short lag
constexpr int kDiscard = 344; // index of the first output's word
constexpr float kRandMax = 2147483647.f;  // RAND_MAX as a float: 2^31

// State: ring[i % 31] holds r[i] for the 31 most recent words; `next` is the
// index of the word the next draw produces.
inline void seed(p2z_ref_rng *g, uint32_t s) {
  int32_t r[kDiscard];
  r[0] = s == 0 ? 1 : (int32_t)s;
  for (int i = 1; i < kLag; ++i) {
    const int64_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
    int64_t w = 16807 * lo - 2836 * hi;
    if (w < 0) w += 2147483647;
    r[i] = (int32_t)w;
  }
  for (int i = kLag; i < kLag + kShort; ++i) r[i] = r[i - kLag];
  for (int i = kLag + kShort; i < kDiscard; ++i) r[i] = (int32_t)((uint32_t)r[i - kLag] + (uint32_t)r[i - kShort]);
  for (int i = kDiscard - kLag; i < kDiscard; ++i) g->ring[i % kLag] = (uint32_t)r[i];
  g->next = kDiscard;
  g->have_second = 0;
  g->second = 0.f;
}

// One rand() output, in [0, 2^31).
inline int32_t draw(p2z_ref_rng *g) {
  const int64_t i = g->next++;
  const int j = (int)(i % kLag);
  const uint32_t w = g->ring[j] + g->ring[(i - kShort) % kLag];  // r[i-31] + r[i-3]
  g->ring[j] = w;
  return (int32_t)(w >> 1);
}

// One attempt of the polar method on two draws, with the reference's types:
// U = -1 + ((float)rand()/RAND_MAX)*2 in float, W = pow(U1,2) + pow(U2,2) in
// double stored to float.  Returns W (accepted when 0 < W < 1).  Shared by
// the host stream and the device generator (p2z_prep.cu).
P2Z_RNG_HD float attempt(int32_t d1, int32_t d2, float *u1, float *u2) {
  *u1 = -1 + ((float)d1 / kRandMax) * 2;
  *u2 = -1 + ((float)d2 / kRandMax) * 2;
  return (float)((double)*u1 * (double)*u1 + (double)*u2 * (double)*u2);
}

// randn(0, 1): the two variates of an accepted pair on consecutive calls,
// mult = sqrt(-2 log W / W) in float with the C library's logf and sqrtf.
inline float randn(p2z_ref_rng *g) {
  if (g->have_second) {
    g->have_second = 0;
    return 0.f + 1.f * g->second;
  }
  float u1, u2, w;
  do {
    const int32_t d1 = draw(g);
    const int32_t d2 = draw(g);
    w = attempt(d1, d2, &u1, &u2);
  } while (w >= 1 || w == 0);
  const float mult = sqrtf((-2 * logf(w)) / w);
  g->second = u2 * mult;
  g->have_second = 1;
  return 0.f + 1.f * (u1 * mult);
}

}  // namespace p2z_refrng
