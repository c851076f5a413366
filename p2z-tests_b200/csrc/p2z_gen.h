// p2z_gen.h -- the physics workload generator and the layer-mask generator,
// one track slot at a time, for the host (p2z_host.cpp, g++) and the device
// (p2z_gen.cu, nvcc) alike.  No counterpart in the reference, whose inputs are
// smeared copies of one seed track (its configs 1-2); this is the physics
// sample the benchmark runs: charge +-1, pT log-uniform, phi uniform, eta
// uniform, vertex z Gaussian, a correlated positive-definite covariance around
// the truth, and hits on z planes at the true helix point plus Gaussian noise.
//
// Every draw of slot s is a function of (seed, s, draw index) only (SplitMix64
// on a counter), so slots can be generated in any order or in parallel.  The
// host and the device evaluate the same double expressions; they can differ
// only where the C library's and CUDA's log / exp / sin / cos / tan / atan
// round a double differently (by 1 ulp), which moves a float output by one
// unit in the last place in rare cases.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "p2z.h"

#if defined(__CUDACC__)
#define P2Z_HD __host__ __device__ __forceinline__
#else
#define P2Z_HD inline
#endif

namespace p2z_gen {

constexpr int TRK_WORDS = 28;
constexpr int HIT_WORDS = 9;
constexpr double kPi = 3.141592653589793;

// SplitMix64 (Steele, Lea, Flood 2014) finaliser applied to a per-track key
// and a counter: the i-th draw of track t depends only on (seed, t, i).
P2Z_HD uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct TrackRng {
  uint64_t key, ctr;
  P2Z_HD TrackRng(uint64_t seed, uint64_t stream) : key(mix64(seed + 0x9E3779B97F4A7C15ull * (stream + 1))), ctr(0) {}
  P2Z_HD uint64_t bits() { return mix64(key + 0x9E3779B97F4A7C15ull * (++ctr)); }
  P2Z_HD double uniform() { return ((double)(bits() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }  // (0,1)
  P2Z_HD double normal() {  // Box-Muller, one variate per call
    const double u1 = uniform(), u2 = uniform();
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

// Cholesky of a symmetric 6x6 (row-major); false if not positive definite.
P2Z_HD bool cholesky6(const double A[6][6], double L[6][6]) {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) L[i][j] = 0.0;
  for (int j = 0; j < 6; ++j) {
    double d = A[j][j];
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
    if (!(d > 1e-12)) return false;
    L[j][j] = sqrt(d);
    for (int i = j + 1; i < 6; ++i) {
      double s = A[i][j];
      for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
      L[i][j] = s / L[j][j];
    }
  }
  return true;
}

P2Z_HD int sym(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Where the words of slot s live: AOSOA batches of width B (element e of the
// track at tb[t + e*B], of the hit on layer l at hb(l)[t + e*B]).
struct SlotView {
  float *tb;   // first word of the slot's batch
  float *hb0;  // first word of the batch's layer-0 hit batch
  int t, B;
};

// One real track slot: the state and covariance, and its hits on all layers.
// kf: the field constant (kfact); stream: the slot's global index.
P2Z_HD void generate_slot(const p2z_physics_params &p, double kf, int nlayer, uint64_t stream, const SlotView &v) {
  const int B = v.B, t = v.t;
  float *tb = v.tb;
  const double lpt0 = log(p.pt_min), lpt1 = log(p.pt_max);
  TrackRng r(p.seed, stream);
  const int q = r.uniform() < 0.5 ? -1 : 1;
  const double pt = exp(lpt0 + (lpt1 - lpt0) * r.uniform());
  const double ipt = 1.0 / pt;
  const double phi = -kPi + 2.0 * kPi * r.uniform();
  const double eta = p.eta_min + (p.eta_max - p.eta_min) * r.uniform();
  const double theta = 2.0 * atan(exp(-eta));
  const double vz = p.sigma_vz * r.normal();
  const double truth[6] = {0.0, 0.0, vz, ipt, phi, theta};
  const double sig[6] = {p.sig_xy, p.sig_xy, p.sig_z, p.rel_sig_ipt * ipt, p.sig_phi, p.sig_theta};
  // random correlation, |rho| <= rho_max, positive definite
  double rho[6][6], L[6][6];
  bool ok = false;
  for (int attempt = 0; attempt < 64 && !ok; ++attempt) {
    const double shrink = attempt < 32 ? 1.0 : pow(0.5, attempt - 31);
    for (int i = 0; i < 6; ++i) {
      rho[i][i] = 1.0;
      for (int j = 0; j < i; ++j) rho[i][j] = rho[j][i] = shrink * p.rho_max * (2.0 * r.uniform() - 1.0);
    }
    ok = cholesky6(rho, L);
  }
  if (!ok) {
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) rho[i][j] = i == j ? 1.0 : 0.0;
    cholesky6(rho, L);
  }
  // initial state = truth + D L n
  double n6[6];
  for (int i = 0; i < 6; ++i) n6[i] = r.normal();
  for (int i = 0; i < 6; ++i) {
    double acc = 0.0;
    for (int k = 0; k <= i; ++k) acc += L[i][k] * n6[k];
    tb[t + i * B] = (float)(truth[i] + sig[i] * acc);
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) tb[t + (6 + sym(i, j)) * B] = (float)(sig[i] * rho[i][j] * sig[j]);
  memcpy(&tb[t + 27 * B], &q, sizeof q);
  // hits on the planes, at the true helix point plus noise
  const double k = q * kf;
  const double cP = cos(phi), sP = sin(phi);
  const double tanT = tan(theta);
  for (int l = 0; l < nlayer; ++l) {
    const double zl = nlayer > 1 ? p.z_first + (p.z_last - p.z_first) * l / (nlayer - 1) : p.z_first;
    const double alpha = (zl - vz) * tanT * ipt / k;
    const double sa = sin(alpha), ca = cos(alpha);
    const double hx = truth[0] + k * pt * (cP * sa - sP * (1.0 - ca));
    const double hy = truth[1] + k * pt * (sP * sa + cP * (1.0 - ca));
    float *hb = v.hb0 + (int64_t)l * HIT_WORDS * B;
    hb[t + 0 * B] = (float)(hx + p.hit_sig_xy * r.normal());
    hb[t + 1 * B] = (float)(hy + p.hit_sig_xy * r.normal());
    hb[t + 2 * B] = (float)(zl + p.hit_sig_z * r.normal());
    const float vxy = (float)(p.hit_sig_xy * p.hit_sig_xy), vz2 = (float)(p.hit_sig_z * p.hit_sig_z);
    hb[t + 3 * B] = vxy;
    hb[t + 4 * B] = 0.f;
    hb[t + 5 * B] = vxy;
    hb[t + 6 * B] = 0.f;
    hb[t + 7 * B] = 0.f;
    hb[t + 8 * B] = vz2;
  }
}

// A padding slot: zero track and hits.
P2Z_HD void zero_slot(int nlayer, const SlotView &v) {
  for (int w = 0; w < TRK_WORDS; ++w) v.tb[v.t + w * v.B] = 0.f;
  for (int l = 0; l < nlayer; ++l)
    for (int w = 0; w < HIT_WORDS; ++w) v.hb0[(int64_t)l * HIT_WORDS * v.B + v.t + w * v.B] = 0.f;
}

// The layer mask of one real track (p2z_mask_layers): a contiguous run of L
// layers from layer 0, L uniform in [min_hits, max_hits], then each layer
// dropped with probability drop_prob while more than min_hits remain.
P2Z_HD uint32_t mask_slot(uint64_t seed, uint64_t stream, int min_hits, int max_hits, double drop_prob) {
  TrackRng r(seed ^ 0x5bd1e995ull, stream);
  const double span = (double)(max_hits - min_hits);
  const double f = floor(r.uniform() * (max_hits - min_hits + 1));
  const int L = min_hits + (int)(span < f ? span : f);
  uint32_t m = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
  int count = L;
  for (int l = 0; l < L; ++l) {
    if (count > min_hits && r.uniform() < drop_prob) {
      m &= ~(1u << l);
      --count;
    }
  }
  return m;
}

}  // namespace p2z_gen
