/*
 * p2z_physics_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C restatement of the physics workload that the benchmark runs (the
 * library's p2z_generate_physics): charge +-1, pT log-uniform, phi uniform,
 * eta uniform, vertex z Gaussian, a random positive-definite correlation
 * around diag(sigma), the initial state smeared from the truth with that
 * covariance, and hits on z planes at the true helix point plus Gaussian
 * noise with a diagonal 3x3 covariance.
 *
 * Purpose: the reference arm of the benchmark (the reference's own OpenMP
 * hot loop, compiled from its source into oracle/_ref) needs the same inputs
 * as the GPU arm without loading the product library.  A CPU test checks that
 * this file's output equals p2z_generate_physics word for word.
 *
 * The sample has no counterpart in the reference, whose inputs are smeared
 * copies of one seed track (src/propagate-toz-test_OMP.cpp:243-293); its
 * array layout is the reference's AOSOA (MPTRK / MPHIT, :69-125) with the
 * hits of a batch's layers contiguous (bHit, :215-217).
 *
 * Every draw of track slot s is a function of (seed, s, draw index) only:
 * SplitMix64's finaliser (Steele, Lea and Flood, 2014) applied to a per-slot
 * key plus a counter, uniform variates from its top 53 bits, normal variates
 * by Box-Muller (one per call).  Compiled with -ffp-contract=off, like the
 * library's host generator, so the double expressions round the same way.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define OPH_PI 3.141592653589793
#define OPH_GOLDEN 0x9E3779B97F4A7C15ull

/* The parameter block of the sample; field order and types are those of the
 * library's p2z_physics_params, so a caller can pass either. */
typedef struct oph_params {
  uint64_t seed;
  double pt_min, pt_max, eta_min, eta_max, sigma_vz;
  double sig_xy, sig_z, rel_sig_ipt, sig_phi, sig_theta, rho_max;
  double z_first, z_last;
  double hit_sig_xy, hit_sig_z;
  float kfact;
  int32_t nthreads;
} oph_params;

static uint64_t oph_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

typedef struct {
  uint64_t key, n;
} oph_rng;

static oph_rng oph_rng_for(uint64_t seed, uint64_t slot) {
  oph_rng r;
  r.key = oph_mix(seed + OPH_GOLDEN * (slot + 1));
  r.n = 0;
  return r;
}

static double oph_uniform(oph_rng *r) { /* in (0, 1) */
  r->n += 1;
  const uint64_t b = oph_mix(r->key + OPH_GOLDEN * r->n);
  return ((double)(b >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static double oph_normal(oph_rng *r) {
  const double u1 = oph_uniform(r);
  const double u2 = oph_uniform(r);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* Lower Cholesky factor of a symmetric 6x6; 0 when not positive definite
 * (a pivot at or below 1e-12). */
static int oph_chol(double a[6][6], double l[6][6]) {
  memset(l, 0, sizeof(double) * 36);
  for (int j = 0; j < 6; ++j) {
    double d = a[j][j];
    for (int k = 0; k < j; ++k) d -= l[j][k] * l[j][k];
    if (!(d > 1e-12)) return 0;
    l[j][j] = sqrt(d);
    for (int i = j + 1; i < 6; ++i) {
      double s = a[i][j];
      for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
      l[i][j] = s / l[j][j];
    }
  }
  return 1;
}

static int oph_packed(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

/* One track slot: tb is the first word of its MPTRK batch, hb the first word
 * of the batch's layer-0 MPHIT, t its lane, B the batch width. */
static void oph_slot(const oph_params *p, double kf, int nlayer, uint64_t slot, float *tb, float *hb, int t, int B) {
  const double lo = log(p->pt_min), hi = log(p->pt_max);
  oph_rng r = oph_rng_for(p->seed, slot);
  const int q = oph_uniform(&r) < 0.5 ? -1 : 1;
  const double pt = exp(lo + (hi - lo) * oph_uniform(&r));
  const double ipt = 1.0 / pt;
  const double phi = -OPH_PI + 2.0 * OPH_PI * oph_uniform(&r);
  const double eta = p->eta_min + (p->eta_max - p->eta_min) * oph_uniform(&r);
  const double theta = 2.0 * atan(exp(-eta));
  const double vz = p->sigma_vz * oph_normal(&r);
  const double truth[6] = {0.0, 0.0, vz, ipt, phi, theta};
  const double sig[6] = {p->sig_xy, p->sig_xy, p->sig_z, p->rel_sig_ipt * ipt, p->sig_phi, p->sig_theta};
  /* correlation: off-diagonals uniform in +-rho_max; redrawn while not
   * positive definite, halving the range after 32 draws; identity after 64 */
  double rho[6][6], l[6][6];
  int ok = 0;
  for (int a = 0; a < 64 && !ok; ++a) {
    const double shrink = a < 32 ? 1.0 : pow(0.5, a - 31);
    for (int i = 0; i < 6; ++i) {
      rho[i][i] = 1.0;
      for (int j = 0; j < i; ++j) {
        const double v = shrink * p->rho_max * (2.0 * oph_uniform(&r) - 1.0);
        rho[i][j] = v;
        rho[j][i] = v;
      }
    }
    ok = oph_chol(rho, l);
  }
  if (!ok) {
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) rho[i][j] = i == j ? 1.0 : 0.0;
    oph_chol(rho, l);
  }
  double n6[6];
  for (int i = 0; i < 6; ++i) n6[i] = oph_normal(&r);
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
    for (int k = 0; k <= i; ++k) s += l[i][k] * n6[k];
    tb[t + i * B] = (float)(truth[i] + sig[i] * s);
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) tb[t + (6 + oph_packed(i, j)) * B] = (float)(sig[i] * rho[i][j] * sig[j]);
  memcpy(&tb[t + 27 * B], &q, sizeof q);
  /* hits at the true helix point: the propagateToZ helix from the vertex
   * (src/propagate-toz-test_OMP.cpp:627-647) evaluated in double */
  const double k = q * kf;
  const double cp = cos(phi), sp = sin(phi), tt = tan(theta);
  const float vxy = (float)(p->hit_sig_xy * p->hit_sig_xy), vzz = (float)(p->hit_sig_z * p->hit_sig_z);
  for (int ly = 0; ly < nlayer; ++ly) {
    const double z = nlayer > 1 ? p->z_first + (p->z_last - p->z_first) * ly / (nlayer - 1) : p->z_first;
    const double al = (z - vz) * tt * ipt / k;
    const double sa = sin(al), ca = cos(al);
    const double x = truth[0] + k * pt * (cp * sa - sp * (1.0 - ca));
    const double y = truth[1] + k * pt * (sp * sa + cp * (1.0 - ca));
    float *h = hb + (int64_t)ly * 9 * B;
    h[t + 0 * B] = (float)(x + p->hit_sig_xy * oph_normal(&r));
    h[t + 1 * B] = (float)(y + p->hit_sig_xy * oph_normal(&r));
    h[t + 2 * B] = (float)(z + p->hit_sig_z * oph_normal(&r));
    h[t + 3 * B] = vxy;
    h[t + 4 * B] = 0.f;
    h[t + 5 * B] = vxy;
    h[t + 6 * B] = 0.f;
    h[t + 7 * B] = 0.f;
    h[t + 8 * B] = vzz;
  }
}

/* Uniform events: nevts * ntrks tracks (ntrks a multiple of bsize) in
 * nevts*ntrks/bsize MPTRK batches (trk_out) and nlayer MPHIT per batch
 * (hits_out).  kfact 0 in the parameters selects the reference's
 * 100/(-0.299792458*3.8112).  Returns 0, or 1 on a bad size. */
int oph_generate(const oph_params *p, int bsize, int64_t nevts, int64_t ntrks, int nlayer, float *trk_out,
                 float *hits_out) {
  if (bsize <= 0 || nevts < 0 || ntrks < 0 || ntrks % bsize || nlayer < 1 || nlayer > 32) return 1;
  const double kf = p->kfact != 0.f ? p->kfact : (double)(float)(100. / (-0.299792458 * 3.8112));
  const int64_t nslots = nevts * ntrks;
  for (int64_t s = 0; s < nslots; ++s) {
    const int64_t b = s / bsize;
    const int t = (int)(s % bsize);
    oph_slot(p, kf, nlayer, (uint64_t)s, trk_out + b * 28 * (int64_t)bsize,
             hits_out + b * (int64_t)nlayer * 9 * bsize, t, bsize);
  }
  return 0;
}
