/*
 * p2z_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * This file is the CPU oracle (the checker) for the propagate-to-z + Kalman
 * update hot path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it.  The product library never links
 * or calls it.
 *
 * It restates, in plain C, the reference benchmark's per-track arithmetic:
 *
 *   propagateToZ           src/propagate-toz-test_OMP.cpp:622-682
 *   MultHelixPropEndcap    src/propagate-toz-test_OMP.cpp:296-341
 *   MultHelixPropTranspEndcap src/propagate-toz-test_OMP.cpp:343-373
 *   KalmanUpdate_v2        src/propagate-toz-test_OMP.cpp:503-620
 *   driver hot loop        src/propagate-toz-test_OMP.cpp:731-748
 *
 * Three arithmetic flavours are provided:
 *
 *  - "f32": the reference's own FP32 semantics.  Every sub-expression keeps the
 *    C type the reference gives it: the double literals `1.` in
 *    `1./ipt`, `1.0/cosT`, `(1.-cosa)`, `(1.-sinP*sCosPsina)`, `(1.-cCosPsina)`
 *    promote their sub-expression to double, the 2x2 determinant is formed in
 *    double and `1.f/det` is a double division.  Sums are evaluated left to
 *    right exactly as written in the reference.  Compiled with
 *    -ffp-contract=off this reproduces the reference (also built with
 *    -ffp-contract=off) bit for bit; the tests check that.
 *
 *  - "f64": the same estimator with every quantity in double and sin/cos in
 *    double.  This is the FP64 host oracle against which the error of every
 *    output parameter and covariance element is stated.
 *
 *  - "3x3 Joseph" (f64 only): a full (x,y,z) measurement update with the 3x3
 *    residual covariance H C H^T + V inverted by cofactors and the covariance
 *    updated in the symmetric Joseph form (I-KH) C (I-KH)^T + K V K^T.  The
 *    reference's KalmanUpdate (v1, src/propagate-toz-test_OMP.cpp:375-501) is
 *    a 3x3 update but it indexes the packed covariance as if it were a full
 *    6x6 and writes pt into the ipt slot; it is off the reference's active
 *    path (:743 is commented out).  This oracle states the correct 3x3 algebra
 *    instead; it is the reference for the product's 3x3 variants only.
 *
 * Data layout (the reference's "matriplex" AOSOA, :57-125): a batch of B
 * tracks stores element p of track t at data[t + p*B].  One MPTRK batch is
 * 6*B floats of parameters, 21*B floats of packed lower-triangular
 * covariance and B ints of charge.  One MPHIT batch is 3*B floats of
 * position and 6*B floats of packed 3x3 covariance.  Hits of one track batch
 * are stored layer-contiguous: hit batch index = layer + nlayer*batch
 * (bHit, :215-217).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Built twice: with the C library's sinf/cosf (the reference's own calls) and,
 * with -DORC_CR_TRIG, with correctly rounded sin/cos (a double evaluation
 * rounded once to float). */
#ifdef ORC_CR_TRIG
static inline float orc_sinf(float x) { return (float)sin((double)x); }
static inline float orc_cosf(float x) { return (float)cos((double)x); }
#define sinf orc_sinf
#define cosf orc_cosf
#endif

#define ORC_NPAR 6
#define ORC_NCOV 21
#define ORC_TRK_WORDS 28 /* 6 par + 21 cov + 1 charge, per track, per batch lane */
#define ORC_HIT_WORDS 9  /* 3 pos + 6 cov */

/* kfact of the OMP/TBB/CUDA_v4 family, src/propagate-toz-test_OMP.cpp:622:
 * 100/(-0.299792458*3.8112), evaluated in double and stored as float. */
float orc_default_kfact(void) { return (float)(100. / (-0.299792458 * 3.8112)); }

/* ------------------------------------------------------------------------ */
/* AOSOA <-> per-track gathers                                               */
/* ------------------------------------------------------------------------ */

typedef struct { float par[6]; float cov[21]; int q; } orc_trk32;
typedef struct { double par[6]; double cov[21]; int q; } orc_trk64;

static void gather_trk32(const float *batch, int B, int t, orc_trk32 *o) {
  for (int p = 0; p < 6; ++p) o->par[p] = batch[t + p * B];
  for (int p = 0; p < 21; ++p) o->cov[p] = batch[6 * B + t + p * B];
  int qv;
  memcpy(&qv, &batch[27 * B + t], sizeof(int));
  o->q = qv;
}

static void scatter_trk32(float *batch, int B, int t, const orc_trk32 *o) {
  for (int p = 0; p < 6; ++p) batch[t + p * B] = o->par[p];
  for (int p = 0; p < 21; ++p) batch[6 * B + t + p * B] = o->cov[p];
  memcpy(&batch[27 * B + t], &o->q, sizeof(int));
}

static void gather_hit(const float *hb, int B, int t, float pos[3], float cov[6]) {
  for (int p = 0; p < 3; ++p) pos[p] = hb[t + p * B];
  for (int p = 0; p < 6; ++p) cov[p] = hb[3 * B + t + p * B];
}

/* ------------------------------------------------------------------------ */
/* FP32 restatement with the reference's promotion rules                     */
/* ------------------------------------------------------------------------ */

/* Helix propagation of one track to the plane z = hpos[2].
 * Follows src/propagate-toz-test_OMP.cpp:627-682.  The Jacobian J (6x6,
 * identity plus 11 entries) is applied as C' = J C J^T in the two steps
 * of MultHelixPropEndcap (T = J C, :306-340) and MultHelixPropTranspEndcap
 * (C' = T J^T, :353-372), keeping their summation order. */
static void propagate_f32(orc_trk32 *s, const float hpos[3], float kfact) {
  const float zout = hpos[2];
  const float k = s->q * kfact;
  const float deltaZ = zout - s->par[2];
  const float ipt = s->par[3];
  const float pt = 1. / ipt;               /* double division, stored float */
  const float cosP = cosf(s->par[4]);
  const float sinP = sinf(s->par[4]);
  const float cosT = cosf(s->par[5]);
  const float sinT = sinf(s->par[5]);
  const float pxin = cosP * pt;
  const float pyin = sinP * pt;
  const float icosT = 1.0 / cosT;          /* double division, stored float */
  const float icosTk = icosT / k;
  const float alpha = deltaZ * sinT * ipt * icosTk;
  const float sina = sinf(alpha);
  const float cosa = cosf(alpha);

  const float x0 = s->par[0], y0 = s->par[1], phi0 = s->par[4];
  /* (1.-cosa) is double, so the bracket and the product with k are double */
  s->par[0] = x0 + k * (pxin * sina - pyin * (1. - cosa));
  s->par[1] = y0 + k * (pyin * sina + pxin * (1. - cosa));
  s->par[2] = zout;
  s->par[4] = phi0 + alpha;

  const float sCosPsina = sinf(cosP * sina);
  const float cCosPsina = cosf(cosP * sina);

  /* J stored row-major 6x6; only the non-identity entries are non-zero. */
  float J[36];
  for (int i = 0; i < 36; ++i) J[i] = 0.f;
  for (int i = 0; i < 6; ++i) J[i * 6 + i] = 1.f;
  J[0 * 6 + 2] = cosP * sinT * (sinP * cosa * sCosPsina - cosa) * icosT;
  J[0 * 6 + 3] = cosP * sinT * deltaZ * cosa * (1. - sinP * sCosPsina) * (icosT * pt) -
                 k * (cosP * sina - sinP * (1. - cCosPsina)) * (pt * pt);
  J[0 * 6 + 4] = (k * pt) * (-sinP * sina + sinP * sinP * sina * sCosPsina - cosP * (1. - cCosPsina));
  J[0 * 6 + 5] = cosP * deltaZ * cosa * (1. - sinP * sCosPsina) * (icosT * icosT);
  J[1 * 6 + 2] = cosa * sinT * (cosP * cosP * sCosPsina - sinP) * icosT;
  J[1 * 6 + 3] = sinT * deltaZ * cosa * (cosP * cosP * sCosPsina + sinP) * (icosT * pt) -
                 k * (sinP * sina + cosP * (1. - cCosPsina)) * (pt * pt);
  J[1 * 6 + 4] = (k * pt) * (-sinP * (1. - cCosPsina) - sinP * cosP * sina * sCosPsina + cosP * sina);
  J[1 * 6 + 5] = deltaZ * cosa * (cosP * cosP * sCosPsina + sinP) * (icosT * icosT);
  J[4 * 6 + 2] = -ipt * sinT * (icosTk);
  J[4 * 6 + 3] = sinT * deltaZ * (icosTk);
  J[4 * 6 + 5] = ipt * deltaZ * (icosT * icosTk);

  const float *a = J;
  const float *b = s->cov;
  float t[36];
  /* T = J C.  Rows 0, 1 and 4 carry the Jacobian; row 2 (z) is zero, rows 3
   * and 5 are copies of C's rows (ipt and theta are not changed). */
  t[0] = b[0] + a[2] * b[3] + a[3] * b[6] + a[4] * b[10] + a[5] * b[15];
  t[1] = b[1] + a[2] * b[4] + a[3] * b[7] + a[4] * b[11] + a[5] * b[16];
  t[2] = b[3] + a[2] * b[5] + a[3] * b[8] + a[4] * b[12] + a[5] * b[17];
  t[3] = b[6] + a[2] * b[8] + a[3] * b[9] + a[4] * b[13] + a[5] * b[18];
  t[4] = b[10] + a[2] * b[12] + a[3] * b[13] + a[4] * b[14] + a[5] * b[19];
  t[5] = b[15] + a[2] * b[17] + a[3] * b[18] + a[4] * b[19] + a[5] * b[20];
  t[6] = b[1] + a[8] * b[3] + a[9] * b[6] + a[10] * b[10] + a[11] * b[15];
  t[7] = b[2] + a[8] * b[4] + a[9] * b[7] + a[10] * b[11] + a[11] * b[16];
  t[8] = b[4] + a[8] * b[5] + a[9] * b[8] + a[10] * b[12] + a[11] * b[17];
  t[9] = b[7] + a[8] * b[8] + a[9] * b[9] + a[10] * b[13] + a[11] * b[18];
  t[10] = b[11] + a[8] * b[12] + a[9] * b[13] + a[10] * b[14] + a[11] * b[19];
  t[11] = b[16] + a[8] * b[17] + a[9] * b[18] + a[10] * b[19] + a[11] * b[20];
  t[12] = 0; t[13] = 0; t[14] = 0; t[15] = 0; t[16] = 0; t[17] = 0;
  t[18] = b[6]; t[19] = b[7]; t[20] = b[8]; t[21] = b[9]; t[22] = b[13]; t[23] = b[18];
  t[24] = a[26] * b[3] + a[27] * b[6] + b[10] + a[29] * b[15];
  t[25] = a[26] * b[4] + a[27] * b[7] + b[11] + a[29] * b[16];
  t[26] = a[26] * b[5] + a[27] * b[8] + b[12] + a[29] * b[17];
  t[27] = a[26] * b[8] + a[27] * b[9] + b[13] + a[29] * b[18];
  t[28] = a[26] * b[12] + a[27] * b[13] + b[14] + a[29] * b[19];
  t[29] = a[26] * b[17] + a[27] * b[18] + b[19] + a[29] * b[20];
  t[30] = b[15]; t[31] = b[16]; t[32] = b[17]; t[33] = b[18]; t[34] = b[19]; t[35] = b[20];

  /* C' = T J^T, packed lower triangle (:353-372). */
  float *c = s->cov;
  const float *tb = t;
  c[0] = tb[0] + tb[2] * a[2] + tb[3] * a[3] + tb[4] * a[4] + tb[5] * a[5];
  c[1] = tb[6] + tb[8] * a[2] + tb[9] * a[3] + tb[10] * a[4] + tb[11] * a[5];
  c[2] = tb[7] + tb[8] * a[8] + tb[9] * a[9] + tb[10] * a[10] + tb[11] * a[11];
  c[3] = tb[12] + tb[14] * a[2] + tb[15] * a[3] + tb[16] * a[4] + tb[17] * a[5];
  c[4] = tb[13] + tb[14] * a[8] + tb[15] * a[9] + tb[16] * a[10] + tb[17] * a[11];
  c[5] = 0;
  c[6] = tb[18] + tb[20] * a[2] + tb[21] * a[3] + tb[22] * a[4] + tb[23] * a[5];
  c[7] = tb[19] + tb[20] * a[8] + tb[21] * a[9] + tb[22] * a[10] + tb[23] * a[11];
  c[8] = 0;
  c[9] = tb[21];
  c[10] = tb[24] + tb[26] * a[2] + tb[27] * a[3] + tb[28] * a[4] + tb[29] * a[5];
  c[11] = tb[25] + tb[26] * a[8] + tb[27] * a[9] + tb[28] * a[10] + tb[29] * a[11];
  c[12] = 0;
  c[13] = tb[27];
  c[14] = tb[26] * a[26] + tb[27] * a[27] + tb[28] + tb[29] * a[29];
  c[15] = tb[30] + tb[32] * a[2] + tb[33] * a[3] + tb[34] * a[4] + tb[35] * a[5];
  c[16] = tb[31] + tb[32] * a[8] + tb[33] * a[9] + tb[34] * a[10] + tb[35] * a[11];
  c[17] = 0;
  c[18] = tb[33];
  c[19] = tb[32] * a[26] + tb[33] * a[27] + tb[34] + tb[35] * a[29];
  c[20] = tb[35];
}

/* 2-D (x,y) Kalman update, src/propagate-toz-test_OMP.cpp:503-620.
 * R = C[0..2] + V[0..2]; its determinant is formed in double from the float
 * entries and 1.f/det is a double division rounded to float; the gain K is
 * 6x2; the covariance update is C - K (H C) with H selecting x and y. */
static void update_v2_f32(orc_trk32 *s, const float hpos[3], const float hcov[6]) {
  float *C = s->cov;
  float r00 = C[0] + hcov[0];
  float r01 = C[1] + hcov[1];
  float r11 = C[2] + hcov[2];
  {
    const double det = (double)r00 * r11 - (double)r01 * r01;
    const float sc = 1.f / det;
    const float tmp = sc * r11;
    r01 *= -sc;
    r11 = sc * r00;
    r00 = tmp;
  }
  float K[12];
  K[0] = C[0] * r00 + C[1] * r01;
  K[1] = C[0] * r01 + C[1] * r11;
  K[2] = C[1] * r00 + C[2] * r01;
  K[3] = C[1] * r01 + C[2] * r11;
  K[4] = C[3] * r00 + C[4] * r01;
  K[5] = C[3] * r01 + C[4] * r11;
  K[6] = C[6] * r00 + C[7] * r01;
  K[7] = C[6] * r01 + C[7] * r11;
  K[8] = C[10] * r00 + C[11] * r01;
  K[9] = C[10] * r01 + C[11] * r11;
  K[10] = C[15] * r00 + C[16] * r01;
  K[11] = C[15] * r01 + C[16] * r11;

  const float res0 = hpos[0] - s->par[0];
  const float res1 = hpos[1] - s->par[1];
  float *P = s->par;
  P[0] = P[0] + K[0] * res0 + K[1] * res1;
  P[1] = P[1] + K[2] * res0 + K[3] * res1;
  P[2] = P[2] + K[4] * res0 + K[5] * res1;
  P[3] = P[3] + K[6] * res0 + K[7] * res1;
  P[4] = P[4] + K[8] * res0 + K[9] * res1;
  P[5] = P[5] + K[10] * res0 + K[11] * res1;

  float e[21];
  e[0] = K[0] * C[0] + K[1] * C[1];
  e[1] = K[2] * C[0] + K[3] * C[1];
  e[2] = K[2] * C[1] + K[3] * C[2];
  e[3] = K[4] * C[0] + K[5] * C[1];
  e[4] = K[4] * C[1] + K[5] * C[2];
  e[5] = K[4] * C[3] + K[5] * C[4];
  e[6] = K[6] * C[0] + K[7] * C[1];
  e[7] = K[6] * C[1] + K[7] * C[2];
  e[8] = K[6] * C[3] + K[7] * C[4];
  e[9] = K[6] * C[6] + K[7] * C[7];
  e[10] = K[8] * C[0] + K[9] * C[1];
  e[11] = K[8] * C[1] + K[9] * C[2];
  e[12] = K[8] * C[3] + K[9] * C[4];
  e[13] = K[8] * C[6] + K[9] * C[7];
  e[14] = K[8] * C[10] + K[9] * C[11];
  e[15] = K[10] * C[0] + K[11] * C[1];
  e[16] = K[10] * C[1] + K[11] * C[2];
  e[17] = K[10] * C[3] + K[11] * C[4];
  e[18] = K[10] * C[6] + K[11] * C[7];
  e[19] = K[10] * C[10] + K[11] * C[11];
  e[20] = K[10] * C[15] + K[11] * C[16];
  for (int i = 0; i < 21; ++i) C[i] = C[i] - e[i];
}

/* ------------------------------------------------------------------------ */
/* FP64 oracle: same estimator, all arithmetic in double                     */
/* ------------------------------------------------------------------------ */

/* Packed lower-triangular index of (i,j) in a symmetric n x n matrix. */
static int sym_idx(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

static void propagate_f64(orc_trk64 *s, const double hpos[3], double kfact) {
  const double zout = hpos[2];
  const double k = s->q * kfact;
  const double dz = zout - s->par[2];
  const double ipt = s->par[3];
  const double pt = 1.0 / ipt;
  const double cP = cos(s->par[4]), sP = sin(s->par[4]);
  const double cT = cos(s->par[5]), sT = sin(s->par[5]);
  const double px = cP * pt, py = sP * pt;
  const double icT = 1.0 / cT;
  const double icTk = icT / k;
  const double alpha = dz * sT * ipt * icTk;
  const double sa = sin(alpha), ca = cos(alpha);
  s->par[0] += k * (px * sa - py * (1.0 - ca));
  s->par[1] += k * (py * sa + px * (1.0 - ca));
  s->par[2] = zout;
  s->par[4] += alpha;
  const double sC = sin(cP * sa), cC = cos(cP * sa);

  double J[6][6];
  memset(J, 0, sizeof J);
  for (int i = 0; i < 6; ++i) J[i][i] = 1.0;
  J[0][2] = cP * sT * (sP * ca * sC - ca) * icT;
  J[0][3] = cP * sT * dz * ca * (1.0 - sP * sC) * (icT * pt) - k * (cP * sa - sP * (1.0 - cC)) * (pt * pt);
  J[0][4] = (k * pt) * (-sP * sa + sP * sP * sa * sC - cP * (1.0 - cC));
  J[0][5] = cP * dz * ca * (1.0 - sP * sC) * (icT * icT);
  J[1][2] = ca * sT * (cP * cP * sC - sP) * icT;
  J[1][3] = sT * dz * ca * (cP * cP * sC + sP) * (icT * pt) - k * (sP * sa + cP * (1.0 - cC)) * (pt * pt);
  J[1][4] = (k * pt) * (-sP * (1.0 - cC) - sP * cP * sa * sC + cP * sa);
  J[1][5] = dz * ca * (cP * cP * sC + sP) * (icT * icT);
  J[4][2] = -ipt * sT * icTk;
  J[4][3] = sT * dz * icTk;
  J[4][5] = ipt * dz * (icT * icTk);
  /* The reference's Endcap products set row/column 2 (z) of the result to
   * zero: T row 2 is written as 0 and C'(2,j) is 0.  Use J with row 2 zeroed
   * to reproduce that algebra exactly. */
  for (int j = 0; j < 6; ++j) J[2][j] = 0.0;

  double Cf[6][6], T[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Cf[i][j] = s->cov[sym_idx(i, j)];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double acc = 0.0;
      for (int m = 0; m < 6; ++m) acc += J[i][m] * Cf[m][j];
      T[i][j] = acc;
    }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double acc = 0.0;
      for (int m = 0; m < 6; ++m) acc += T[i][m] * J[j][m];
      s->cov[sym_idx(i, j)] = acc;
    }
}

static void update_v2_f64(orc_trk64 *s, const double hpos[3], const double hcov[6]) {
  double *C = s->cov;
  const double r00 = C[0] + hcov[0], r01 = C[1] + hcov[1], r11 = C[2] + hcov[2];
  const double det = r00 * r11 - r01 * r01;
  const double i00 = r11 / det, i01 = -r01 / det, i11 = r00 / det;
  /* rows of C H^T: (C_i0, C_i1) for i = 0..5 */
  double K[6][2];
  for (int i = 0; i < 6; ++i) {
    const double ci0 = C[sym_idx(i, 0)], ci1 = C[sym_idx(i, 1)];
    K[i][0] = ci0 * i00 + ci1 * i01;
    K[i][1] = ci0 * i01 + ci1 * i11;
  }
  const double r0 = hpos[0] - s->par[0], r1 = hpos[1] - s->par[1];
  for (int i = 0; i < 6; ++i) s->par[i] += K[i][0] * r0 + K[i][1] * r1;
  double n[21];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j)
      n[sym_idx(i, j)] = C[sym_idx(i, j)] - (K[i][0] * C[sym_idx(0, j)] + K[i][1] * C[sym_idx(1, j)]);
  memcpy(C, n, sizeof n);
}

/* 3-D (x,y,z) update with the Joseph-form covariance. */
static void update_3x3_joseph_f64(orc_trk64 *s, const double hpos[3], const double hcov[6]) {
  double *C = s->cov;
  double R[3][3], V[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      V[i][j] = hcov[sym_idx(i, j)];
      R[i][j] = C[sym_idx(i, j)] + V[i][j];
    }
  /* cofactor inverse */
  const double c00 = R[1][1] * R[2][2] - R[1][2] * R[2][1];
  const double c01 = R[1][2] * R[2][0] - R[1][0] * R[2][2];
  const double c02 = R[1][0] * R[2][1] - R[1][1] * R[2][0];
  const double det = R[0][0] * c00 + R[0][1] * c01 + R[0][2] * c02;
  double Ri[3][3];
  Ri[0][0] = c00 / det;
  Ri[0][1] = (R[0][2] * R[2][1] - R[0][1] * R[2][2]) / det;
  Ri[0][2] = (R[0][1] * R[1][2] - R[0][2] * R[1][1]) / det;
  Ri[1][0] = c01 / det;
  Ri[1][1] = (R[0][0] * R[2][2] - R[0][2] * R[2][0]) / det;
  Ri[1][2] = (R[0][2] * R[1][0] - R[0][0] * R[1][2]) / det;
  Ri[2][0] = c02 / det;
  Ri[2][1] = (R[0][1] * R[2][0] - R[0][0] * R[2][1]) / det;
  Ri[2][2] = (R[0][0] * R[1][1] - R[0][1] * R[1][0]) / det;

  double K[6][3];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int m = 0; m < 3; ++m) acc += C[sym_idx(i, m)] * Ri[m][j];
      K[i][j] = acc;
    }
  const double r[3] = {hpos[0] - s->par[0], hpos[1] - s->par[1], hpos[2] - s->par[2]};
  for (int i = 0; i < 6; ++i) s->par[i] += K[i][0] * r[0] + K[i][1] * r[1] + K[i][2] * r[2];

  /* P = (I - K H) C ; C'' = P (I - K H)^T + K V K^T */
  double Cf[6][6], P[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Cf[i][j] = C[sym_idx(i, j)];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) P[i][j] = Cf[i][j] - (K[i][0] * Cf[0][j] + K[i][1] * Cf[1][j] + K[i][2] * Cf[2][j]);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double a = P[i][j] - (P[i][0] * K[j][0] + P[i][1] * K[j][1] + P[i][2] * K[j][2]);
      double kvk = 0.0;
      for (int m = 0; m < 3; ++m)
        for (int n = 0; n < 3; ++n) kvk += K[i][m] * V[m][n] * K[j][n];
      C[sym_idx(i, j)] = a + kvk;
    }
}

/* ------------------------------------------------------------------------ */
/* Public oracle entry points                                                */
/* ------------------------------------------------------------------------ */

enum { ORC_UPDATE_V2 = 0, ORC_UPDATE_3X3_JOSEPH = 1 };

static int layer_present(const uint32_t *mask, int64_t slot, int layer) {
  return mask == NULL || ((mask[slot] >> layer) & 1u);
}

/* FP32 run in the reference's semantics over nbatch AOSOA batches of width B:
 * out = trk; for each layer present: propagate then update_v2 (:739-745).
 * mask (optional, one word per track slot, bit l = layer l present) skips
 * both steps on absent layers. */
void orc_run_f32(const float *trk, const float *hits, float *out, int64_t nbatch, int B, int nlayer,
                 const uint32_t *mask, float kfact) {
  for (int64_t ib = 0; ib < nbatch; ++ib) {
    const float *tb = trk + ib * (int64_t)ORC_TRK_WORDS * B;
    float *ob = out + ib * (int64_t)ORC_TRK_WORDS * B;
    for (int t = 0; t < B; ++t) {
      orc_trk32 s;
      gather_trk32(tb, B, t, &s);
      for (int l = 0; l < nlayer; ++l) {
        if (!layer_present(mask, ib * B + t, l)) continue;
        const float *hb = hits + ((int64_t)l + (int64_t)nlayer * ib) * ORC_HIT_WORDS * B;
        float hp[3], hc[6];
        gather_hit(hb, B, t, hp, hc);
        propagate_f32(&s, hp, kfact);
        update_v2_f32(&s, hp, hc);
      }
      scatter_trk32(ob, B, t, &s);
    }
  }
}

/* One step on one batch, for layer-by-layer checks.  which: 0 = propagate,
 * 1 = update_v2. */
void orc_step_f32(float *batch, const float *hitbatch, int B, int which, float kfact) {
  for (int t = 0; t < B; ++t) {
    orc_trk32 s;
    gather_trk32(batch, B, t, &s);
    float hp[3], hc[6];
    gather_hit(hitbatch, B, t, hp, hc);
    if (which == 0) propagate_f32(&s, hp, kfact);
    else update_v2_f32(&s, hp, hc);
    scatter_trk32(batch, B, t, &s);
  }
}

/* FP64 oracle run.  Inputs are the same float AOSOA arrays; outputs are per
 * track (slot order ib*B + t) 27 doubles: 6 parameters then 21 packed
 * covariance elements.  update: ORC_UPDATE_V2 or ORC_UPDATE_3X3_JOSEPH. */
void orc_run_f64(const float *trk, const float *hits, double *out, int64_t nbatch, int B, int nlayer,
                 const uint32_t *mask, double kfact, int update) {
  for (int64_t ib = 0; ib < nbatch; ++ib) {
    const float *tb = trk + ib * (int64_t)ORC_TRK_WORDS * B;
    for (int t = 0; t < B; ++t) {
      orc_trk32 s32;
      gather_trk32(tb, B, t, &s32);
      orc_trk64 s;
      for (int p = 0; p < 6; ++p) s.par[p] = s32.par[p];
      for (int p = 0; p < 21; ++p) s.cov[p] = s32.cov[p];
      s.q = s32.q;
      for (int l = 0; l < nlayer; ++l) {
        if (!layer_present(mask, ib * B + t, l)) continue;
        const float *hb = hits + ((int64_t)l + (int64_t)nlayer * ib) * ORC_HIT_WORDS * B;
        float hp32[3], hc32[6];
        gather_hit(hb, B, t, hp32, hc32);
        double hp[3], hc[6];
        for (int p = 0; p < 3; ++p) hp[p] = hp32[p];
        for (int p = 0; p < 6; ++p) hc[p] = hc32[p];
        propagate_f64(&s, hp, kfact);
        if (update == ORC_UPDATE_3X3_JOSEPH) update_3x3_joseph_f64(&s, hp, hc);
        else update_v2_f64(&s, hp, hc);
      }
      double *o = out + (ib * B + t) * 27;
      for (int p = 0; p < 6; ++p) o[p] = s.par[p];
      for (int p = 0; p < 21; ++p) o[6 + p] = s.cov[p];
    }
  }
}
