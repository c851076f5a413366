// p2z_math.cuh -- per-track device arithmetic of the propagate-to-z + Kalman
// update hot path.
//
// Each function works on one track held in registers.  The algebra is the
// reference's propagateToZ (src/propagate-toz-test_OMP.cpp:623-682) with its two
// covariance products MultHelixPropEndcap (:296-341) and
// MultHelixPropTranspEndcap (:343-373), followed by KalmanUpdate_v2 (:503-620).
//
// Two evaluation forms of that algebra are provided:
//
// FORM_PRECISE (the default): FP32 arithmetic, no FP64 instruction, evaluated
//   so that it agrees with an all-FP64 evaluation to a few 1e-6 in the
//   parameters.  Three changes from the reference's FP32 evaluation, all exact
//   in real arithmetic:
//   * 1 - cos(a), for the helix angle a = alpha and for a = cosP*sin(alpha),
//     is computed as the versine directly (a Taylor series of
//     a^2/2 - a^4/24 + ..., or 2 sin^2(a/2)) instead of subtracting a rounded
//     cosine from 1.  For high-pT tracks R*(1 - cos alpha) is the curvature
//     (sagitta) signal and the subtraction in FP32 loses most of its digits,
//     which the reference's FP32 build turns into ~1e-4 relative error in q/pT
//     and ~1e-3 in the covariance.
//   * x and y are carried as anchored positions (the last hit's coordinate,
//     exact, plus an FP32 offset) -- or as float pairs, or in FP64 for the
//     all-FP64 kernel: positions of tens of cm held in FP32 round at ~4e-6 cm,
//     which against 30 um hits biases the curvature.
//   * the direction (cos/sin phi, tan theta) is an anchor advanced once per
//     step by the angle increments summed since the anchor, instead of sin/cos
//     of rounded accumulated angles (see Trk and propagate_params_precise).
// FORM_REFERENCE: the reference's FP32 evaluation operation for operation,
//   including its C type promotions (the double literals in `1./ipt`,
//   `1.0/cosT`, `(1.-cosa)` ... and the double determinant), for callers who
//   want the reference's own rounding.  Compiled without FMA contraction and
//   with correctly rounded sin/cos, it reproduces the reference built with
//   -ffp-contract=off.
//
// Structure exploited (exact for finite inputs, both forms):
//  * The Endcap products zero row and column 2 (z) of the propagated
//    covariance, so after the first propagation only 15 of 21 covariance
//    elements are live; every product with a z entry is a product with +-0.
//  * The update after a propagation then has a zero z row in its gain: z stays
//    at the hit's z and the z row/column stays zero.
// The first present layer of a track therefore runs the general propagation
// on the full 21-element input covariance; later layers run the reduced form.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

namespace p2z {

enum { SC_ACCURATE = 0, SC_FAST = 1 };
enum { FORM_PRECISE = 0, FORM_REFERENCE = 1 };

// ---------------------------------------------------------------------------
// Accumulators for x, y, phi
// ---------------------------------------------------------------------------
// A float pair (hi + lo) with error-free additions (Knuth's TwoSum followed by
// a Fast2Sum renormalisation) -- the FP64-free wide accumulator.
struct DF {
  float hi, lo;
};

// An anchored position: the last hit's coordinate a (a float read from
// memory, exact) plus a float offset u.  Offsets stay of the order of one
// step, so they round ~10x finer than the coordinate itself, and the Kalman
// residual (h - a) - u is formed without cancellation error beyond the
// rounding of h - a.  All FP32, full rate.
struct AP {
  float a, u;
};

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(AP v) { return v.a + v.u; }
__device__ __forceinline__ float tof(double v) { return (float)v; }
__device__ __forceinline__ float tof(DF v) { return v.hi + v.lo; }

__device__ __forceinline__ void acc_set(float &a, float v) { a = v; }
__device__ __forceinline__ void acc_set(double &a, float v) { a = v; }
__device__ __forceinline__ void acc_set(double &a, double v) { a = v; }
__device__ __forceinline__ void acc_set(DF &a, float v) { a.hi = v; a.lo = 0.f; }
__device__ __forceinline__ void acc_set(AP &a, float v) { a.a = v; a.u = 0.f; }
__device__ __forceinline__ void acc_add(AP &a, float d) { a.u += d; }

// A float accumulator adds with an explicit rounding: an increment that is also
// used elsewhere (the helix angle, the Kalman corrections of phi and theta) must
// not be fused into the addition in one kernel and not in another, so that
// every schedule computes the same bits.
__device__ __forceinline__ void acc_add(float &a, float d) { a = __fadd_rn(a, d); }
__device__ __forceinline__ void acc_add(double &a, float d) { a += (double)d; }
__device__ __forceinline__ void acc_add(double &a, double d) { a += d; }
__device__ __forceinline__ void acc_add(DF &a, float d) {
  const float s = __fadd_rn(a.hi, d);
  const float bp = __fsub_rn(s, a.hi);
  const float e = __fadd_rn(__fsub_rn(a.hi, __fsub_rn(s, bp)), __fsub_rn(d, bp));  // exact: a.hi + d - s
  const float lo = __fadd_rn(a.lo, e);
  const float hi = __fadd_rn(s, lo);
  a.lo = __fsub_rn(lo, __fsub_rn(hi, s));
  a.hi = hi;
}

// h - a, rounded to float (the Kalman residual against a wide accumulator).
__device__ __forceinline__ float acc_res(float h, float a) { return h - a; }
__device__ __forceinline__ float acc_res(float h, double a) { return (float)((double)h - a); }
__device__ __forceinline__ float acc_res(float h, DF a) { return __fsub_rn(__fsub_rn(h, a.hi), a.lo); }
__device__ __forceinline__ double acc_res(double h, double a) { return h - a; }
__device__ __forceinline__ float acc_res(float h, AP a) { return (h - a.a) - a.u; }

// After a Kalman update with residual res = h - x and increment inc, the new
// position is x + inc.  AP re-anchors at the hit: x + inc = h + (inc - res).
__device__ __forceinline__ void acc_update(AP &a, float h, float res, float inc) {
  a.a = h;
  a.u = inc - res;
}
template <typename A, typename T>
__device__ __forceinline__ void acc_update(A &a, T h, T res, T inc) {
  (void)h;
  (void)res;
  acc_add(a, inc);
}

// Reciprocal: MUFU approximation refined by one Newton-Raphson step,
// r' = r + r (1 - x r); within about 1 ulp of 1/x for normal x, no branch.
__device__ __forceinline__ float rcp_nr(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  const float e = fmaf(-x, r, 1.0f);
  return fmaf(r, e, r);
}

// Packed FP32 pairs: one sm_100 instruction performs two independent FP32
// operations on a register pair (per component exactly __fmaf_rn / __fmul_rn),
// halving the issue slots of paired arithmetic.
#ifndef P2Z_PACKED_F32X2
#define P2Z_PACKED_F32X2 1
#endif
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// ---------------------------------------------------------------------------
// sin / cos / versine
// ---------------------------------------------------------------------------
// Taylor series about 0 for |a| <= 0.5: sin(a) = a - a^3/3! + a^5/5! - a^7/7!
// (truncation below a^9/9! ~ 5.4e-9 |a| at |a| = 0.5) and the versine
// 1 - cos(a) = a^2/2! - a^4/4! + a^6/6! - a^8/8! (truncation below
// a^10/10! ~ 2.2e-9 of the versine at |a| = 0.5).  The coefficients are
// (-1)^n/(2n+1)! and (-1)^n/(2n)!, rounded to float.
__device__ __forceinline__ void sv_series(float a, float *s, float *v) {
  const float a2 = a * a;
  float ps = fmaf(a2, -1.9841270e-4f, 8.3333333e-3f);
  ps = fmaf(a2, ps, -1.6666667e-1f);
  *s = fmaf(a * a2, ps, a);
  float pv = fmaf(a2, 2.4801587e-5f, -1.3888889e-3f);
  pv = fmaf(a2, pv, 4.1666667e-2f);
  pv = fmaf(a2, -pv, 0.5f);
  *v = a2 * pv;
}

// tan(t + d) from tA = tan(t) and an offset d (the theta offset, which sums
// Kalman corrections: of order 1e-3 rad on well-measured tracks, up to ~0.15
// rad in one update when the initial angles are off by a few 1e-2):
//   tan(t + d) = tA + u (1 + tA^2) / (1 - tA u),
//   u = tan d = d + d^3/3 + 2 d^5/15 + 17 d^7/315 + ...
// u's series is truncated after d^7 (the next term, 62 d^9/2835, is below
// 1.2e-8 absolute for |d| <= 0.2); the quotient is exact up to a Newton-refined
// reciprocal.  The increment is formed first and added to tA last (one
// rounding at the size of the result).
__device__ __forceinline__ float tan_offset(float tA, float d) {
  const float d2 = d * d;
  float p = fmaf(d2, 5.3968254e-2f, 1.3333334e-1f);
  p = fmaf(d2, p, 3.3333334e-1f);
  const float u = fmaf(d * d2, p, d);
  const float r = u * fmaf(tA, tA, 1.f);
  return fmaf(r, rcp_nr(fmaf(-tA, u, 1.f)), tA);
}

// sin(a) and 1 - cos(a) without cancellation.
template <int SC>
__device__ __forceinline__ void sin_versine(float a, float *s, float *v) {
  if (SC == SC_FAST && fabsf(a) <= 0.5f) {
    sv_series(a, s, v);
  } else {
    float sh, ch;
    sincosf(0.5f * a, &sh, &ch);
    *s = 2.f * sh * ch;
    *v = 2.f * sh * sh;
  }
}

// sin and cos rounded once from a double evaluation: the correctly rounded
// float result except within ~1e-16 of a rounding midpoint.
__device__ __forceinline__ float sinf_cr(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float cosf_cr(float x) { return (float)cos((double)x); }

// The unit vector (c, s) = (cos t, sin t) rotated to t + d, given w = sin d
// and v = 1 - cos d: cos(t+d) = c - (c*v + s*w), sin(t+d) = s - (s*v - c*w).
// (Scalar: as packed pairs the register-pair moves cost more than they save.)
__device__ __forceinline__ void rotated(float c, float s, float w, float v, float *cn, float *sn) {
  *cn = c - fmaf(c, v, s * w);
  *sn = s - fmaf(s, v, -(c * w));
}

// Re-anchoring thresholds of the carried phi and theta offsets.  After a
// propagation |dP| <= 0.4, so the next step evaluates its phi offset (plus
// that step's Kalman correction, of order 1e-3 rad) inside the 0.5 rad range
// of sv_series; |dT| <= 0.02 at the start of a propagation keeps the theta
// offset of the next one (plus one Kalman correction) inside the range of
// tan_offset.
constexpr float kAnchorPhi = 0.4f;
constexpr float kAnchorTheta = 0.02f;
// Ranges of the offset evaluations (sv_series: |dP| <= 0.5; tan_offset:
// |dT| <= 0.2).  An offset beyond them -- after a Kalman correction of more
// than ~0.1 rad, which only a track whose covariance no longer describes it
// receives -- or a non-finite one re-anchors the direction at the track's own
// angles (sincosf, as the first layer does) before the step, so the
// polynomials are never evaluated outside their range: such a track stays
// finite wherever the angles themselves are.
constexpr float kRangePhi = 0.5f;
constexpr float kRangeTheta = 0.2f;

// ---------------------------------------------------------------------------
// Track state in registers
// ---------------------------------------------------------------------------
// T: element type of the bulk arithmetic; A: type of the x, y, phi accumulators.
// Covariance: the 15 live elements, named by (row, column); packed indices in
// comments.
// With anchored positions (AP) phi is a plain float: it is only an output (the
// propagation uses the anchored direction below), and its 40 roundings per
// track stay below 1.5e-6 relative on the 9.6M-track physics workload -- so
// the default form uses no FP64 at all.
template <typename A>
struct PhiOf {
  using type = A;
};
template <>
struct PhiOf<AP> {
  using type = float;
};

template <typename T, typename A>
struct Trk {
  A x, y;
  typename PhiOf<A>::type phi;
  T z, ipt, theta;
  // FORM_PRECISE: an anchor direction -- (cP, sP) = cos/sin of phi and
  // tT = tan(theta) at some earlier point of the track -- and dP, dT the
  // angle increments summed since then (alpha in the propagation, the Kalman
  // corrections in the update).  The direction a step uses is the anchor
  // advanced once by the offset, so the rounding of that evaluation enters
  // one step only instead of accumulating over the track; the anchor moves
  // (re-anchoring) only when an offset outgrows its series' range.
  T cP, sP, tT;
  T dP, dT;
  T c00, c10, c11;            // 0 1 2
  T c30, c31, c33;            // 6 7 9
  T c40, c41, c43, c44;       // 10 11 13 14
  T c50, c51, c53, c54, c55;  // 15 16 18 19 20
};

// Helix quantities shared by the parameter update and the Jacobian.  omc and
// omcC are 1 - cos(alpha) and 1 - cos(cosP*sin(alpha)).
//   FORM_PRECISE / FP64 fields: tanT = tan(theta), icT2 = 1/cos^2(theta),
//     dzk = deltaZ/k, kpt = k*pt, m1 = cosP*sina, m2 = sinP*sina.
//   FORM_REFERENCE fields: sinT, icosT, icosTk (the reference's own scalars).
template <typename T>
struct Helix {
  T deltaZ, pt, cosP, sinP, sina, cosa, omc, sCPs, omcC;
  T tanT, icT2, dzk, kpt, m1, m2;
  T sinT, icosT, icosTk;
};

// The Jacobian entries that act on a covariance with zero z row (reference
// :655-666 without column 2), and those of column 2 for the first layer.
template <typename T>
struct Jac {
  T a3, a4, a5;    // J(0,3) J(0,4) J(0,5)
  T a9, a10, a11;  // J(1,3) J(1,4) J(1,5)
  T a27, a29;      // J(4,3) J(4,5)
  T a2, a8, a26;   // J(0,2) J(1,2) J(4,2): first layer only
};

// ---- FORM_PRECISE -----------------------------------------------------------

// First evaluation of the carried direction of a track: the anchors at the
// input angles, zero offsets.
template <typename A>
__device__ __forceinline__ void init_direction(Trk<float, A> &s) {
  sincosf(tof(s.phi), &s.sP, &s.cP);
  float sT, cT;
  sincosf(s.theta, &sT, &cT);
  s.tT = __fdiv_rn(sT, cT);
  s.dP = 0.f;
  s.dT = 0.f;
}

// Parameter propagation (reference :627-647), with the reference's products
// regrouped around shared factors (exact in real arithmetic):
//   alpha = deltaZ*sinT*ipt*icosT/k = (deltaZ/k)*tanT*ipt,
//   x += k*(pxin*sina - pyin*(1-cosa)) = k*pt*(cosP*sina - sinP*omc),
//   y += k*(pyin*sina + pxin*(1-cosa)) = k*pt*(sinP*sina + cosP*omc).
// With SC_FAST, deltaZ/k is taken as deltaZ * (1/k): one rounding more than a
// division.  sin and 1 - cos of cosP*sina, used only by the Jacobian, come from
// the series of sv_series with no range branch: |cosP*sina| <= 1, where the
// series' truncation is below 3.3e-6 relative (sin) and 6.1e-7 (versine) --
// far inside what the covariance needs -- and below 1e-8 for |a| <= 0.5.
//
// The direction: (cosP, sinP) is the phi anchor rotated by dP, tan(theta) the
// theta anchor advanced by dT, and 1/cos^2(theta) = 1 + tan^2(theta).
// Afterwards dP advances by alpha; when that takes it past kAnchorPhi the
// anchor moves to the direction after the step (rotated from (cosP, sinP) by
// alpha with sina and omc) and dP restarts at 0.  A theta offset past
// kAnchorTheta moves the theta anchor to this step's tan(theta).  Selects, no
// branch.
template <int SC, typename A>
__device__ __forceinline__ Helix<float> propagate_params_precise(Trk<float, A> &s, float zout, float k, float ik) {
  Helix<float> h;
  if (__builtin_expect(!(fabsf(s.dP) <= kRangePhi && fabsf(s.dT) <= kRangeTheta), 0)) init_direction(s);
  h.deltaZ = zout - s.z;
  h.pt = rcp_nr(s.ipt);
  {
    // SC_FAST: |dP| <= kAnchorPhi + one Kalman correction, inside the series'
    // range, so no range branch (a branch would end the basic block and keep
    // the scheduler from overlapping this with the previous update)
    float w, v;
    if (SC == SC_FAST) sv_series(s.dP, &w, &v);
    else sin_versine<SC>(s.dP, &w, &v);
    rotated(s.cP, s.sP, w, v, &h.cosP, &h.sinP);
  }
  h.tanT = tan_offset(s.tT, s.dT);
  h.icT2 = fmaf(h.tanT, h.tanT, 1.f);
  const bool moveT = fabsf(s.dT) > kAnchorTheta;
  s.tT = moveT ? h.tanT : s.tT;
  s.dT = moveT ? 0.f : s.dT;
  h.dzk = (SC == SC_FAST) ? h.deltaZ * ik : __fdiv_rn(h.deltaZ, k);
  const float alpha = (h.dzk * h.tanT) * s.ipt;
  sin_versine<SC>(alpha, &h.sina, &h.omc);
  h.cosa = 1.f - h.omc;
  h.kpt = k * h.pt;
  h.m1 = h.cosP * h.sina;
  h.m2 = h.sinP * h.sina;
  acc_add(s.x, h.kpt * fmaf(-h.sinP, h.omc, h.m1));
  acc_add(s.y, h.kpt * fmaf(h.cosP, h.omc, h.m2));
  s.z = zout;
  acc_add(s.phi, alpha);
  if (SC == SC_FAST) sv_series(h.m1, &h.sCPs, &h.omcC);
  else sin_versine<SC>(h.m1, &h.sCPs, &h.omcC);
  const float dP = __fadd_rn(s.dP, alpha);
  const bool moveP = fabsf(dP) > kAnchorPhi;
  // (cos, sin) of phi + alpha from sin(alpha) and the versine
  const float cPn = h.cosP - fmaf(h.cosP, h.omc, h.m2);
  const float sPn = h.sinP - fmaf(h.sinP, h.omc, -h.m1);
  s.cP = moveP ? cPn : s.cP;
  s.sP = moveP ? sPn : s.sP;
  s.dP = moveP ? 0.f : dP;
  return h;
}

// A Kalman correction of phi and theta, added to the offsets from the
// anchors (the output angles accumulate it separately).
template <typename A>
__device__ __forceinline__ void turn_direction(Trk<float, A> &s, float dphi, float dth) {
  s.dP = __fadd_rn(s.dP, dphi);
  s.dT = __fadd_rn(s.dT, dth);
}

// The Jacobian entries (reference :655-666) with the shared factors taken out
// (exact in real arithmetic; fewer products):
//   B = 1 - sinP*sC,  D = cosP^2*sC + sinP,  u = cosP*dZ*cosa*B,  v = dZ*cosa*D,
//   J03 = u*tanT*pt - k*pt^2*(cosP*sina - sinP*omcC)   J05 = u/cosT^2
//   J13 = v*tanT*pt - k*pt^2*(sinP*sina + cosP*omcC)   J15 = v/cosT^2
//   J04 = -k*pt*(sinP*sina*B + cosP*omcC)               J14 = k*pt*(cosP*sina*B - sinP*omcC)
//   J43 = (dZ/k)*tanT                                   J45 = (dZ/k)*ipt/cosT^2
// and, for the first layer, J02 = -cosP*tanT*cosa*B, J12 = cosa*tanT*(cosP^2*sC - sinP),
// J42 = -ipt*tanT/k.
template <typename T, bool GENERAL = false>
__device__ __forceinline__ Jac<T> jacobian_precise(const Helix<T> &h, T k, T ipt) {
  Jac<T> J;
  const T cosP = h.cosP, sinP = h.sinP;
  const T dzc = h.deltaZ * h.cosa;
  const T B = T(1) - sinP * h.sCPs;
  const T cc = cosP * cosP * h.sCPs;
  const T D = cc + sinP;
  const T stp = h.tanT * h.pt;
  const T kpt = h.kpt;
  const T kpt2 = kpt * h.pt;
  const T m1 = h.m1, m2 = h.m2;
  const T n1 = cosP * h.omcC, n2 = sinP * h.omcC;
  const T u = cosP * dzc * B;
  const T v = dzc * D;
  J.a3 = u * stp - kpt2 * (m1 - n2);
  J.a5 = u * h.icT2;
  J.a9 = v * stp - kpt2 * (m2 + n1);
  J.a11 = v * h.icT2;
  J.a4 = -kpt * (m2 * B + n1);
  J.a10 = kpt * (m1 * B - n2);
  J.a27 = h.dzk * h.tanT;
  J.a29 = (h.dzk * ipt) * h.icT2;
  if constexpr (GENERAL) {
    J.a2 = -(cosP * h.tanT) * (h.cosa * B);
    J.a8 = h.cosa * h.tanT * (cc - sinP);
    J.a26 = -(ipt * h.tanT) / k;
  } else {
    J.a2 = J.a8 = J.a26 = T(0);
  }
  return J;
}

// ---- FORM_REFERENCE ---------------------------------------------------------

// The reference's propagateToZ scalars with its types: the double literals
// promote the marked sub-expressions to double; sin/cos correctly rounded
// (the reference calls the C library's sinf/cosf).
__device__ __forceinline__ Helix<float> propagate_params_ref(Trk<float, float> &s, float zout, float k) {
  Helix<float> h;
  h.deltaZ = zout - s.z;
  h.pt = 1. / s.ipt;
  h.cosP = cosf_cr(s.phi);
  h.sinP = sinf_cr(s.phi);
  const float cosT = cosf_cr(s.theta);
  h.sinT = sinf_cr(s.theta);
  const float pxin = h.cosP * h.pt;
  const float pyin = h.sinP * h.pt;
  h.icosT = 1.0 / cosT;
  h.icosTk = h.icosT / k;
  const float alpha = h.deltaZ * h.sinT * s.ipt * h.icosTk;
  h.sina = sinf_cr(alpha);
  h.cosa = cosf_cr(alpha);
  s.x = s.x + k * (pxin * h.sina - pyin * (1. - h.cosa));
  s.y = s.y + k * (pyin * h.sina + pxin * (1. - h.cosa));
  s.z = zout;
  s.phi = s.phi + alpha;
  h.sCPs = sinf_cr(h.cosP * h.sina);
  const float cC = cosf_cr(h.cosP * h.sina);
  h.omcC = cC;  // FORM_REFERENCE keeps cos(cosP*sina) itself here
  h.omc = 0.f;
  return h;
}

__device__ __forceinline__ Jac<float> jacobian_ref(const Helix<float> &h, float k, float ipt) {
  Jac<float> J;
  const float cosP = h.cosP, sinP = h.sinP, sinT = h.sinT, cosa = h.cosa, sina = h.sina;
  const float sCosPsina = h.sCPs, cCosPsina = h.omcC;
  const float deltaZ = h.deltaZ, icosT = h.icosT, icosTk = h.icosTk, pt = h.pt;
  J.a3 = cosP * sinT * deltaZ * cosa * (1. - sinP * sCosPsina) * (icosT * pt) -
         k * (cosP * sina - sinP * (1. - cCosPsina)) * (pt * pt);
  J.a4 = (k * pt) * (-sinP * sina + sinP * sinP * sina * sCosPsina - cosP * (1. - cCosPsina));
  J.a5 = cosP * deltaZ * cosa * (1. - sinP * sCosPsina) * (icosT * icosT);
  J.a9 = sinT * deltaZ * cosa * (cosP * cosP * sCosPsina + sinP) * (icosT * pt) -
         k * (sinP * sina + cosP * (1. - cCosPsina)) * (pt * pt);
  J.a10 = (k * pt) * (-sinP * (1. - cCosPsina) - sinP * cosP * sina * sCosPsina + cosP * sina);
  J.a11 = deltaZ * cosa * (cosP * cosP * sCosPsina + sinP) * (icosT * icosT);
  J.a27 = sinT * deltaZ * (icosTk);
  J.a29 = ipt * deltaZ * (icosT * icosTk);
  // column 2 (first layer): reference :655, :659, :663
  J.a2 = cosP * sinT * (sinP * cosa * sCosPsina - cosa) * icosT;
  J.a8 = cosa * sinT * (cosP * cosP * sCosPsina - sinP) * icosT;
  J.a26 = -ipt * sinT * (icosTk);
  return J;
}

// ---- FP64 everything --------------------------------------------------------

__device__ __forceinline__ Helix<double> propagate_params_f64(Trk<double, double> &s, double zout, double k) {
  Helix<double> h;
  h.deltaZ = zout - s.z;
  h.pt = 1.0 / s.ipt;
  double cosT, sinT;
  sincos(s.phi, &h.sinP, &h.cosP);
  sincos(s.theta, &sinT, &cosT);
  h.tanT = sinT / cosT;
  h.icT2 = 1.0 / (cosT * cosT);
  h.dzk = h.deltaZ / k;
  const double alpha = h.dzk * h.tanT * s.ipt;
  sincos(alpha, &h.sina, &h.cosa);
  h.omc = 1.0 - h.cosa;
  h.kpt = k * h.pt;
  h.m1 = h.cosP * h.sina;
  h.m2 = h.sinP * h.sina;
  s.x += h.kpt * (h.m1 - h.sinP * h.omc);
  s.y += h.kpt * (h.m2 + h.cosP * h.omc);
  s.z = zout;
  s.phi += alpha;
  double cC;
  sincos(h.m1, &h.sCPs, &cC);
  h.omcC = 1.0 - cC;
  return h;
}

// ---------------------------------------------------------------------------
// Covariance propagation C' = J C J^T
// ---------------------------------------------------------------------------

// Reduced form: C with zero z row/column.  Sums in the reference's order
// (t<n>: element n of T = J C row-major; c<n>: packed output n).
template <typename T, typename A>
__device__ __forceinline__ void propagate_cov_reduced(Trk<T, A> &s, const Jac<T> &J) {
  // T = J C, rows 0, 1 and 4 (rows 3 and 5 are C's, row 2 is zero)
  const T t0 = s.c00 + J.a3 * s.c30 + J.a4 * s.c40 + J.a5 * s.c50;
  const T t3 = s.c30 + J.a3 * s.c33 + J.a4 * s.c43 + J.a5 * s.c53;
  const T t4 = s.c40 + J.a3 * s.c43 + J.a4 * s.c44 + J.a5 * s.c54;
  const T t5 = s.c50 + J.a3 * s.c53 + J.a4 * s.c54 + J.a5 * s.c55;
  const T t6 = s.c10 + J.a9 * s.c30 + J.a10 * s.c40 + J.a11 * s.c50;
  const T t7 = s.c11 + J.a9 * s.c31 + J.a10 * s.c41 + J.a11 * s.c51;
  const T t9 = s.c31 + J.a9 * s.c33 + J.a10 * s.c43 + J.a11 * s.c53;
  const T t10 = s.c41 + J.a9 * s.c43 + J.a10 * s.c44 + J.a11 * s.c54;
  const T t11 = s.c51 + J.a9 * s.c53 + J.a10 * s.c54 + J.a11 * s.c55;
  const T t24 = J.a27 * s.c30 + s.c40 + J.a29 * s.c50;
  const T t25 = J.a27 * s.c31 + s.c41 + J.a29 * s.c51;
  const T t27 = J.a27 * s.c33 + s.c43 + J.a29 * s.c53;
  const T t28 = J.a27 * s.c43 + s.c44 + J.a29 * s.c54;
  const T t29 = J.a27 * s.c53 + s.c54 + J.a29 * s.c55;
  const T t18 = s.c30, t19 = s.c31, t21 = s.c33, t22 = s.c43, t23 = s.c53;
  const T t30 = s.c50, t31 = s.c51, t33 = s.c53, t34 = s.c54, t35 = s.c55;
  // C' = T J^T
  s.c00 = t0 + t3 * J.a3 + t4 * J.a4 + t5 * J.a5;        // c0
  s.c10 = t6 + t9 * J.a3 + t10 * J.a4 + t11 * J.a5;      // c1
  s.c11 = t7 + t9 * J.a9 + t10 * J.a10 + t11 * J.a11;    // c2
  s.c30 = t18 + t21 * J.a3 + t22 * J.a4 + t23 * J.a5;    // c6
  s.c31 = t19 + t21 * J.a9 + t22 * J.a10 + t23 * J.a11;  // c7
  s.c33 = t21;                                           // c9
  s.c40 = t24 + t27 * J.a3 + t28 * J.a4 + t29 * J.a5;    // c10
  s.c41 = t25 + t27 * J.a9 + t28 * J.a10 + t29 * J.a11;  // c11
  s.c43 = t27;                                           // c13
  s.c44 = t27 * J.a27 + t28 + t29 * J.a29;               // c14
  s.c50 = t30 + t33 * J.a3 + t34 * J.a4 + t35 * J.a5;    // c15
  s.c51 = t31 + t33 * J.a9 + t34 * J.a10 + t35 * J.a11;  // c16
  s.c53 = t33;                                           // c18
  s.c54 = t33 * J.a27 + t34 + t35 * J.a29;               // c19
  s.c55 = t35;                                           // c20
}

// The same reduced form with the row-0/row-1 Jacobian pairs (a3, a9),
// (a4, a10), (a5, a11) and the covariance pairs (c00, c10), (c30, c31),
// (c40, c41), (c50, c51) in packed FP32 pairs.  Each component is the scalar
// form's chain of fused multiply-adds in the same order, so the results are
// identical bit for bit; the pairs only halve the instructions.  Identities
// used: the new (c30, c31) is T's (t3, t9), the new (c50, c51) is (t5, t11),
// the new c54 is t29 and the new c43 is t27.
template <typename A>
__device__ __forceinline__ void propagate_cov_reduced_packed(Trk<float, A> &s, const Jac<float> &J) {
  const float2 A3 = make_float2(J.a3, J.a9), A4 = make_float2(J.a4, J.a10), A5 = make_float2(J.a5, J.a11);
  const float2 P0 = make_float2(s.c00, s.c10), P3 = make_float2(s.c30, s.c31);
  const float2 P4 = make_float2(s.c40, s.c41), P5 = make_float2(s.c50, s.c51);
  // T = J C: rows 0 and 1 in pairs (columns 0, 3, 4, 5), row 1 column 1, row 4
  const float2 T0 = fma2(A5, bc2(s.c50), fma2(A4, bc2(s.c40), fma2(A3, bc2(s.c30), P0)));  // (t0, t6)
  const float2 T3 = fma2(A5, bc2(s.c53), fma2(A4, bc2(s.c43), fma2(A3, bc2(s.c33), P3)));  // (t3, t9)
  const float2 T4 = fma2(A5, bc2(s.c54), fma2(A4, bc2(s.c44), fma2(A3, bc2(s.c43), P4)));  // (t4, t10)
  const float2 T5 = fma2(A5, bc2(s.c55), fma2(A4, bc2(s.c54), fma2(A3, bc2(s.c53), P5)));  // (t5, t11)
  const float t7 = s.c11 + J.a9 * s.c31 + J.a10 * s.c41 + J.a11 * s.c51;
  const float2 T24 = fma2(bc2(J.a29), P5, fma2(bc2(J.a27), P3, P4));                        // (t24, t25)
  const float t27 = J.a27 * s.c33 + s.c43 + J.a29 * s.c53;
  const float t28 = J.a27 * s.c43 + s.c44 + J.a29 * s.c54;
  const float t29 = J.a27 * s.c53 + s.c54 + J.a29 * s.c55;
  // C' = T J^T
  const float2 N0 = fma2(T5, bc2(J.a5), fma2(T4, bc2(J.a4), fma2(T3, bc2(J.a3), T0)));      // (c00, c10)
  const float c11 = t7 + T3.y * J.a9 + T4.y * J.a10 + T5.y * J.a11;
  const float2 N4 = fma2(A5, bc2(t29), fma2(A4, bc2(t28), fma2(A3, bc2(t27), T24)));       // (c40, c41)
  s.c00 = N0.x; s.c10 = N0.y;
  s.c11 = c11;
  s.c30 = T3.x; s.c31 = T3.y;
  s.c40 = N4.x; s.c41 = N4.y;
  s.c43 = t27;
  s.c44 = t27 * J.a27 + t28 + t29 * J.a29;
  s.c50 = T5.x; s.c51 = T5.y;
  s.c54 = t29;
}

// Two threads per track: lanes 2i (j = 0) and 2i+1 (j = 1) of a warp hold the
// same track.  Each lane evaluates component j of every pair of the packed
// form above -- row j of T = J C and of the propagated measured columns -- as
// one scalar fused multiply-add per packed one, in the same order, and takes
// the other component from its partner lane with one shuffle per pair, so
// both lanes end with the packed form's results bit for bit.  The scalar
// chains (t7, t27..t29, c44) are evaluated by both lanes; c11 needs row 1 of
// T, which lane 1 holds, and comes from there.  pm names the two lanes.
__device__ __forceinline__ void pair_join(float own, bool j, unsigned pm, float &x, float &y) {
  const float other = __shfl_xor_sync(pm, own, 1);
  x = j ? other : own;
  y = j ? own : other;
}

template <typename A>
__device__ __forceinline__ void propagate_cov_reduced_pair(Trk<float, A> &s, const Jac<float> &J, bool j,
                                                           unsigned pm) {
  const float A3 = j ? J.a9 : J.a3, A4 = j ? J.a10 : J.a4, A5 = j ? J.a11 : J.a5;
  const float P0 = j ? s.c10 : s.c00, P3 = j ? s.c31 : s.c30, P4 = j ? s.c41 : s.c40, P5 = j ? s.c51 : s.c50;
  const float T0 = fmaf(A5, s.c50, fmaf(A4, s.c40, fmaf(A3, s.c30, P0)));  // t0 | t6
  const float T3 = fmaf(A5, s.c53, fmaf(A4, s.c43, fmaf(A3, s.c33, P3)));  // t3 | t9
  const float T4 = fmaf(A5, s.c54, fmaf(A4, s.c44, fmaf(A3, s.c43, P4)));  // t4 | t10
  const float T5 = fmaf(A5, s.c55, fmaf(A4, s.c54, fmaf(A3, s.c53, P5)));  // t5 | t11
  const float t7 = s.c11 + J.a9 * s.c31 + J.a10 * s.c41 + J.a11 * s.c51;
  const float T24 = fmaf(J.a29, P5, fmaf(J.a27, P3, P4));                  // t24 | t25
  const float t27 = J.a27 * s.c33 + s.c43 + J.a29 * s.c53;
  const float t28 = J.a27 * s.c43 + s.c44 + J.a29 * s.c54;
  const float t29 = J.a27 * s.c53 + s.c54 + J.a29 * s.c55;
  const float N0 = fmaf(T5, J.a5, fmaf(T4, J.a4, fmaf(T3, J.a3, T0)));    // c00 | c10
  const float c11 = t7 + T3 * J.a9 + T4 * J.a10 + T5 * J.a11;              // the result on lane 1
  const float N4 = fmaf(A5, t29, fmaf(A4, t28, fmaf(A3, t27, T24)));       // c40 | c41
  pair_join(N0, j, pm, s.c00, s.c10);
  pair_join(T3, j, pm, s.c30, s.c31);
  pair_join(N4, j, pm, s.c40, s.c41);
  pair_join(T5, j, pm, s.c50, s.c51);
  const float c11o = __shfl_xor_sync(pm, c11, 1);
  s.c11 = j ? c11 : c11o;
  s.c43 = t27;
  s.c44 = t27 * J.a27 + t28 + t29 * J.a29;
  s.c54 = t29;
}

// General form on the full 21-element input covariance b[] (the first
// propagation of a track), including the Jacobian's z column a2 = J(0,2),
// a8 = J(1,2), a26 = J(4,2) (reference :655, :659, :663), which the Jacobian
// functions fill for the first layer.
template <typename T, typename A>
__device__ __forceinline__ void propagate_cov_general(Trk<T, A> &s, const T *b, const Helix<T> &h,
                                                      const Jac<T> &J) {
  (void)h;
  const T a2 = J.a2, a8 = J.a8, a26 = J.a26;
  const T a3 = J.a3, a4 = J.a4, a5 = J.a5, a9 = J.a9, a10 = J.a10, a11 = J.a11, a27 = J.a27, a29 = J.a29;
  const T t0 = b[0] + a2 * b[3] + a3 * b[6] + a4 * b[10] + a5 * b[15];
  const T t2 = b[3] + a2 * b[5] + a3 * b[8] + a4 * b[12] + a5 * b[17];
  const T t3 = b[6] + a2 * b[8] + a3 * b[9] + a4 * b[13] + a5 * b[18];
  const T t4 = b[10] + a2 * b[12] + a3 * b[13] + a4 * b[14] + a5 * b[19];
  const T t5 = b[15] + a2 * b[17] + a3 * b[18] + a4 * b[19] + a5 * b[20];
  const T t6 = b[1] + a8 * b[3] + a9 * b[6] + a10 * b[10] + a11 * b[15];
  const T t7 = b[2] + a8 * b[4] + a9 * b[7] + a10 * b[11] + a11 * b[16];
  const T t8 = b[4] + a8 * b[5] + a9 * b[8] + a10 * b[12] + a11 * b[17];
  const T t9 = b[7] + a8 * b[8] + a9 * b[9] + a10 * b[13] + a11 * b[18];
  const T t10 = b[11] + a8 * b[12] + a9 * b[13] + a10 * b[14] + a11 * b[19];
  const T t11 = b[16] + a8 * b[17] + a9 * b[18] + a10 * b[19] + a11 * b[20];
  const T t18 = b[6], t19 = b[7], t20 = b[8], t21 = b[9], t22 = b[13], t23 = b[18];
  const T t24 = a26 * b[3] + a27 * b[6] + b[10] + a29 * b[15];
  const T t25 = a26 * b[4] + a27 * b[7] + b[11] + a29 * b[16];
  const T t26 = a26 * b[5] + a27 * b[8] + b[12] + a29 * b[17];
  const T t27 = a26 * b[8] + a27 * b[9] + b[13] + a29 * b[18];
  const T t28 = a26 * b[12] + a27 * b[13] + b[14] + a29 * b[19];
  const T t29 = a26 * b[17] + a27 * b[18] + b[19] + a29 * b[20];
  const T t30 = b[15], t31 = b[16], t32 = b[17], t33 = b[18], t34 = b[19], t35 = b[20];
  s.c00 = t0 + t2 * a2 + t3 * a3 + t4 * a4 + t5 * a5;
  s.c10 = t6 + t8 * a2 + t9 * a3 + t10 * a4 + t11 * a5;
  s.c11 = t7 + t8 * a8 + t9 * a9 + t10 * a10 + t11 * a11;
  s.c30 = t18 + t20 * a2 + t21 * a3 + t22 * a4 + t23 * a5;
  s.c31 = t19 + t20 * a8 + t21 * a9 + t22 * a10 + t23 * a11;
  s.c33 = t21;
  s.c40 = t24 + t26 * a2 + t27 * a3 + t28 * a4 + t29 * a5;
  s.c41 = t25 + t26 * a8 + t27 * a9 + t28 * a10 + t29 * a11;
  s.c43 = t27;
  s.c44 = t26 * a26 + t27 * a27 + t28 + t29 * a29;
  s.c50 = t30 + t32 * a2 + t33 * a3 + t34 * a4 + t35 * a5;
  s.c51 = t31 + t32 * a8 + t33 * a9 + t34 * a10 + t35 * a11;
  s.c53 = t33;
  s.c54 = t32 * a26 + t33 * a27 + t34 + t35 * a29;
  s.c55 = t35;
}

// ---------------------------------------------------------------------------
// Measurement updates
// ---------------------------------------------------------------------------

// Compensated a*d - b*c (Kahan's algorithm with one FMA error term).
__device__ __forceinline__ float det2_comp(float a, float b, float c, float d) {
  const float w = b * c;
  const float e = fmaf(-b, c, w);  // exact: w - b*c
  const float f = fmaf(a, d, -w);
  return f + e;
}

// Apply the 2-D (x,y) gain: K(i,:) = (C(i,0), C(i,1)) * Rinv for the live rows
// (the z row is zero), the parameter update with the residual (hx - x,
// hy - y), and the covariance update, C - K H C (reference :534-617).
// FORM_PRECISE, FP32 with packed pairs: the gain rows (K_i0, K_i1) as
// c_i0 (i00, i01) + c_i1 (i01, i11); rows x, y, ipt, phi, theta of C's
// measured columns as pairs B_i = (c_i0, c_i1); A = the measured 2x2 block.
//
// C - K H C subtracts nearly equal numbers where the update shrinks C by a
// large factor in some direction, and there a gain rounded by a few ulp (its
// relative error grows with R's condition number) costs many digits: on a
// track whose first hit is 200x more precise than the track in one
// direction, C then stops describing the track, and the gains of later
// layers with it.  That happens at a track's first update, where its prior
// covariance meets a measurement.  There, when g = det(V)/det(R) =
// det(I - K H) is at or below kJosephShrink (a shrink of 100 or more in area),
// the update takes the Joseph form (I-KH) C (I-KH)^T + K V K^T instead,
// evaluated as C'' = P - E K^T with P = C - K H C and E = P H^T - K V, the
// residual of the gain equation, which cancels K's rounding errors to first
// order.  K V is formed from error-free products (p = K0*v, e = fma(K0, v,
// -p)): with an elongated V the two products cancel, and a rounded first
// product would leave an error of eps*|K||V| in E.  The reference's own
// known-answer hits are such a V (eigenvalues 1e6 apart) and their first
// updates shrink little in area (g > 0.01); there C - K H C is the more
// accurate evaluation (1e-4 against the Joseph form's 7.5e-4 in q/pT), as it
// is everywhere after a track's first update, where C is already a fit of
// the track.  The test is per track, so a track's result does not depend on
// its neighbours.  Measured on one B200 (1000 x 9600 physics sample, flat
// launch; without the first-layer test 1.770 ms): the test 1.786 ms, the
// Joseph form on every first layer unconditionally 1.841 ms, on every layer
// 1.961 ms, with the same results on the single-seed, physics and sweep
// samples.
constexpr float kJosephShrink = 0.01f;

// Joseph form of a track's first update (see above).
template <typename A>
__device__ __forceinline__ void update_v2_apply_joseph(Trk<float, A> &s, float i00, float i01, float i11, float hx,
                                                       float hy, float v00, float v01, float v11) {
  const float2 I0 = make_float2(i00, i01), I1 = make_float2(i01, i11);
  const float2 A0 = make_float2(s.c00, s.c10), A1 = make_float2(s.c10, s.c11);
  const float2 B3 = make_float2(s.c30, s.c31), B4 = make_float2(s.c40, s.c41), B5 = make_float2(s.c50, s.c51);
  const float2 Kx = fma2(bc2(s.c10), I1, mul2(bc2(s.c00), I0));  // (K0, K1)
  const float2 Ky = fma2(bc2(s.c11), I1, mul2(bc2(s.c10), I0));  // (K2, K3)
  const float2 Ki = fma2(bc2(B3.y), I1, mul2(bc2(B3.x), I0));    // (K6, K7)
  const float2 Kp = fma2(bc2(B4.y), I1, mul2(bc2(B4.x), I0));    // (K8, K9)
  const float2 Kt = fma2(bc2(B5.y), I1, mul2(bc2(B5.x), I0));    // (K10, K11)
  const float res0 = acc_res(hx, s.x), res1 = acc_res(hy, s.y);
  acc_update(s.x, hx, res0, Kx.x * res0 + Kx.y * res1);
  acc_update(s.y, hy, res1, Ky.x * res0 + Ky.y * res1);
  const float dphi = Kp.x * res0 + Kp.y * res1;
  const float dth = Kt.x * res0 + Kt.y * res1;
  acc_add(s.phi, dphi);
  s.theta = __fadd_rn(s.theta, dth);
  turn_direction(s, dphi, dth);
  s.ipt = s.ipt + Ki.x * res0 + Ki.y * res1;
  // P = C - K H C on the measured columns of every live row
  const float2 Px = fma2(bc2(-Kx.y), A1, fma2(bc2(-Kx.x), A0, A0));
  const float2 Py = fma2(bc2(-Ky.y), A1, fma2(bc2(-Ky.x), A0, A1));
  const float2 Pi = fma2(bc2(-Ki.y), A1, fma2(bc2(-Ki.x), A0, B3));
  const float2 Pp = fma2(bc2(-Kp.y), A1, fma2(bc2(-Kp.x), A0, B4));
  const float2 Pt = fma2(bc2(-Kt.y), A1, fma2(bc2(-Kt.x), A0, B5));
  // E_i = P_i - K_i V (K V from error-free products), then
  // C''(i, m) = P(i, m) - E_i . K_m for the measured columns and
  // C''(a, b) = C(a, b) - K_a . B_b - E_a . K_b on the unmeasured block.
  const float2 V0 = make_float2(v00, v01), V1 = make_float2(v01, v11);
  const float2 Kc0 = make_float2(Kx.x, Ky.x), Kc1 = make_float2(Kx.y, Ky.y);
  auto resid = [&](const float2 P, const float2 K) {
    const float2 p = mul2(bc2(-K.x), V0);
    const float2 e = fma2(bc2(-K.x), V0, make_float2(-p.x, -p.y));  // exact: -K0 V0 - p
    return __fadd2_rn(__fadd2_rn(fma2(bc2(-K.y), V1, p), e), P);
  };
  const float2 Ex = resid(Px, Kx), Ey = resid(Py, Ky), Ei = resid(Pi, Ki), Ep = resid(Pp, Kp), Et = resid(Pt, Kt);
  const float2 Nx = fma2(bc2(-Ex.y), Kc1, fma2(bc2(-Ex.x), Kc0, Px));
  const float2 Ny = fma2(bc2(-Ey.y), Kc1, fma2(bc2(-Ey.x), Kc0, Py));
  const float2 Ni = fma2(bc2(-Ei.y), Kc1, fma2(bc2(-Ei.x), Kc0, Pi));
  const float2 Np = fma2(bc2(-Ep.y), Kc1, fma2(bc2(-Ep.x), Kc0, Pp));
  const float2 Nt = fma2(bc2(-Et.y), Kc1, fma2(bc2(-Et.x), Kc0, Pt));
  s.c33 = fmaf(-Ei.y, Ki.y, fmaf(-Ei.x, Ki.x, fmaf(-Ki.y, B3.y, fmaf(-Ki.x, B3.x, s.c33))));
  s.c43 = fmaf(-Ep.y, Ki.y, fmaf(-Ep.x, Ki.x, fmaf(-Kp.y, B3.y, fmaf(-Kp.x, B3.x, s.c43))));
  s.c44 = fmaf(-Ep.y, Kp.y, fmaf(-Ep.x, Kp.x, fmaf(-Kp.y, B4.y, fmaf(-Kp.x, B4.x, s.c44))));
  s.c53 = fmaf(-Et.y, Ki.y, fmaf(-Et.x, Ki.x, fmaf(-Kt.y, B3.y, fmaf(-Kt.x, B3.x, s.c53))));
  s.c54 = fmaf(-Et.y, Kp.y, fmaf(-Et.x, Kp.x, fmaf(-Kt.y, B4.y, fmaf(-Kt.x, B4.x, s.c54))));
  s.c55 = fmaf(-Et.y, Kt.y, fmaf(-Et.x, Kt.x, fmaf(-Kt.y, B5.y, fmaf(-Kt.x, B5.x, s.c55))));
  s.c00 = Nx.x;
  s.c10 = Ny.x; s.c11 = Ny.y;
  s.c30 = Ni.x; s.c31 = Ni.y;
  s.c40 = Np.x; s.c41 = Np.y;
  s.c50 = Nt.x; s.c51 = Nt.y;
}

// Every later update: the reference's C - K H C with the column-0/1 pairs of
// rows y, ipt, phi, theta updated together:
//   (c_i0, c_i1)' = (c_i0, c_i1) - K_i0 (c00, c10) - K_i1 (c10, c11).
template <bool FIRST, typename A>
__device__ __forceinline__ void update_v2_apply_packed(Trk<float, A> &s, float r00, float r01, float r11, float hx,
                                                       float hy, float v00, float v01, float v11) {
  if constexpr (FIRST) {
    // shrink test: det(I - K H) = det(V) / det(R), and r00 r11 - r01^2 = 1/det(R)
    const float g = fmaf(v00, v11, -(v01 * v01)) * fmaf(r00, r11, -(r01 * r01));
    if (!(g > kJosephShrink)) {
      update_v2_apply_joseph(s, r00, r01, r11, hx, hy, v00, v01, v11);
      return;
    }
  }
  (void)v00;
  (void)v01;
  (void)v11;
  const float2 R0 = make_float2(r00, r01), R1 = make_float2(r01, r11);
  const float2 Kx = fma2(bc2(s.c10), R1, mul2(bc2(s.c00), R0));  // (K0, K1)
  const float2 Ky = fma2(bc2(s.c11), R1, mul2(bc2(s.c10), R0));  // (K2, K3)
  const float2 Ki = fma2(bc2(s.c31), R1, mul2(bc2(s.c30), R0));  // (K6, K7)
  const float2 Kp = fma2(bc2(s.c41), R1, mul2(bc2(s.c40), R0));  // (K8, K9)
  const float2 Kt = fma2(bc2(s.c51), R1, mul2(bc2(s.c50), R0));  // (K10, K11)
  const float res0 = acc_res(hx, s.x), res1 = acc_res(hy, s.y);
  acc_update(s.x, hx, res0, Kx.x * res0 + Kx.y * res1);
  acc_update(s.y, hy, res1, Ky.x * res0 + Ky.y * res1);
  const float dphi = Kp.x * res0 + Kp.y * res1;
  const float dth = Kt.x * res0 + Kt.y * res1;
  acc_add(s.phi, dphi);
  s.theta = __fadd_rn(s.theta, dth);
  turn_direction(s, dphi, dth);
  s.ipt = s.ipt + Ki.x * res0 + Ki.y * res1;
  const float2 P0 = make_float2(s.c00, s.c10), Q = make_float2(s.c10, s.c11);
  const float c30 = s.c30, c31 = s.c31, c40 = s.c40, c41 = s.c41, c50 = s.c50, c51 = s.c51;
  s.c00 = fmaf(-Kx.y, s.c10, fmaf(-Kx.x, s.c00, s.c00));
  const float2 Ny = fma2(bc2(-Ky.y), Q, fma2(bc2(-Ky.x), P0, Q));
  const float2 Ni = fma2(bc2(-Ki.y), Q, fma2(bc2(-Ki.x), P0, make_float2(c30, c31)));
  const float2 Np = fma2(bc2(-Kp.y), Q, fma2(bc2(-Kp.x), P0, make_float2(c40, c41)));
  const float2 Nt = fma2(bc2(-Kt.y), Q, fma2(bc2(-Kt.x), P0, make_float2(c50, c51)));
  s.c10 = Ny.x; s.c11 = Ny.y;
  s.c30 = Ni.x; s.c31 = Ni.y;
  s.c40 = Np.x; s.c41 = Np.y;
  s.c50 = Nt.x; s.c51 = Nt.y;
  s.c33 = fmaf(-Ki.y, c31, fmaf(-Ki.x, c30, s.c33));
  s.c43 = fmaf(-Kp.y, c31, fmaf(-Kp.x, c30, s.c43));
  s.c44 = fmaf(-Kp.y, c41, fmaf(-Kp.x, c40, s.c44));
  s.c53 = fmaf(-Kt.y, c31, fmaf(-Kt.x, c30, s.c53));
  s.c54 = fmaf(-Kt.y, c41, fmaf(-Kt.x, c40, s.c54));
  s.c55 = fmaf(-Kt.y, c51, fmaf(-Kt.x, c50, s.c55));
}

// The generic form (FP64 kernel, reference rounding, unpacked FP32): the
// reference's C - K (H C).  v (the hit covariance) is used by the packed FP32
// form only.
template <typename T, typename A, int FORM, bool FIRST = false>
__device__ __forceinline__ void update_v2_apply(Trk<T, A> &s, T r00, T r01, T r11, T hx, T hy, const T (&v)[3]) {
  if constexpr (P2Z_PACKED_F32X2 && FORM == FORM_PRECISE && std::is_same<T, float>::value) {
    update_v2_apply_packed<FIRST>(s, r00, r01, r11, hx, hy, v[0], v[1], v[2]);
    return;
  }
  (void)v;
  const T K0 = s.c00 * r00 + s.c10 * r01, K1 = s.c00 * r01 + s.c10 * r11;
  const T K2 = s.c10 * r00 + s.c11 * r01, K3 = s.c10 * r01 + s.c11 * r11;
  const T K6 = s.c30 * r00 + s.c31 * r01, K7 = s.c30 * r01 + s.c31 * r11;
  const T K8 = s.c40 * r00 + s.c41 * r01, K9 = s.c40 * r01 + s.c41 * r11;
  const T K10 = s.c50 * r00 + s.c51 * r01, K11 = s.c50 * r01 + s.c51 * r11;
  const T res0 = acc_res(hx, s.x), res1 = acc_res(hy, s.y);
  if constexpr (FORM == FORM_REFERENCE) {
    // reference order: p + K0*r0 + K1*r1, left to right
    acc_set(s.x, tof(s.x) + K0 * res0 + K1 * res1);
    acc_set(s.y, tof(s.y) + K2 * res0 + K3 * res1);
    acc_set(s.phi, tof(s.phi) + K8 * res0 + K9 * res1);
    s.theta = s.theta + K10 * res0 + K11 * res1;
  } else if constexpr (std::is_same<T, float>::value) {
    acc_update(s.x, hx, res0, K0 * res0 + K1 * res1);
    acc_update(s.y, hy, res1, K2 * res0 + K3 * res1);
    const float dphi = K8 * res0 + K9 * res1;
    const float dth = K10 * res0 + K11 * res1;
    acc_add(s.phi, dphi);
    s.theta = __fadd_rn(s.theta, dth);
    turn_direction(s, dphi, dth);
  } else {
    acc_add(s.x, K0 * res0 + K1 * res1);
    acc_add(s.y, K2 * res0 + K3 * res1);
    acc_add(s.phi, K8 * res0 + K9 * res1);
    s.theta = s.theta + K10 * res0 + K11 * res1;
  }
  s.ipt = s.ipt + K6 * res0 + K7 * res1;
  if constexpr (FORM == FORM_PRECISE && std::is_same<T, float>::value) {
    // C - K (H C), each element as two fused multiply-adds: C - K_i0 C_0j - K_i1 C_1j
    const T c00 = s.c00, c10 = s.c10, c11 = s.c11, c30 = s.c30, c31 = s.c31, c40 = s.c40, c41 = s.c41;
    const T c50 = s.c50, c51 = s.c51;
    s.c00 = fmaf(-K1, c10, fmaf(-K0, c00, c00));
    s.c10 = fmaf(-K3, c10, fmaf(-K2, c00, c10));
    s.c11 = fmaf(-K3, c11, fmaf(-K2, c10, c11));
    s.c30 = fmaf(-K7, c10, fmaf(-K6, c00, c30));
    s.c31 = fmaf(-K7, c11, fmaf(-K6, c10, c31));
    s.c33 = fmaf(-K7, c31, fmaf(-K6, c30, s.c33));
    s.c40 = fmaf(-K9, c10, fmaf(-K8, c00, c40));
    s.c41 = fmaf(-K9, c11, fmaf(-K8, c10, c41));
    s.c43 = fmaf(-K9, c31, fmaf(-K8, c30, s.c43));
    s.c44 = fmaf(-K9, c41, fmaf(-K8, c40, s.c44));
    s.c50 = fmaf(-K11, c10, fmaf(-K10, c00, c50));
    s.c51 = fmaf(-K11, c11, fmaf(-K10, c10, c51));
    s.c53 = fmaf(-K11, c31, fmaf(-K10, c30, s.c53));
    s.c54 = fmaf(-K11, c41, fmaf(-K10, c40, s.c54));
    s.c55 = fmaf(-K11, c51, fmaf(-K10, c50, s.c55));
  } else {
    const T e0 = K0 * s.c00 + K1 * s.c10;
    const T e1 = K2 * s.c00 + K3 * s.c10;
    const T e2 = K2 * s.c10 + K3 * s.c11;
    const T e6 = K6 * s.c00 + K7 * s.c10;
    const T e7 = K6 * s.c10 + K7 * s.c11;
    const T e9 = K6 * s.c30 + K7 * s.c31;
    const T e10 = K8 * s.c00 + K9 * s.c10;
    const T e11 = K8 * s.c10 + K9 * s.c11;
    const T e13 = K8 * s.c30 + K9 * s.c31;
    const T e14 = K8 * s.c40 + K9 * s.c41;
    const T e15 = K10 * s.c00 + K11 * s.c10;
    const T e16 = K10 * s.c10 + K11 * s.c11;
    const T e18 = K10 * s.c30 + K11 * s.c31;
    const T e19 = K10 * s.c40 + K11 * s.c41;
    const T e20 = K10 * s.c50 + K11 * s.c51;
    s.c00 = s.c00 - e0;  s.c10 = s.c10 - e1;  s.c11 = s.c11 - e2;
    s.c30 = s.c30 - e6;  s.c31 = s.c31 - e7;  s.c33 = s.c33 - e9;
    s.c40 = s.c40 - e10; s.c41 = s.c41 - e11; s.c43 = s.c43 - e13; s.c44 = s.c44 - e14;
    s.c50 = s.c50 - e15; s.c51 = s.c51 - e16; s.c53 = s.c53 - e18; s.c54 = s.c54 - e19; s.c55 = s.c55 - e20;
  }
}

// KalmanUpdate_v2 (reference :503-620): R = C(xy) + V(xy), its inverse by
// Cramer's rule, gain, parameter and covariance update.
// FORM_REFERENCE: the determinant in FP64 from the float entries and 1.f/det as
// a double division rounded to float, as the reference.
// FORM_PRECISE: Kahan's compensated FP32 determinant (error <= 2 ulp of the
// exact determinant of the float entries, the same bound as the FP64 product
// rounded to float) and a correctly rounded float reciprocal -- no FP64.
// Returns true when det <= 0 (or NaN).
template <typename A, int FORM, bool FIRST = false>
__device__ __forceinline__ bool update_v2(Trk<float, A> &s, const float (&hp)[3], const float (&hc)[3]) {
  float r00 = s.c00 + hc[0];
  float r01 = s.c10 + hc[1];
  float r11 = s.c11 + hc[2];
  float sc;
  bool bad;
  if constexpr (FORM == FORM_REFERENCE) {
    const double det = (double)r00 * r11 - (double)r01 * r01;
    sc = 1.f / det;
    bad = !(det > 0.0);
  } else {
    const float det = det2_comp(r00, r01, r01, r11);
    sc = rcp_nr(det);
    bad = !(det > 0.0f);
  }
  const float tmp = sc * r11;
  r01 *= -sc;
  r11 = sc * r00;
  r00 = tmp;
  update_v2_apply<float, A, FORM, FIRST>(s, r00, r01, r11, hp[0], hp[1], hc);
  return bad;
}

// FP64 2-D update for the all-FP64 kernel.
__device__ __forceinline__ bool update_v2_f64(Trk<double, double> &s, const double (&hp)[3], const double (&hc)[3]) {
  const double r00 = s.c00 + hc[0], r01 = s.c10 + hc[1], r11 = s.c11 + hc[2];
  const double det = r00 * r11 - r01 * r01;
  const double id = 1.0 / det;
  update_v2_apply<double, double, FORM_PRECISE>(s, r11 * id, -r01 * id, r00 * id, hp[0], hp[1], hc);
  return !(det > 0.0);
}

// 3-D (x,y,z) measurement update with a Joseph-form covariance update, in
// precision U (double: the FP64 island; float: FP64-free with compensated
// cofactors).  The hit covariance is the packed 3x3 (V00 V10 V11 V20 V21 V22).
// After a propagation C's z row is zero, so R = [[C00+V00, C10+V10, V20],
// [., C11+V11, V21], [., ., V22]], the gain's z row is zero and the z
// residual is exactly 0.
template <typename U>
__device__ __forceinline__ U cof2(U a, U b, U c, U d) { return a * d - b * c; }
template <>
__device__ __forceinline__ float cof2<float>(float a, float b, float c, float d) { return det2_comp(a, b, c, d); }

template <typename U, typename A>
__device__ __forceinline__ bool update_3x3_joseph(Trk<float, A> &s, const float (&hp)[3], const float (&hv)[6]) {
  const U v00 = hv[0], v10 = hv[1], v11 = hv[2], v20 = hv[3], v21 = hv[4], v22 = hv[5];
  // C's live elements as they enter the update, in float (converted where used)
  const float f00 = s.c00, f10 = s.c10, f11 = s.c11, f30 = s.c30, f31 = s.c31, f33 = s.c33;
  const float f40 = s.c40, f41 = s.c41, f43 = s.c43, f44 = s.c44;
  const float f50 = s.c50, f51 = s.c51, f53 = s.c53, f54 = s.c54, f55 = s.c55;
  const U C00 = f00, C10 = f10, C11 = f11, C30 = f30, C31 = f31, C40 = f40, C41 = f41, C50 = f50, C51 = f51;
  const U R00 = C00 + v00, R10 = C10 + v10, R11 = C11 + v11, R20 = v20, R21 = v21, R22 = v22;
  // cofactors of the symmetric R; cof2(a, b, c, d) = a*d - b*c
  const U A00 = cof2<U>(R11, R21, R21, R22);  // R11*R22 - R21*R21
  const U A10 = cof2<U>(R20, R10, R22, R21);  // R20*R21 - R10*R22
  const U A20 = cof2<U>(R10, R20, R11, R21);  // R10*R21 - R20*R11
  const U A11 = cof2<U>(R00, R20, R20, R22);  // R00*R22 - R20*R20
  const U A21 = cof2<U>(R20, R00, R21, R10);  // R20*R10 - R00*R21
  const U A22 = cof2<U>(R00, R10, R10, R11);  // R00*R11 - R10*R10
  const U det = R00 * A00 + R10 * A10 + R20 * A20;
  const U id = U(1) / det;
  const U I00 = A00 * id, I10 = A10 * id, I20 = A20 * id, I11 = A11 * id, I21 = A21 * id, I22 = A22 * id;
  (void)I22;
  // K = C H^T R^-1 for the live rows x, y, ipt, phi, theta; (C H^T)(i,:) = (C(i,0), C(i,1), 0).
  const U K[5][3] = {{C00 * I00 + C10 * I10, C00 * I10 + C10 * I11, C00 * I20 + C10 * I21},
                     {C10 * I00 + C11 * I10, C10 * I10 + C11 * I11, C10 * I20 + C11 * I21},
                     {C30 * I00 + C31 * I10, C30 * I10 + C31 * I11, C30 * I20 + C31 * I21},
                     {C40 * I00 + C41 * I10, C40 * I10 + C41 * I11, C40 * I20 + C41 * I21},
                     {C50 * I00 + C51 * I10, C50 * I10 + C51 * I11, C50 * I20 + C51 * I21}};
  // residual: z residual is hz - z = 0 after the propagation to z = hz
  const float r0 = acc_res(hp[0], s.x), r1 = acc_res(hp[1], s.y);
  acc_update(s.x, hp[0], r0, float(K[0][0] * U(r0) + K[0][1] * U(r1)));
  acc_update(s.y, hp[1], r1, float(K[1][0] * U(r0) + K[1][1] * U(r1)));
  s.ipt = float(U(s.ipt) + (K[2][0] * U(r0) + K[2][1] * U(r1)));
  const float dphi = float(K[3][0] * U(r0) + K[3][1] * U(r1));
  const float theta_new = float(U(s.theta) + (K[4][0] * U(r0) + K[4][1] * U(r1)));
  const float dth = theta_new - s.theta;
  acc_add(s.phi, dphi);
  s.theta = theta_new;
  turn_direction(s, dphi, dth);
  // Joseph form C'' = (I - K H) C (I - K H)^T + K V K^T, evaluated as
  // C'' = P - E K^T with P = (I - K H) C and E = P H^T - K V: exact for any
  // gain, since P (I - K H)^T = P - P H^T K^T.  P(i,j) = C(i,j) - K(i,0) C(0,j)
  // - K(i,1) C(1,j) (C(2,j) = 0) and P(i,2) = 0, so E(i,m) = P(i,m) - (K V)(i,m)
  // for m = x, y and E(i,z) = -(K V)(i,z).  Three products per element of C''
  // instead of the five of P - P H^T K^T + K V K^T.
  // One row of C'' at a time (rows x, y, ipt, phi, theta of the live 5x5
  // block), so that only the gain, C's rows x and y (the measured columns, kept
  // as they were) and the current row are live: C'' is written into the track
  // as each row is finished.
  const float Cr0[5] = {f00, f10, f30, f40, f50};  // C(0, j)
  const float Cr1[5] = {f10, f11, f31, f41, f51};  // C(1, j)
  float *const out[5][5] = {{&s.c00, nullptr, nullptr, nullptr, nullptr},
                            {&s.c10, &s.c11, nullptr, nullptr, nullptr},
                            {&s.c30, &s.c31, &s.c33, nullptr, nullptr},
                            {&s.c40, &s.c41, &s.c43, &s.c44, nullptr},
                            {&s.c50, &s.c51, &s.c53, &s.c54, &s.c55}};
  const float Crow[5][5] = {{f00, f10, f30, f40, f50},
                            {f10, f11, f31, f41, f51},
                            {f30, f31, f33, f43, f53},
                            {f40, f41, f43, f44, f54},
                            {f50, f51, f53, f54, f55}};
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    U P[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) P[j] = U(Crow[i][j]) - (K[i][0] * U(Cr0[j]) + K[i][1] * U(Cr1[j]));
    const U E0 = P[0] - (K[i][0] * v00 + K[i][1] * v10 + K[i][2] * v20);
    const U E1 = P[1] - (K[i][0] * v10 + K[i][1] * v11 + K[i][2] * v21);
    const U E2 = -(K[i][0] * v20 + K[i][1] * v21 + K[i][2] * v22);
#pragma unroll
    for (int j = 0; j <= i; ++j) *out[i][j] = float(P[j] - (E0 * K[j][0] + E1 * K[j][1] + E2 * K[j][2]));
  }
  return !(det > U(0));
}

}  // namespace p2z
