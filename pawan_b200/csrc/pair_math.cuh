// Per-pair regularised Biot-Savart / stretching / diffusion terms of PAWAN's
// vortex-particle kernels, for FP32 (compensated accumulation around it) and
// FP64: the Gaussian kernel (below, and the FP32 three-regime form further
// down) and the high-order algebraic kernel (pair_terms_ho).
//
// Reference algorithm (src/interaction/gaussian.h:20-60 and
// src/interaction/interaction_utils.h:55-105, 344-378, 523-576), per ordered
// pair (target t, source s), d = x_t - x_s, rho = |d|,
// sigma^2 = (sigma_s^2 + sigma_t^2)/2, u = rho^2 / sigma^2:
//   zeta = exp(-u/2) / ((2 pi)^(3/2) sigma^3)
//   q    = (erf(sqrt(u/2)) / (4 pi sigma^3 sqrt(u)) - zeta) / u
//   F    = (zeta - 3 q) / rho^2
//   u_t  += q (a_s x d)
//   da_t += q (a_t x a_s) + F (d . (a_t x a_s)) d + nu zeta/(sigma^2/2) (v_t a_s - v_s a_t)
//
// Everything here is carried in units scaled by 4 pi (q' = 4 pi q, F' = 4 pi F,
// z' = 4 pi zeta) so no per-pair constant multiplies are needed; the caller
// multiplies the accumulated sums by 1/(4 pi) once per target.  With
// k1 = sqrt(2/pi) = 4 pi / (2 pi)^(3/2) and r = 1/rho, s = 1/sigma:
//   z' = k1 s^3 e^{-u/2}
//   q' = r^2 (erf(sqrt(u/2)) r - k1 e^{-u/2} s)
//   F' = (z' - 3 q') r^2
//
// Small-u branch.  The closed form cancels catastrophically as u -> 0 (q loses
// about log10(3/u) digits, F about log10(15/u^2)).  Below a threshold the
// series of the same functions is used instead, derived from
//   g(x) = erf(x/sqrt2) - sqrt(2/pi) x e^{-x^2/2} = sqrt(2/pi) int_0^x t^2 e^{-t^2/2} dt
// which gives, with u = x^2,
//   q' = k1 s^3 S(u),   S(u) = sum_k (-1)^k u^k / (2^k k! (2k+3))
//   F' = -k1 s^5 T(u),  T(u) = sum_m (-1)^m u^m / (2^m m! (2m+5))
// Both are finite at u = 0; the series branch (the only one a zero distance
// reaches) zeroes all three terms at rho = 0, so the self pair contributes
// exact zeros without an index comparison in the inner loop.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace pgpu {

// Packed particle record as stored in HBM and staged in shared memory:
// P = (x, y, z, sigma^2/2), Q = (alpha_x, alpha_y, alpha_z, volume).
template <typename T> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };
template <typename T> using v4_t = typename V4<T>::type;

constexpr double kK1 = 0.7978845608028654;       // sqrt(2/pi)
constexpr double kInv4Pi = 0.07957747154594767;  // 1/(4 pi)
constexpr double kNegHalfLog2e = -0.7213475204444817;  // -0.5 / ln 2
constexpr double kInv2Pi15 = 0.06349363593424097;     // (2 pi)^-1.5

// Series coefficients S_k = (-1)^k/(2^k k!(2k+3)), T_m = (-1)^m/(2^m m!(2m+5)).
#define PGPU_S0 0.3333333333333333
#define PGPU_S1 -0.1
#define PGPU_S2 0.017857142857142856
#define PGPU_S3 -0.0023148148148148147
#define PGPU_S4 0.00023674242424242425
#define PGPU_S5 -2.0032051282051282e-05
#define PGPU_S6 1.4467592592592592e-06
#define PGPU_S7 -9.118230625583566e-08
#define PGPU_S8 5.099010547201337e-09
#define PGPU_T0 0.2
#define PGPU_T1 -0.07142857142857142
#define PGPU_T2 0.013888888888888888
#define PGPU_T3 -0.001893939393939394
#define PGPU_T4 0.00020032051282051281
#define PGPU_T5 -1.736111111111111e-05
#define PGPU_T6 1.2765522875816993e-06
#define PGPU_T7 -8.158416875522139e-08
#define PGPU_T8 4.613390495086924e-09

// Threshold on u below which the series is used.  FP32: the closed form keeps
// ~1e-6 relative accuracy for F at u = 1, and 9 terms of the series are
// accurate to ~1e-8 on [0, 1].  FP64: at u = 1e-2 the closed form keeps
// ~3e-14 and 9 terms are exact to rounding.
template <typename T> struct SeriesCut;
template <> struct SeriesCut<float> { static constexpr float value = 1.0f; };
template <> struct SeriesCut<double> { static constexpr double value = 1.0e-2; };

__device__ __forceinline__ float fast_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fast_exp2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <typename T> struct PairTerms {
  T q;   // 4 pi q
  T F;   // 4 pi F
  T zd;  // 4 pi zeta / sigma^2   (diffusion weight before the factor 2 nu)
};

// r2 = rho^2, s2 = sigma_ts^2.
__device__ __forceinline__ PairTerms<float> pair_terms(float r2, float s2) {
  PairTerms<float> o;
  const float is = fast_rsqrt(s2);
  const float is2 = is * is;
  const float u = r2 * is2;
  const float E = fast_exp2(u * (float)kNegHalfLog2e);
  const float zk = (float)kK1 * is * is2;  // k1 / sigma^3
  const float z = zk * E;
  if (u < SeriesCut<float>::value) {
    float S = (float)PGPU_S8;
    S = fmaf(S, u, (float)PGPU_S7); S = fmaf(S, u, (float)PGPU_S6); S = fmaf(S, u, (float)PGPU_S5);
    S = fmaf(S, u, (float)PGPU_S4); S = fmaf(S, u, (float)PGPU_S3); S = fmaf(S, u, (float)PGPU_S2);
    S = fmaf(S, u, (float)PGPU_S1); S = fmaf(S, u, (float)PGPU_S0);
    float Tt = (float)PGPU_T8;
    Tt = fmaf(Tt, u, (float)PGPU_T7); Tt = fmaf(Tt, u, (float)PGPU_T6); Tt = fmaf(Tt, u, (float)PGPU_T5);
    Tt = fmaf(Tt, u, (float)PGPU_T4); Tt = fmaf(Tt, u, (float)PGPU_T3); Tt = fmaf(Tt, u, (float)PGPU_T2);
    Tt = fmaf(Tt, u, (float)PGPU_T1); Tt = fmaf(Tt, u, (float)PGPU_T0);
    // rho = 0 only for the self pair (or coincident particles, where PAWAN's
    // closed form yields NaN): it contributes nothing.
    const float m = r2 > 0.0f ? 1.0f : 0.0f;
    o.q = zk * S * m;
    o.F = -zk * is2 * Tt * m;
    o.zd = z * is2 * m;
  } else {
    const float ir = fast_rsqrt(r2);
    const float ir2 = ir * ir;
    const float y = r2 * ir * (is * 0.70710678118654752f);  // rho / (sigma sqrt 2)
    const float er = erff(y);
    o.q = ir2 * fmaf(-(float)kK1 * is, E, er * ir);
    o.F = fmaf(-3.0f, o.q, z) * ir2;
    o.zd = z * is2;
  }
  return o;
}

__device__ __forceinline__ PairTerms<double> pair_terms(double r2, double s2) {
  PairTerms<double> o;
  const double is = rsqrt(s2);
  const double is2 = is * is;
  const double u = r2 * is2;
  const double E = exp(-0.5 * u);
  const double zk = kK1 * is * is2;
  const double z = zk * E;
  if (u < SeriesCut<double>::value) {
    double S = PGPU_S8;
    S = fma(S, u, PGPU_S7); S = fma(S, u, PGPU_S6); S = fma(S, u, PGPU_S5); S = fma(S, u, PGPU_S4);
    S = fma(S, u, PGPU_S3); S = fma(S, u, PGPU_S2); S = fma(S, u, PGPU_S1); S = fma(S, u, PGPU_S0);
    double Tt = PGPU_T8;
    Tt = fma(Tt, u, PGPU_T7); Tt = fma(Tt, u, PGPU_T6); Tt = fma(Tt, u, PGPU_T5); Tt = fma(Tt, u, PGPU_T4);
    Tt = fma(Tt, u, PGPU_T3); Tt = fma(Tt, u, PGPU_T2); Tt = fma(Tt, u, PGPU_T1); Tt = fma(Tt, u, PGPU_T0);
    const double m = r2 > 0.0 ? 1.0 : 0.0;
    o.q = zk * S * m;
    o.F = -zk * is2 * Tt * m;
    o.zd = z * is2 * m;
  } else {
    const double rho = sqrt(r2);
    const double ir = 1.0 / rho;
    const double ir2 = ir * ir;
    const double er = erf(rho * is * 0.70710678118654752440);
    o.q = ir2 * (er * ir - kK1 * is * E);
    o.F = (z - 3.0 * o.q) * ir2;
    o.zd = z * is2;
  }
  return o;
}

// ---------------------------------------------------------------- high-order algebraic kernel
// PAWAN's second regularisation (src/interaction/highorder.h:20-60), selected
// in PAWAN at compile time (interaction_utils.h:13-20).  With rb = rho/sigma,
// w = rb^2 + 1:
//   zeta = 1.875 / (pi sigma^3 w^3.5)                       (ZETASIG)
//   q    = rb^3 (rb^2 + 2.5) / (4 pi w^2.5 rho^3)           (QSIG)
//   eta  = 13.125 / (pi sigma^3 w^4.5)                      (ETASIG, the diffusion kernel)
//   F    = (zeta - 3 q) / rho^2                             (KERNEL)
// In the 4 pi scaled units of PairTerms, with s2 = sigma^2, r2 = rho^2 and
// R = r2 + s2 (so that rb^2 + 1 = R / s2 and every power of sigma cancels):
//   q'   = (r2 + 2.5 s2) R^-2.5
//   F'   = (7.5 s2^2 R^-3.5 - 3 q') / r2 = -3 (r2 + 3.5 s2) R^-3.5
//   zd'  = 4 pi eta / s2 = 52.5 s2^2 R^-4.5
//   zeta = 1.875 / pi s2^2 R^-3.5
// The reduced F' is PAWAN's (zeta - 3 q)/rho^2 with the 1/rho^2 cancelled by
// hand, so it has no cancellation as rho -> 0, and all terms come from one
// reciprocal square root of R, a sum of two positive numbers.  As for the
// Gaussian kernel, the terms are zeroed at rho = 0: the self pair (and
// coincident particles, where PAWAN's QSIG is 0/0) contributes exact zeros;
// with contracted multiply-adds v_t a_t - v_t a_t would not be.
//
// FP32: F' carries R^-3.5, so a relative error e of the reciprocal square
// root becomes 3.5 e.  The hardware approximation's error is a fixed function
// of its input, so it does not average out over the sum; one Newton step
// brings the root to about one rounding.
struct HighOrder {
  static constexpr double kQ0 = 2.5, kF0 = 3.5, kZd = 52.5, kZeta = 7.5;
};

// 1/sqrt(x) for normal x > 0: the approximation plus one Newton step
// y (3 - x y^2) / 2.
__device__ __forceinline__ float rsqrt_nr(float x) {
  const float y = fast_rsqrt(x);
  return y * fmaf(-0.5f * x * y, y, 1.5f);
}

__device__ __forceinline__ PairTerms<float> pair_terms_ho(float r2, float s2) {
  const float m = r2 > 0.0f ? 1.0f : 0.0f;
  const float iR = rsqrt_nr(r2 + s2);
  const float iR2 = iR * iR;
  const float iR5 = iR2 * iR2 * iR;
  const float iR7 = iR5 * iR2;
  PairTerms<float> o;
  o.q = fmaf((float)HighOrder::kQ0, s2, r2) * (iR5 * m);
  o.F = fmaf((float)HighOrder::kF0, s2, r2) * (iR7 * (-3.0f * m));
  o.zd = ((float)HighOrder::kZd * s2 * s2) * (iR7 * iR2 * m);
  return o;
}

__device__ __forceinline__ PairTerms<double> pair_terms_ho(double r2, double s2) {
  const double m = r2 > 0.0 ? 1.0 : 0.0;
  const double iR = 1.0 / sqrt(r2 + s2);
  const double iR2 = iR * iR;
  const double iR5 = iR2 * iR2 * iR;
  const double iR7 = iR5 * iR2;
  PairTerms<double> o;
  o.q = fma(HighOrder::kQ0, s2, r2) * (iR5 * m);
  o.F = fma(HighOrder::kF0, s2, r2) * (iR7 * (-3.0 * m));
  o.zd = (HighOrder::kZd * s2 * s2) * (iR7 * iR2 * m);
  return o;
}

// Kernel selection (PGPU_KERNEL_GAUSSIAN = 0, PGPU_KERNEL_HIGHORDER = 1).
constexpr int kGaussian = 0;
constexpr int kHighOrder = 1;

// ---------------------------------------------------------------- FP32 three-regime form
// The FP32 pair kernel splits pairs by u = rho^2 / sigma^2:
//
//   far   u >= 50: erf(sqrt(u/2)) rounds to 1 and e^{-u/2} < 1.4e-11, so at
//         FP32 precision q' = r^3, F' = -3 r^5 and zeta' = 0 (the dropped
//         terms are below 1e-9 of q and F).  ~33 instructions per pair.
//   mid   1 <= u < 50: closed form, with erf(y) = 1 - e^{-y^2} erfcx(y),
//         y = sqrt(u/2), so the exponential already needed for zeta serves
//         both.  erfcx is the project's own fit (below).
//   near  u < 1: the series S(u), T(u) above.
//
// erfcx(y) = e^{y^2} erfc(y) on y in [1/sqrt2, 5] (u in [1, 50]) is fitted as
// erfcx(y) = z P(t), z = 1/y in [0.2, sqrt2], t = a z + b in [-1, 1], P a
// degree-10 polynomial: weighted Chebyshev least squares against SciPy's
// erfcx, converted to the monomial basis in t.  In FP32 arithmetic the
// resulting erf(y) has absolute error <= 5e-8 on the whole interval
// (checked on 4e5 points against FP64 erfcx).
constexpr float kFarU = 50.0f;
constexpr float kErfcxA = 1.6471567153930664f;   // t = a z + b
constexpr float kErfcxB = -1.3294312953948975f;
#define PGPU_E0 0.45859402418136597f
#define PGPU_E1 -0.10109120607376099f
#define PGPU_E2 0.009336095303297043f
#define PGPU_E3 0.0067022028379142284f
#define PGPU_E4 -0.005510672926902771f
#define PGPU_E5 0.0025757858529686928f
#define PGPU_E6 -0.0008601871086284518f
#define PGPU_E7 0.00020045014389324933f
#define PGPU_E8 8.555142267141491e-05f
#define PGPU_E9 -0.00018502288730815053f
#define PGPU_E10 8.057637023739517e-05f

// P(t); erfcx(y) = z P(t).
__device__ __forceinline__ float erfcx_poly(float t) {
  float p = PGPU_E10;
  p = fmaf(p, t, PGPU_E9); p = fmaf(p, t, PGPU_E8); p = fmaf(p, t, PGPU_E7); p = fmaf(p, t, PGPU_E6);
  p = fmaf(p, t, PGPU_E5); p = fmaf(p, t, PGPU_E4); p = fmaf(p, t, PGPU_E3); p = fmaf(p, t, PGPU_E2);
  p = fmaf(p, t, PGPU_E1); p = fmaf(p, t, PGPU_E0);
  return p;
}

// Non-far FP32 terms (u < 50).  With r = 1/rho, s = 1/sigma, A = r^2,
// z = sqrt2 sigma r:
//   q' = r^2 (erf r - k1 s E) = A r - E A (r z P + k1 s)
__device__ __forceinline__ PairTerms<float> pair_terms_near(float r2, float s2) {
  PairTerms<float> o;
  const float is = fast_rsqrt(s2);
  const float is2 = is * is;
  const float u = r2 * is2;
  const float E = fast_exp2(u * (float)kNegHalfLog2e);
  const float zk = (float)kK1 * is * is2;
  const float z = zk * E;
  if (u < SeriesCut<float>::value) {
    float S = (float)PGPU_S8;
    S = fmaf(S, u, (float)PGPU_S7); S = fmaf(S, u, (float)PGPU_S6); S = fmaf(S, u, (float)PGPU_S5);
    S = fmaf(S, u, (float)PGPU_S4); S = fmaf(S, u, (float)PGPU_S3); S = fmaf(S, u, (float)PGPU_S2);
    S = fmaf(S, u, (float)PGPU_S1); S = fmaf(S, u, (float)PGPU_S0);
    float Tt = (float)PGPU_T8;
    Tt = fmaf(Tt, u, (float)PGPU_T7); Tt = fmaf(Tt, u, (float)PGPU_T6); Tt = fmaf(Tt, u, (float)PGPU_T5);
    Tt = fmaf(Tt, u, (float)PGPU_T4); Tt = fmaf(Tt, u, (float)PGPU_T3); Tt = fmaf(Tt, u, (float)PGPU_T2);
    Tt = fmaf(Tt, u, (float)PGPU_T1); Tt = fmaf(Tt, u, (float)PGPU_T0);
    const float m = r2 > 0.0f ? 1.0f : 0.0f;  // self pair contributes nothing
    o.q = zk * S * m;
    o.F = -zk * is2 * Tt * m;
    o.zd = z * is2 * m;
  } else {
    const float ir = fast_rsqrt(r2);
    const float A = ir * ir;
    const float zs = (1.41421356237309515f * s2) * is;  // sqrt2 sigma
    const float t = fmaf(kErfcxA * zs, ir, kErfcxB);
    const float P = erfcx_poly(t);
    const float B = fmaf(zs * A, P, (float)kK1 * is);
    o.q = fmaf(-(E * A), B, A * ir);
    o.F = fmaf(-3.0f, o.q, z) * A;
    o.zd = z * is2;
  }
  return o;
}

// Two pairs at once (lanes .x and .y of every float2, packed FP32 of sm_100):
// the mid branch of pair_terms_near, valid for u = r2 / s2 >= 1.  For
// u >= 50 its e^{-u/2} terms fall below 1.4e-11 and it equals the far limit
// to FP32 rounding.  Lanes with u < 1 (the self pair among them) must be
// redone with pair_terms_near.  -P and -B are formed with negated
// coefficients, so each lane rounds exactly as the scalar branch does.
struct PairTerms2 {
  float2 q, F, zd;
};
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

__device__ __forceinline__ PairTerms2 pair_terms_mid2(float2 r2, float2 s2) {
  const float2 is = make_float2(fast_rsqrt(s2.x), fast_rsqrt(s2.y));
  const float2 is2 = __fmul2_rn(is, is);
  const float2 ea = __fmul2_rn(__fmul2_rn(r2, is2), dup2((float)kNegHalfLog2e));
  const float2 E = make_float2(fast_exp2(ea.x), fast_exp2(ea.y));
  const float2 z = __fmul2_rn(__fmul2_rn(__fmul2_rn(dup2((float)kK1), is), is2), E);  // (k1 s) s^2 E
  const float2 ir = make_float2(fast_rsqrt(r2.x), fast_rsqrt(r2.y));
  const float2 A = __fmul2_rn(ir, ir);
  const float2 zs = __fmul2_rn(__fmul2_rn(dup2(1.41421356237309515f), s2), is);  // sqrt2 sigma
  const float2 t = __ffma2_rn(__fmul2_rn(dup2(kErfcxA), zs), ir, dup2(kErfcxB));
  float2 np = dup2(-PGPU_E10);
  np = __ffma2_rn(np, t, dup2(-PGPU_E9)); np = __ffma2_rn(np, t, dup2(-PGPU_E8));
  np = __ffma2_rn(np, t, dup2(-PGPU_E7)); np = __ffma2_rn(np, t, dup2(-PGPU_E6));
  np = __ffma2_rn(np, t, dup2(-PGPU_E5)); np = __ffma2_rn(np, t, dup2(-PGPU_E4));
  np = __ffma2_rn(np, t, dup2(-PGPU_E3)); np = __ffma2_rn(np, t, dup2(-PGPU_E2));
  np = __ffma2_rn(np, t, dup2(-PGPU_E1)); np = __ffma2_rn(np, t, dup2(-PGPU_E0));
  const float2 nB = __ffma2_rn(__fmul2_rn(zs, A), np, __fmul2_rn(dup2(-(float)kK1), is));
  PairTerms2 o;
  o.q = __ffma2_rn(__fmul2_rn(E, A), nB, __fmul2_rn(A, ir));
  o.F = __fmul2_rn(__ffma2_rn(dup2(-3.0f), o.q, z), A);
  o.zd = __fmul2_rn(z, is2);
  return o;
}

// Error-free addition (Knuth two-sum): hi + lo == a + b exactly.  The
// explicit _rn intrinsics keep the compiler from contracting or reordering.
__device__ __forceinline__ void two_sum_acc(float &hi, float &lo, float b) {
  const float s = __fadd_rn(hi, b);
  const float bb = __fsub_rn(s, hi);
  const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  hi = s;
  lo = __fadd_rn(lo, e);
}
__device__ __forceinline__ void two_sum_acc(double &hi, double &lo, double b) {
  const double s = __dadd_rn(hi, b);
  const double bb = __dsub_rn(s, hi);
  const double e = __dadd_rn(__dsub_rn(hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  hi = s;
  lo = __dadd_rn(lo, e);
}

}  // namespace pgpu
