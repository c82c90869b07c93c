// WENO3 / WENO5 point reconstructions.
//
// `weno3_exact` / `weno5_exact` evaluate the same expressions, in the same
// order, as the reference's generated point kernels
// (Project/CPU/Src/wenoUpwinds.cc:5-33 and 36-83): smoothness indicators
// accumulated term by term from zero, alpha_k = d_k / (1e-16 + beta_k^2),
// weights by division by the alpha sum, stencils accumulated term by term.
// Compiled without FMA contraction (-fmad=false) they are bit-identical to the
// reference's x86-64 build.  The downwind value at a face is the same
// function applied to the mirrored stencil (Project/CPU/Src/weno.cc:145-164,
// 208-228), so only the upwind form exists here.
//
// `weno3_fast2` / `weno5_fast2` are the FP32 forms of the mixed-precision
// path: the same Jiang-Shu weights, regrouped for FMA, with approximate
// reciprocals, evaluating the upwind and downwind sides of a face together.
#pragma once

namespace mth {

__device__ __forceinline__ double weno3_exact(double v0, double v1, double v2) {
  const double eps = 1e-16;
  double b0 = 0, b1 = 0, s0 = 0, s1 = 0;
  b0 += 1.0 * v1 * v1;
  b0 += -2.0 * v0 * v1;
  b0 += 1.0 * v0 * v0;
  double a0 = 0.3333333333333333 / (eps + b0 * b0);
  b1 += 1.0 * v2 * v2;
  b1 += -2.0 * v1 * v2;
  b1 += 1.0 * v1 * v1;
  double a1 = 0.6666666666666666 / (eps + b1 * b1);
  double asum = a0 + a1;
  double w0 = a0 / asum;
  double w1 = a1 / asum;
  s0 += 1.5 * v1;
  s0 += -0.5 * v0;
  s1 += 0.5 * v2;
  s1 += 0.5 * v1;
  return (w0 * s0 + w1 * s1);
}

__device__ __forceinline__ double weno5_exact(double v0, double v1, double v2, double v3,
                                              double v4) {
  const double eps = 1e-16;
  double b0 = 0, b1 = 0, b2 = 0, s0 = 0, s1 = 0, s2 = 0;
  b0 += 3.3333333333333335 * v2 * v2;
  b0 += -10.333333333333334 * v1 * v2;
  b0 += 8.333333333333334 * v1 * v1;
  b0 += 3.6666666666666665 * v0 * v2;
  b0 += -6.333333333333333 * v0 * v1;
  b0 += 1.3333333333333333 * v0 * v0;
  double a0 = 0.1 / (eps + b0 * b0);
  b1 += 1.3333333333333333 * v3 * v3;
  b1 += -4.333333333333333 * v2 * v3;
  b1 += 4.333333333333333 * v2 * v2;
  b1 += 1.6666666666666667 * v1 * v3;
  b1 += -4.333333333333333 * v1 * v2;
  b1 += 1.3333333333333333 * v1 * v1;
  double a1 = 0.6 / (eps + b1 * b1);
  b2 += 1.3333333333333333 * v4 * v4;
  b2 += -6.333333333333333 * v3 * v4;
  b2 += 8.333333333333334 * v3 * v3;
  b2 += 3.6666666666666665 * v2 * v4;
  b2 += -10.333333333333334 * v2 * v3;
  b2 += 3.3333333333333335 * v2 * v2;
  double a2 = 0.3 / (eps + b2 * b2);
  double asum = a0 + a1 + a2;
  double w0 = a0 / asum;
  double w1 = a1 / asum;
  double w2 = a2 / asum;
  s0 += 1.8333333333333333 * v2;
  s0 += -1.1666666666666667 * v1;
  s0 += 0.3333333333333333 * v0;
  s1 += 0.3333333333333333 * v3;
  s1 += 0.8333333333333334 * v2;
  s1 += -0.16666666666666666 * v1;
  s2 += -0.16666666666666666 * v4;
  s2 += 0.8333333333333334 * v3;
  s2 += 0.3333333333333333 * v2;
  return (w0 * s0 + w1 * s1 + w2 * s2);
}

// FP32 forms: the upwind (.x) and downwind (.y) reconstructions of one face
// in FP32x2 arithmetic (sm_100 __ffma2_rn / __fadd2_rn / __fmul2_rn: one
// instruction for both sides, each lane rounded as the scalar operation).
// Linear weights are taken times 3 (WENO3) and times 10 (WENO5), and the
// WENO5 Jiang-Shu indicators times 4, 13/3 (a - 2b + c)^2 + (.)^2, with eps
// times 16: none of these scalings changes the normalised weights.
//
// One reciprocal per side: with q_k = eps + beta_k^2 the weights
// (d_k / q_k) / sum_j (d_j / q_j) equal d_k P_k / sum_j d_j P_j with P_k the
// product of the other stencils' q (WENO5; for WENO3 simply the other q), so
// only the final normalisation divides.  WENO5 first scales the three q by
// the power of two that brings the largest into [1, 2) (exponent bits only,
// exact), so the products neither overflow for large flux jumps nor
// underflow below the largest weight's scale.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__device__ __forceinline__ float2 rcp2(float2 q) {
  return make_float2(__fdividef(1.0f, q.x), __fdividef(1.0f, q.y));
}

// 2^-floor(log2 m) for a positive normal m below 2^126, from the exponent bits.
__device__ __forceinline__ float pow2_inv(float m) {
  return __int_as_float(0x7F000000 - (__float_as_int(m) & 0x7F800000));
}

__device__ __forceinline__ float2 weno3_fast2(float2 v0, float2 v1, float2 v2) {
  const float2 d0 = __ffma2_rn(f2(-1.0f), v0, v1), d1 = __ffma2_rn(f2(-1.0f), v1, v2);
  const float2 b0 = __fmul2_rn(d0, d0), b1 = __fmul2_rn(d1, d1);
  const float2 q0 = __ffma2_rn(b0, b0, f2(1e-16f)), q1 = __ffma2_rn(b1, b1, f2(1e-16f));
  const float2 s0 = __ffma2_rn(f2(1.5f), v1, __fmul2_rn(f2(-0.5f), v0));
  const float2 s1 = __fmul2_rn(f2(0.5f), __fadd2_rn(v2, v1));
  // weights 1/q0 : 2/q1  =  q1 : 2 q0
  const float2 a1 = __fmul2_rn(f2(2.0f), q0);
  const float2 num = __ffma2_rn(q1, s0, __fmul2_rn(a1, s1));
  return __fmul2_rn(num, rcp2(__fadd2_rn(q1, a1)));
}

__device__ __forceinline__ float2 weno5_fast2(float2 v0, float2 v1, float2 v2, float2 v3,
                                              float2 v4) {
  const float2 t0 = __fadd2_rn(__ffma2_rn(f2(-2.0f), v1, v0), v2);
  const float2 u0 = __ffma2_rn(f2(3.0f), v2, __ffma2_rn(f2(-4.0f), v1, v0));
  const float2 t1 = __fadd2_rn(__ffma2_rn(f2(-2.0f), v2, v1), v3);
  const float2 u1 = __ffma2_rn(f2(-1.0f), v3, v1);
  const float2 t2 = __fadd2_rn(__ffma2_rn(f2(-2.0f), v3, v2), v4);
  const float2 u2 = __ffma2_rn(f2(3.0f), v2, __ffma2_rn(f2(-4.0f), v3, v4));
  const float2 c13 = f2(13.0f / 3.0f);
  const float2 b0 = __ffma2_rn(__fmul2_rn(c13, t0), t0, __fmul2_rn(u0, u0));
  const float2 b1 = __ffma2_rn(__fmul2_rn(c13, t1), t1, __fmul2_rn(u1, u1));
  const float2 b2 = __ffma2_rn(__fmul2_rn(c13, t2), t2, __fmul2_rn(u2, u2));
  float2 q0 = __ffma2_rn(b0, b0, f2(16e-16f));
  float2 q1 = __ffma2_rn(b1, b1, f2(16e-16f));
  float2 q2 = __ffma2_rn(b2, b2, f2(16e-16f));
  const float2 sc = make_float2(pow2_inv(fmaxf(fmaxf(q0.x, q1.x), q2.x)),
                                pow2_inv(fmaxf(fmaxf(q0.y, q1.y), q2.y)));
  q0 = __fmul2_rn(q0, sc);
  q1 = __fmul2_rn(q1, sc);
  q2 = __fmul2_rn(q2, sc);
  // linear weights 1 : 6 : 3 (x10) over q0 : q1 : q2, times q0 q1 q2
  const float2 a0 = __fmul2_rn(q1, q2);
  const float2 a1 = __fmul2_rn(__fmul2_rn(f2(6.0f), q0), q2);
  const float2 a2 = __fmul2_rn(__fmul2_rn(f2(3.0f), q0), q1);
  // candidate stencils at the face, the 1/6 folded into the coefficients
  const float2 c3 = f2(1.0f / 3.0f), c6 = f2(-1.0f / 6.0f), c56 = f2(5.0f / 6.0f);
  const float2 s0 = __ffma2_rn(f2(11.0f / 6.0f), v2,
                               __ffma2_rn(f2(-7.0f / 6.0f), v1, __fmul2_rn(c3, v0)));
  const float2 s1 = __ffma2_rn(c3, v3, __ffma2_rn(c56, v2, __fmul2_rn(c6, v1)));
  const float2 s2 = __ffma2_rn(c6, v4, __ffma2_rn(c56, v3, __fmul2_rn(c3, v2)));
  const float2 num = __ffma2_rn(a0, s0, __ffma2_rn(a1, s1, __fmul2_rn(a2, s2)));
  return __fmul2_rn(num, rcp2(__fadd2_rn(__fadd2_rn(a0, a1), a2)));
}

}  // namespace mth
