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
// `weno3_fast` / `weno5_fast` are the FP32 forms of the mixed-precision path:
// the same Jiang-Shu weights, regrouped for FMA and one reciprocal per face.
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

// FP32 forms (mixed-precision path).  Same weights, factored smoothness
// indicators, one reciprocal for the normalisation.
__device__ __forceinline__ float weno3_fast(float v0, float v1, float v2) {
  const float eps = 1e-16f;
  float d0 = v1 - v0, d1 = v2 - v1;
  float b0 = d0 * d0, b1 = d1 * d1;
  float a0 = __fdividef(1.0f / 3.0f, fmaf(b0, b0, eps));
  float a1 = __fdividef(2.0f / 3.0f, fmaf(b1, b1, eps));
  float s0 = fmaf(1.5f, v1, -0.5f * v0);
  float s1 = 0.5f * (v2 + v1);
  float num = fmaf(a0, s0, a1 * s1);
  return __fdividef(num, a0 + a1);
}

__device__ __forceinline__ float weno5_fast(float v0, float v1, float v2, float v3, float v4) {
  // Jiang-Shu indicators times 4: 13/3 (a - 2b + c)^2 + (.)^2.  The factor
  // scales every alpha by 1/16 once eps is scaled by 16, and the linear
  // weights (0.1, 0.6, 0.3) are taken times 10; neither changes the
  // normalised weights.
  const float eps16 = 16e-16f;
  const float t0 = fmaf(-2.0f, v1, v0) + v2, u0 = fmaf(3.0f, v2, fmaf(-4.0f, v1, v0));
  const float t1 = fmaf(-2.0f, v2, v1) + v3, u1 = v1 - v3;
  const float t2 = fmaf(-2.0f, v3, v2) + v4, u2 = fmaf(3.0f, v2, fmaf(-4.0f, v3, v4));
  const float c13 = 13.0f / 3.0f;
  const float b0 = fmaf(c13 * t0, t0, u0 * u0);
  const float b1 = fmaf(c13 * t1, t1, u1 * u1);
  const float b2 = fmaf(c13 * t2, t2, u2 * u2);
  const float a0 = __fdividef(1.0f, fmaf(b0, b0, eps16));
  const float a1 = __fdividef(6.0f, fmaf(b1, b1, eps16));
  const float a2 = __fdividef(3.0f, fmaf(b2, b2, eps16));
  // candidate stencils at the face, the 1/6 folded into the coefficients
  const float s0 = fmaf(11.0f / 6.0f, v2, fmaf(-7.0f / 6.0f, v1, (1.0f / 3.0f) * v0));
  const float s1 = fmaf(1.0f / 3.0f, v3, fmaf(5.0f / 6.0f, v2, (-1.0f / 6.0f) * v1));
  const float s2 = fmaf(-1.0f / 6.0f, v4, fmaf(5.0f / 6.0f, v3, (1.0f / 3.0f) * v2));
  return __fdividef(fmaf(a0, s0, fmaf(a1, s1, a2 * s2)), a0 + a1 + a2);
}

}  // namespace mth
