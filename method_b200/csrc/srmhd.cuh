// Ideal special-relativistic MHD (SRMHD) cell physics.
//
// Variables (Project/CPU/Src/srmhd.cc:25-55):
//   cons  D, Sx, Sy, Sz, tau, Bx, By, Bz, phi                  (9)
//   prims rho, vx, vy, vz, p, Bx, By, Bz                       (8)
//   aux   h, W, e, c, b0, bx, by, bz, bsq, vsq, BS, Bsq, Ssq   (13)
// Every expression below keeps the reference's association order so that the
// FP64 build without FMA contraction reproduces the reference bit for bit.
#pragma once
#include "common.cuh"
#include "minpack.cuh"

namespace mth {
namespace srmhd {

constexpr int NC = 9, NP = 8, NA = 13;

// FP32 form of the same fluxes (mixed path): B^d / W and the total pressure
// p + b^2/2 are formed once per cell instead of once per term.
__device__ __forceinline__ void flux_fast(const float* c, const float* p, const float* a, int dir,
                                          float* f) {
  const float iW = __fdividef(1.0f, a[1]);
  const float pt = fmaf(a[8], 0.5f, p[4]);
  if (dir == 0) {
    const float bw = p[5] * iW;
    f[0] = c[0] * p[1];
    f[1] = fmaf(c[1], p[1], pt) - a[5] * bw;
    f[2] = c[2] * p[1] - a[6] * bw;
    f[3] = c[3] * p[1] - a[7] * bw;
    f[4] = (c[4] + pt) * p[1] - a[4] * bw;
    f[5] = c[8];
    f[6] = p[6] * p[1] - p[5] * p[2];
    f[7] = p[7] * p[1] - p[5] * p[3];
    f[8] = p[5];
  } else if (dir == 1) {
    const float bw = p[6] * iW;
    f[0] = c[0] * p[2];
    f[1] = c[1] * p[2] - a[5] * bw;
    f[2] = fmaf(c[2], p[2], pt) - a[6] * bw;
    f[3] = c[3] * p[2] - a[7] * bw;
    f[4] = (c[4] + pt) * p[2] - a[4] * bw;
    f[5] = p[5] * p[2] - p[6] * p[1];
    f[6] = c[8];
    f[7] = p[7] * p[2] - p[6] * p[3];
    f[8] = p[6];
  } else {
    const float bw = p[7] * iW;
    f[0] = c[0] * p[3];
    f[1] = c[1] * p[3] - a[5] * bw;
    f[2] = c[2] * p[3] - a[6] * bw;
    f[3] = fmaf(c[3], p[3], pt) - a[7] * bw;
    f[4] = (c[4] + pt) * p[3] - a[4] * bw;
    f[5] = p[5] * p[3] - p[7] * p[1];
    f[6] = p[6] * p[3] - p[7] * p[2];
    f[7] = c[8];
    f[8] = p[6];  // as the reference (srmhd.cc:200)
  }
}

// Model::fluxVector for one cell (srmhd.cc:72-206).  Only aux 1, 4-8 are read.
template <typename R>
__device__ __forceinline__ void flux(const R* c, const R* p, const R* a, int dir, R* f) {
  if constexpr (sizeof(R) == 4) {
    flux_fast(c, p, a, dir, f);
    return;
  }
  if (dir == 0) {
    f[0] = c[0] * p[1];
    f[1] = c[1] * p[1] + (p[4] + a[8] * R(0.5)) - a[5] * p[5] / a[1];
    f[2] = c[2] * p[1] - a[6] * p[5] / a[1];
    f[3] = c[3] * p[1] - a[7] * p[5] / a[1];
    f[4] = (c[4] + p[4] + a[8] * R(0.5)) * p[1] - a[4] * p[5] / a[1];
    f[5] = c[8];
    f[6] = p[6] * p[1] - p[5] * p[2];
    f[7] = p[7] * p[1] - p[5] * p[3];
    f[8] = p[5];
  } else if (dir == 1) {
    f[0] = c[0] * p[2];
    f[1] = c[1] * p[2] - a[5] * p[6] / a[1];
    f[2] = c[2] * p[2] + p[4] + a[8] * R(0.5) - a[6] * p[6] / a[1];
    f[3] = c[3] * p[2] - a[7] * p[6] / a[1];
    f[4] = (c[4] + p[4] + a[8] * R(0.5)) * p[2] - a[4] * p[6] / a[1];
    f[5] = p[5] * p[2] - p[6] * p[1];
    f[6] = c[8];
    f[7] = p[7] * p[2] - p[6] * p[3];
    f[8] = p[6];
  } else {
    f[0] = c[0] * p[3];
    f[1] = c[1] * p[3] - a[5] * p[7] / a[1];
    f[2] = c[2] * p[3] - a[6] * p[7] / a[1];
    f[3] = c[3] * p[3] + p[4] + a[8] * R(0.5) - a[7] * p[7] / a[1];
    f[4] = (c[4] + p[4] + a[8] * R(0.5)) * p[3] - a[4] * p[7] / a[1];
    f[5] = p[5] * p[3] - p[7] * p[1];
    f[6] = p[6] * p[3] - p[7] * p[2];
    f[7] = c[8];
    f[8] = p[6];  // the reference's z flux of phi is By (srmhd.cc:200)
  }
}

// C2P residual in the unknowns (v^2, rho h W^2) (srmhd.cc:269-295).
struct Residual {
  double D, g, BS, Bsq, Ssq, tau;
  __device__ __forceinline__ void operator()(const double* x, double* fv) const {
    if (x[0] >= 1.0 || x[1] < 0) {
      fv[0] = fv[1] = 1e6;
      return;
    }
    double W = 1 / sqrt(1 - x[0]);
    double rho = D / W;
    double h = x[1] / (rho * W * W);
    double pr = (h - 1) * rho * (g - 1) / g;
    if (pr < 0 || rho < 0 || h < 0 || W < 1) {
      fv[0] = fv[1] = 1e6;
      return;
    }
    fv[0] = (x[1] + Bsq) * (x[1] + Bsq) * x[0] - (2 * x[1] + Bsq) * BS * BS / (x[1] * x[1]) - Ssq;
    fv[1] = x[1] + Bsq - pr - Bsq / (2 * W * W) - BS * BS / (2 * x[1] * x[1]) - D - tau;
  }
};

// Residual arguments of one cell from its conserved state (srmhd.cc:418-442).
__device__ __forceinline__ Residual residual_args(const double* c, double gamma) {
  Residual r;
  r.D = c[0];
  r.g = gamma;
  r.BS = c[5] * c[1] + c[6] * c[2] + c[7] * c[3];
  r.Bsq = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  r.Ssq = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
  r.tau = c[4];
  return r;
}

// Initial guess (v^2, rho h W^2) from the previous primitive state
// (srmhd.cc:438-442).
__device__ __forceinline__ void guess_from_prims(const double* p, double h, double* sol) {
  sol[0] = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  sol[1] = p[0] * h / (1 - sol[0]);
}

// Closed-form primitives and aux from a converged (v^2, rho h W^2)
// (srmhd.cc:509-560).  `p` and `a` receive all 8 / 13 entries.
__device__ __forceinline__ void from_solution(const double* c, const double* sol, double gamma,
                                              double BS, double Bsq, double Ssq, double* p,
                                              double* a) {
  p[5] = c[5];
  p[6] = c[6];
  p[7] = c[7];
  a[10] = BS;
  a[11] = Bsq;
  a[12] = Ssq;
  a[1] = 1 / sqrt(1 - sol[0]);
  p[0] = c[0] / a[1];
  a[0] = sol[1] / (p[0] * a[1] * a[1]);
  p[4] = (a[0] - 1) * p[0] * (gamma - 1) / gamma;
  a[2] = p[4] / (p[0] * (gamma - 1));
  p[1] = (c[5] * a[10] + c[1] * sol[1]) / (sol[1] * (a[11] + sol[1]));
  p[2] = (c[6] * a[10] + c[2] * sol[1]) / (sol[1] * (a[11] + sol[1]));
  p[3] = (c[7] * a[10] + c[3] * sol[1]) / (sol[1] * (a[11] + sol[1]));
  a[9] = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  a[3] = sqrt(a[2] * gamma * (gamma - 1) / a[0]);
  a[4] = a[1] * (c[5] * p[1] + c[6] * p[2] + c[7] * p[3]);
  a[5] = c[5] / a[1] + a[4] * p[1];
  a[6] = c[6] / a[1] + a[4] * p[2];
  a[7] = c[7] / a[1] + a[4] * p[3];
  a[8] = (p[5] * p[5] + p[6] * p[6] + p[7] * p[7] + a[4] * a[4]) / (a[1] * a[1]);
}

// Model::primsToAll for one cell (srmhd.cc:573-673).
__device__ __forceinline__ void prims_to_all(const double* p, double gamma, double* c, double* a) {
  c[5] = p[5];
  c[6] = p[6];
  c[7] = p[7];
  a[11] = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
  c[8] = 0;
  a[9] = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  a[1] = 1.0 / sqrt(1 - a[9]);
  a[4] = a[1] * (p[1] * p[5] + p[2] * p[6] + p[3] * p[7]);
  a[5] = p[5] / a[1] + a[4] * p[1];
  a[6] = p[6] / a[1] + a[4] * p[2];
  a[7] = p[7] / a[1] + a[4] * p[3];
  a[8] = (p[5] * p[5] + p[6] * p[6] + p[7] * p[7] + a[4] * a[4]) / (a[1] * a[1]);
  a[0] = 1 + p[4] / p[0] * (gamma / (gamma - 1));
  a[2] = p[4] / (p[0] * (gamma - 1));
  a[3] = sqrt(a[2] * gamma * (gamma - 1) / a[0]);
  c[0] = p[0] * a[1];
  c[1] = (p[0] * a[0] + a[8]) * a[1] * a[1] * p[1] - a[4] * a[5];
  c[2] = (p[0] * a[0] + a[8]) * a[1] * a[1] * p[2] - a[4] * a[6];
  c[3] = (p[0] * a[0] + a[8]) * a[1] * a[1] * p[3] - a[4] * a[7];
  a[12] = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
  a[10] = p[5] * c[1] + p[6] * c[2] + p[7] * c[3];
  c[4] = (p[0] * a[0] + a[8]) * a[1] * a[1] - (p[4] + a[8] / 2.0) - a[4] * a[4] - c[0];
}

// Divergence-cleaning source (srmhd.cc:215-250): only phi has one.
__device__ __forceinline__ void source(const double* c, double cp, double* s) {
#pragma unroll
  for (int v = 0; v < NC; ++v) s[v] = 0;
  s[8] = -c[8] / (cp * cp);
}

}  // namespace srmhd

// Model trait used by the stencil kernels.
struct SRMHD {
  static constexpr int NC = 9, NP = 8, NA = 13;
  template <typename R, bool LDG = true>
  __device__ __forceinline__ static void load_flux_inputs(const double* __restrict__ cons,
                                                          const double* __restrict__ prims,
                                                          const double* __restrict__ aux,
                                                          long long N, long long cell, R* c, R* p,
                                                          R* a) {
#pragma unroll
    for (int v = 0; v < NC; ++v) c[v] = R(ld_in<LDG>(cons + v * N + cell));
#pragma unroll
    for (int v = 1; v < 8; ++v) p[v] = R(ld_in<LDG>(prims + v * N + cell));
    a[1] = R(ld_in<LDG>(aux + 1 * N + cell));
#pragma unroll
    for (int v = 4; v < 9; ++v) a[v] = R(ld_in<LDG>(aux + v * N + cell));
  }
  template <typename R>
  __device__ __forceinline__ static void flux(const R* c, const R* p, const R* a, int dir, R* f) {
    srmhd::flux<R>(c, p, a, dir, f);
  }
  // The fused tiles' form, which also passes the grid (the Hybrid model's
  // flux depends on the conductivity parameters).
  template <typename R>
  __device__ __forceinline__ static void flux_g(const Grid&, const R* c, const R* p, const R* a,
                                                int dir, R* f) {
    srmhd::flux<R>(c, p, a, dir, f);
  }
  // Model::sourceTerm of one cell in FP64 (srmhd.cc:215-250): S_phi = -phi/cp^2.
  __device__ __forceinline__ static void cell_source(const double* __restrict__ cons,
                                                     const double*, long long N, long long cell,
                                                     double cp, double* s) {
#pragma unroll
    for (int v = 0; v < NC; ++v) s[v] = 0;
    s[8] = -cons[8 * N + cell] / (cp * cp);
  }
};

}  // namespace mth
