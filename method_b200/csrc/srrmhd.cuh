// Resistive special-relativistic MHD (SRRMHD) cell physics.
//
// Variables (Project/CPU/Src/srrmhd.cc:36-62):
//   cons  D, Sx, Sy, Sz, tau, Bx, By, Bz, Ex, Ey, Ez, psi, phi, qch      (14)
//   prims rho, vx, vy, vz, p, Bx, By, Bz, Ex, Ey, Ez                     (11)
//   aux   h, W, e, c, Jx, Jy, Jz, Bsq, Esq, vsq, rhohWsq, vE,
//         Sbarx, Sbary, Sbarz, Sbarsq, tauBar                             (17)
// Expressions keep the reference's association order (see srmhd.cuh).
// Conductivity is the constant Data::sigma (simData.cc:114-119 with
// functionalSigma = false).
#pragma once
#include "common.cuh"
#include "minpack.cuh"

namespace mth {
namespace srrmhd {

constexpr int NC = 14, NP = 11, NA = 17;

// Model::fluxVector (srrmhd.cc:65-192).  In z the reference writes f[2] twice
// and leaves f[3] holding the y-direction value from the previous call; the
// z branch below reproduces that through `f_sz_from_y`.
template <typename R>
__device__ __forceinline__ void flux(const R* c, const R* p, const R* a, int dir, R* f) {
  if (dir == 0) {
    f[0] = c[0] * p[1];
    f[1] = a[10] * p[1] * p[1] + p[4] - c[8] * c[8] - c[5] * c[5] + R(0.5) * (a[7] + a[8]);
    f[2] = a[10] * p[1] * p[2] - c[8] * c[9] - c[5] * c[6];
    f[3] = a[10] * p[1] * p[3] - c[8] * c[10] - c[5] * c[7];
    f[4] = c[1] - c[0] * p[1];
    f[5] = c[12];
    f[6] = -c[10];
    f[7] = c[9];
    f[8] = c[11];
    f[9] = c[7];
    f[10] = -c[6];
    f[11] = c[8];
    f[12] = c[5];
    f[13] = a[4];
  } else if (dir == 1) {
    f[0] = c[0] * p[2];
    f[1] = a[10] * p[1] * p[2] - c[9] * c[8] - c[6] * c[5];
    f[2] = a[10] * p[2] * p[2] + p[4] - c[9] * c[9] - c[6] * c[6] + R(0.5) * (a[7] + a[8]);
    f[3] = a[10] * p[2] * p[3] - c[9] * c[10] - c[6] * c[7];
    f[4] = c[2] - c[0] * p[2];
    f[5] = c[10];
    f[6] = c[12];
    f[7] = -c[8];
    f[8] = -c[7];
    f[9] = c[11];
    f[10] = c[5];
    f[11] = c[9];
    f[12] = c[6];
    f[13] = a[5];
  } else {
    f[0] = c[0] * p[3];
    f[1] = a[10] * p[1] * p[3] - c[10] * c[8] - c[7] * c[5];
    f[2] = a[10] * p[3] * p[3] + p[4] - c[10] * c[10] - c[7] * c[7] + R(0.5) * (a[7] + a[8]);
    f[3] = a[10] * p[2] * p[3] - c[9] * c[10] - c[6] * c[7];  // y-direction Sz flux
    f[4] = c[3] - c[0] * p[3];
    f[5] = -c[9];
    f[6] = c[8];
    f[7] = c[12];
    f[8] = c[6];
    f[9] = -c[5];
    f[10] = c[11];
    f[11] = c[10];
    f[12] = c[7];
    f[13] = a[6];
  }
}

// Source (srrmhd.cc:194-206): Ohm's-law current drives E, charge and
// divergence cleaning.
__device__ __forceinline__ void source(const double* c, const double* a, double cp, double* s) {
  s[0] = s[1] = s[2] = s[3] = s[4] = s[5] = s[6] = s[7] = s[13] = 0.0;
  s[8] = -a[4];
  s[9] = -a[5];
  s[10] = -a[6];
  s[11] = c[13] - c[11] / (cp * cp);
  s[12] = -c[12] / (cp * cp);
}

// 1D residual in Z = rho h W^2 (srrmhd.cc:512-537).
__device__ __forceinline__ double z_residual(double Z, double Ssq, double D, double tauT, double g) {
  double vsq = Ssq / (Z * Z);
  if (vsq >= 1.0 || Z < 0) return 1.0e6;
  double W = 1 / sqrt(1 - vsq);
  double rho = D / W;
  double h = Z / (rho * W * W);
  double p = (g - 1) * (h - rho) / g;
  if (rho < 0 || p < 0 || W < 1 || h < 0) return 1.0e6;
  return (1 - (g - 1) / (W * W * g)) * Z + ((g - 1) / (W * g) - 1) * D - tauT;
}

// Secant iteration on Z (srrmhd.cc:539-581): x1 = x0 + 1e-4, stop when
// |f(x0)| < 1e-12, at most 50 steps; on failure Z becomes the best iterate.
// Returns true when converged; `iters` receives the residual evaluations.
__device__ __forceinline__ bool z_secant(double& Z, double Ssq, double D, double tauT, double g,
                                         int& evals) {
  double x0 = Z, x1 = x0 + 1.0e-4;
  double f0 = z_residual(x0, Ssq, D, tauT, g);
  double f1 = z_residual(x1, Ssq, D, tauT, g);
  evals += 2;
  double bestX = x0, bestF = f0;
  for (int it = 0; it < 50; ++it) {
    if (fabs(f0) < 1.0e-12) {
      Z = x0;
      return true;
    }
    double x2 = x1 - f1 * (x1 - x0) / (f1 - f0);
    x1 = x0;
    x0 = x2;
    f1 = f0;
    f0 = z_residual(x0, Ssq, D, tauT, g);
    ++evals;
    if (fabs(f0) < fabs(bestF)) {
      bestX = x0;
      bestF = f0;
    }
  }
  Z = bestX;
  return false;
}

// Model::getPrimitiveVarsSingleCell (srrmhd.cc:256-312).  `a[10]` carries the
// guess for Z in and the solution out; all of p and a are written.
__device__ __forceinline__ bool c2p_cell(const double* c, double g, double sigma, double* p,
                                         double* a, int& evals) {
  p[5] = c[5]; p[6] = c[6]; p[7] = c[7];
  p[8] = c[8]; p[9] = c[9]; p[10] = c[10];
  a[7] = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  a[8] = c[8] * c[8] + c[9] * c[9] + c[10] * c[10];
  a[12] = c[1] - (c[9] * c[7] - c[10] * c[6]);
  a[13] = c[2] - (c[10] * c[5] - c[8] * c[7]);
  a[14] = c[3] - (c[8] * c[6] - c[9] * c[5]);
  a[15] = a[12] * a[12] + a[13] * a[13] + a[14] * a[14];
  a[16] = c[4] - 0.5 * (a[7] + a[8]);
  if (!z_secant(a[10], a[15], c[0], a[16], g, evals)) return false;
  a[9] = a[15] / (a[10] * a[10]);
  a[1] = 1.0 / sqrt(1 - a[9]);
  p[0] = c[0] / a[1];
  a[0] = a[10] / (p[0] * a[1] * a[1]);
  a[2] = (a[0] - 1) / g;
  a[3] = sqrt((a[2] * g * (g - 1)) / a[0]);
  p[4] = p[0] * a[2] * (g - 1);
  p[1] = a[12] / a[10];
  p[2] = a[13] / a[10];
  p[3] = a[14] / a[10];
  a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
  a[4] = c[13] * p[1] + a[1] * sigma * (c[8] + (p[2] * c[7] - p[3] * c[6]) - a[11] * p[1]);
  a[5] = c[13] * p[2] + a[1] * sigma * (c[9] + (p[3] * c[5] - p[1] * c[7]) - a[11] * p[2]);
  a[6] = c[13] * p[3] + a[1] * sigma * (c[10] + (p[1] * c[6] - p[2] * c[5]) - a[11] * p[3]);
  return true;
}

// Per-cell part of SRRMHD::primsToAll (srrmhd.cc:358-510).  `qfd` tells
// whether the 4th-order charge-density stencil applies at this cell and
// `divE` is its value.
__device__ __forceinline__ void prims_to_all(const double* p, double g, double sigma0,
                                             double sigma_exp, int functional, bool qfd,
                                             double divE, double* c, double* a) {
  c[11] = c[12] = 0.0;
  c[5] = p[5]; c[6] = p[6]; c[7] = p[7];
  c[8] = p[8]; c[9] = p[9]; c[10] = p[10];
  a[7] = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
  a[8] = p[8] * p[8] + p[9] * p[9] + p[10] * p[10];
  a[9] = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
  a[1] = 1.0 / sqrt(1 - a[9]);
  c[0] = p[0] * a[1];
  a[2] = p[4] / (p[0] * (g - 1));
  a[0] = 1 + a[2] * g;
  a[3] = sqrt((a[2] * g * (g - 1)) / a[0]);
  a[10] = p[0] * a[0] * a[1] * a[1];
  const double sigma = sigma_of(sigma0, sigma_exp, functional, c[0]);  // srrmhd.cc:410
  if (qfd) {
    c[13] = divE;
    a[4] = c[13] * p[1] + a[1] * sigma * (c[8] + p[2] * c[7] - p[3] * c[6] - a[11] * p[1]);
    a[5] = c[13] * p[2] + a[1] * sigma * (c[9] + p[3] * c[5] - p[1] * c[7] - a[11] * p[2]);
    a[6] = c[13] * p[3] + a[1] * sigma * (c[10] + p[1] * c[6] - p[2] * c[5] - a[11] * p[3]);
  } else {
    c[13] = a[4] = a[5] = a[6] = 0.0;
  }
  c[1] = a[10] * p[1] + c[9] * c[7] - c[10] * c[6];
  c[2] = a[10] * p[2] + c[10] * c[5] - c[8] * c[7];
  c[3] = a[10] * p[3] + c[8] * c[6] - c[9] * c[5];
  c[4] = a[10] - p[4] + 0.5 * (a[7] + a[8]) - c[0];
  a[12] = a[10] * p[1];
  a[13] = a[10] * p[2];
  a[14] = a[10] * p[3];
  a[15] = a[12] * a[12] + a[13] * a[13] + a[14] * a[14];
  a[16] = a[10] - p[4] - c[0];
}

// Residuals of the two implicit SSP2(222) stages (SSP2.cc:194-264).  The
// secant guess `Z` persists across evaluations exactly like the reference's
// args.aux[10], so the chain of guesses follows hybrd's evaluation order.
// Residual of one implicit IMEX stage for one cell.  `stage` selects the
// form: 1, 2 = SSP2(222) stages 1, 2 (SSP2.cc:194-264; SSP3(332) stages 1, 2
// use the same expressions, SSP3.cc:237-314); 3 = SSP3(332) stage 3
// (SSP3.cc:335-355); 4, 5, 6 = SSP2(322) stages 1-3 (SSP2322.cc:262-383).
struct ImexResidual {
  const double* u;        // U^n of the cell (14)
  const double* flux1;    // forms 2, 3
  const double* source1;  // forms 2, 3, 5
  const double* flux2;    // forms 3, 6
  const double* source2;  // form 6
  double dt, gam, om2gam, hmgam, g, sigma, cp;
  double sigma_exp;  // functional conductivity sigma * D^sigma_exp when `functional`
  int functional;
  double Z;
  int stage;
  int evals;
  __device__ __forceinline__ void operator()(const double* x, double* fv) {
    double p[NP], a[NA], s[NC];
    a[10] = Z;
    bool ok = c2p_cell(x, g, sigma_of(sigma, sigma_exp, functional, x[0]), p, a, evals);
    Z = a[10];
    if (!ok) {
#pragma unroll
      for (int i = 0; i < NC; ++i) fv[i] = 1.0e6;
      return;
    }
    source(x, a, cp, s);
    if (stage == 1) {
#pragma unroll
      for (int i = 0; i < NC; ++i) fv[i] = x[i] - u[i] - dt * gam * s[i];
    } else if (stage == 2) {
#pragma unroll
      for (int i = 0; i < NC; ++i)
        fv[i] = x[i] - u[i] + dt * (flux1[i] - om2gam * source1[i] - gam * s[i]);
    } else if (stage == 3) {
#pragma unroll
      for (int i = 0; i < NC; ++i)
        fv[i] = x[i] - u[i] + dt * (flux1[i] + flux2[i]) / 4.0 -
                dt * (hmgam * source1[i] + gam * s[i]);
    } else if (stage == 4) {
#pragma unroll
      for (int i = 0; i < NC; ++i) fv[i] = x[i] - u[i] - dt * 0.5 * s[i];
    } else if (stage == 5) {
#pragma unroll
      for (int i = 0; i < NC; ++i) fv[i] = x[i] - u[i] + dt * 0.5 * (source1[i] - s[i]);
    } else {
#pragma unroll
      for (int i = 0; i < NC; ++i)
        fv[i] = x[i] - u[i] + dt * (flux2[i] - 0.5 * source2[i] - 0.5 * s[i]);
    }
  }
};

}  // namespace srrmhd

struct SRRMHD {
  static constexpr int NC = 14, NP = 11, NA = 17;
  template <typename R, bool LDG = true>
  __device__ __forceinline__ static void load_flux_inputs(const double* __restrict__ cons,
                                                          const double* __restrict__ prims,
                                                          const double* __restrict__ aux,
                                                          long long N, long long cell, R* c, R* p,
                                                          R* a) {
#pragma unroll
    for (int v = 0; v < NC; ++v) c[v] = R(ld_in<LDG>(cons + v * N + cell));
#pragma unroll
    for (int v = 1; v < 5; ++v) p[v] = R(ld_in<LDG>(prims + v * N + cell));
#pragma unroll
    for (int v = 4; v < 9; ++v) a[v] = R(ld_in<LDG>(aux + v * N + cell));
    a[10] = R(ld_in<LDG>(aux + 10 * N + cell));
  }
  template <typename R>
  __device__ __forceinline__ static void flux(const R* c, const R* p, const R* a, int dir, R* f) {
    srrmhd::flux<R>(c, p, a, dir, f);
  }
  // The fused tiles' form, which also passes the grid (the Hybrid model's
  // flux depends on the conductivity parameters).
  template <typename R>
  __device__ __forceinline__ static void flux_g(const Grid&, const R* c, const R* p, const R* a,
                                                int dir, R* f) {
    srrmhd::flux<R>(c, p, a, dir, f);
  }
  // Model::sourceTerm of one cell in FP64 (srrmhd.cc:194-206): reads cons
  // 11-13 and aux 4-6 only.
  __device__ __forceinline__ static void cell_source(const double* __restrict__ cons,
                                                     const double* __restrict__ aux, long long N,
                                                     long long cell, double cp, double* s) {
    double c[NC], a[NA];
#pragma unroll
    for (int v = 11; v < 14; ++v) c[v] = cons[v * N + cell];
#pragma unroll
    for (int v = 4; v < 7; ++v) a[v] = aux[v * N + cell];
    srrmhd::source(c, a, cp, s);
  }
};

cudaError_t launch_prims_to_all_srrmhd(const Grid& g, const double* prims, double* cons,
                                       double* aux, cudaStream_t st);

}  // namespace mth
