// Mixed-precision ("chosen") form kernels.  FMA contraction is allowed here.
//
//  * FP32 flux / Lax-Friedrichs split / WENO (the fused 2D stage kernel
//    instantiated with R = float); the conserved-state update stays FP64.
//  * FP64 primitive recovery by a one-dimensional Newton iteration in
//    Z = rho h W^2.  For SRMHD the reference's 2x2 system (srmhd.cc:269-295)
//    is reduced to 1D: its first equation gives v^2(Z) in closed form,
//        v^2 = (S^2 Z^2 + (2Z + B^2)(B.S)^2) / (Z^2 (Z + B^2)^2),
//    and Newton runs on the second.  For SRRMHD the reference's secant
//    residual (srrmhd.cc:512-537) is already 1D and gets its analytic
//    derivative.  The guess comes from the previous state or the guess
//    network; a cell whose Newton iteration does not converge falls back to
//    the previous-state guess and then to the reference Powell-hybrid.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "ensemble.h"
#include "fvs2d.cuh"
#include "hybrid.cuh"
#include "launch.h"
#include "minpack.cuh"
#include "mixed.h"
#include "srmhd.cuh"
#include "srrmhd.cuh"

namespace mth {

namespace {

// Newton in Z for SRMHD, safeguarded by a bracket.  v^2(Z) above is strictly
// decreasing for Z > 0, so "v^2 >= 1 or g < 0" marks the left of the root
// and g > 0 its right; a Newton step that leaves the bracket (or a zero or
// negative slope) is replaced by bisection (geometric while the bracket spans
// decades).  On success Z and vsq hold the root.
//
// One division and one reciprocal square root per evaluation: 1/(Z^2 (Z +
// B^2)^2) also gives 1/Z^2 and 1/Z.
__device__ __forceinline__ bool srmhd_g(double Z, double D, double tau, double BS2, double Bsq,
                                        double Ssq, double k, double& gv, double& dg,
                                        double& v2) {
  const double Z2 = Z * Z, ZB = Z + Bsq;
  const double iDn = 1 / (Z2 * ZB * ZB);
  v2 = fma(Ssq, Z2, (2 * Z + Bsq) * BS2) * iDn;
  if (!(v2 < 1.0)) return false;
  const double iZ2 = iDn * ZB * ZB, iZ = iZ2 * Z;
  const double om = 1 - v2;
  const double is = rsqrt(om), s = om * is;
  const double p = k * (Z * om - D * s);
  gv = Z + Bsq - p - 0.5 * Bsq * om - 0.5 * BS2 * iZ2 - D - tau;
  const double dv2 = (fma(2 * Ssq, Z, 2 * BS2) - v2 * (2 * Z * ZB * (2 * Z + Bsq))) * iDn;
  const double dp = k * (om - Z * dv2 + 0.5 * D * dv2 * is);
  dg = 1 - dp + 0.5 * Bsq * dv2 + BS2 * iZ2 * iZ;
  return true;
}

// The right end of the bracket is searched for only when a step needs it (an
// unusable guess, v^2 >= 1, a step out of the bracket, a non-positive slope);
// a Newton run that converges from a good guess never evaluates it.
__device__ __forceinline__ bool newton_srmhd(double D, double tau, double BS2, double Bsq,
                                             double Ssq, double g, double& Z, double& vsq,
                                             int& iters) {
  const double k = (g - 1) / g;
  double gv, dg, v2;
  double lo = 0.0, hi = 0.0;
  bool have_hi = false;
  auto find_hi = [&]() {
    if (have_hi) return;
    // g(Z) ~ (1 - k) Z for large Z
    hi = fmax(g * (tau + D + Bsq), 1e-300);
    for (int q = 0; q < 64; ++q) {
      double gh, dh, vh;
      if (srmhd_g(hi, D, tau, BS2, Bsq, Ssq, k, gh, dh, vh) && gh > 0) break;
      hi *= 2;
    }
    have_hi = true;
  };
  double Zc = Z;
  if (!(Z > 0 && isfinite(Z))) {
    find_hi();
    Zc = 0.5 * hi;
  }
  for (int it = 0; it < 100; ++it) {
    ++iters;
    double Zn;
    if (!srmhd_g(Zc, D, tau, BS2, Bsq, Ssq, k, gv, dg, v2)) {
      lo = Zc;  // v^2 >= 1: left of the root
      find_hi();
      Zn = lo > 0 ? sqrt(lo * hi) : 0.5 * hi;
    } else {
      if (gv == 0) {
        Z = Zc;
        vsq = v2;
        break;
      }
      if (gv < 0) {
        lo = Zc;
      } else {
        hi = Zc;
        have_hi = true;
      }
      Zn = Zc - gv / dg;
      if (!(dg > 0) || !(Zn > lo && (!have_hi || Zn < hi))) {
        find_hi();
        Zn = (lo > 0 && hi > 4 * lo) ? sqrt(lo * hi) : 0.5 * (lo + hi);
      }
    }
    if (fabs(Zn - Zc) <= 1e-14 * Zn || (have_hi && hi - lo <= 1e-15 * hi)) {
      Zc = Zn;
      if (!srmhd_g(Zc, D, tau, BS2, Bsq, Ssq, k, gv, dg, v2)) return false;
      Z = Zc;
      vsq = v2;
      break;
    }
    Zc = Zn;
    if (it == 99) return false;
  }
  const double rn = D * sqrt(1 - vsq);
  const double pn = k * (Z * (1 - vsq) - rn);
  return pn >= 0 && rn >= 0;
}

// Model primitives and aux from a converged (v^2, Z), the quantities of
// srmhd::from_solution (srmhd.cc:509-560) with reciprocals in place of most
// divisions: W = 1/sqrt(1 - v^2), rho = D/W, h = Z/(rho W^2) = Z/(D W),
// e = (h - 1)/gamma, v = (B (B.S) + S Z)/(Z (B^2 + Z)), c_s^2 = (h - 1)(gamma - 1)/h.
__device__ __forceinline__ void from_solution_fast(const double* c, const double* sol,
                                                   double gamma, double BS, double Bsq,
                                                   double Ssq, double* p, double* a) {
  p[5] = c[5];
  p[6] = c[6];
  p[7] = c[7];
  a[10] = BS;
  a[11] = Bsq;
  a[12] = Ssq;
  const double om = 1 - sol[0];
  const double W = rsqrt(om), iW = om * W;
  a[1] = W;
  p[0] = c[0] * iW;
  a[0] = sol[1] * iW / c[0];
  const double ig = 1 / gamma;
  p[4] = (a[0] - 1) * p[0] * ((gamma - 1) * ig);
  a[2] = (a[0] - 1) * ig;
  const double iq = 1 / (sol[1] * (Bsq + sol[1]));
  p[1] = fma(c[5], BS, c[1] * sol[1]) * iq;
  p[2] = fma(c[6], BS, c[2] * sol[1]) * iq;
  p[3] = fma(c[7], BS, c[3] * sol[1]) * iq;
  a[9] = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
  a[3] = sqrt((a[0] - 1) * (gamma - 1) / a[0]);
  a[4] = W * (c[5] * p[1] + c[6] * p[2] + c[7] * p[3]);
  a[5] = fma(c[5], iW, a[4] * p[1]);
  a[6] = fma(c[6], iW, a[4] * p[2]);
  a[7] = fma(c[7], iW, a[4] * p[3]);
  a[8] = (Bsq + a[4] * a[4]) * om;
}

// Newton in Z for SRRMHD's residual (srrmhd.cc:512-537).
__device__ __forceinline__ bool newton_srrmhd(double Sb2, double D, double tauT, double g,
                                              double& Z, int& iters) {
  const double k = (g - 1) / g;
  double Zc = Z;
  if (!(Zc > 0) || !isfinite(Zc)) return false;
  for (int it = 0; it < 60; ++it) {
    ++iters;
    const double Z2 = Zc * Zc;
    if (!(Sb2 < Z2)) {
      Zc = 2 * sqrt(Sb2) + 1e-300;
      continue;
    }
    // one division and one reciprocal square root per step
    const double iZ = 1 / Zc, Sz = Sb2 * iZ, q = Sz * iZ;
    const double is = rsqrt(1 - q), s = (1 - q) * is;
    const double r = Zc - k * (Zc - Sz) + (k * s - 1) * D - tauT;
    const double dr = 1 - k * (1 + q) + k * D * q * iZ * is;
    double Zn = Zc - r / dr;
    if (!(Zn > 0) || !isfinite(Zn)) Zn = 0.5 * Zc;
    if (fabs(Zn - Zc) <= 1e-13 * Zn) {
      if (!(Sb2 < Zn * Zn)) return false;
      Z = Zn;
      return true;
    }
    Zc = Zn;
  }
  return false;
}

struct NewtonTally {
  long long its = 0, fb_prev = 0, fb_hybrd = 0, bad = 0;
};

struct HybrdOut {
  double x0, x1;
  int nfev, info;
};

// The Powell-hybrid fallback of the SRMHD Newton recovery (srmhd.cc's own
// method, from the previous state's guess), out of line: the Newton path's
// registers are then allocated without it, as no cell of the measured
// workloads takes it.
__device__ __noinline__ HybrdOut hybrd2_fallback(srmhd::Residual R, double x0, double x1) {
  double x[2] = {x0, x1}, fv[2];
  const HybrdResult res = Hybrd<2>::solve(R, x, fv, 1.49011612e-7);
  return {x[0], x[1], res.nfev, res.info};
}

// Mixed-form SRMHD recovery of one cell (Newton in Z, fallbacks).
// LEAN writes only what FVS::F reads back (prims 1-7; aux 1 and 4-8) and no
// solution: the recovered RK2 predictor state feeds nothing but the
// corrector's flux, so the other values would be dead stores.
template <bool LEAN>
__device__ __forceinline__ void c2p_srmhd_newton_cell(const Grid& g, long long cell,
                                                      int guess_mode,
                                                      const double* __restrict__ cons,
                                                      const double* prims_guess,
                                                      const double* aux_guess, double* prims,
                                                      double* aux, double* __restrict__ solution,
                                                      const double* __restrict__ zguess,
                                                      NewtonTally& tl) {
  const long long N = g.Ntot;
  double c[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
  srmhd::Residual R = srmhd::residual_args(c, g.gamma);
  const double BS2 = R.BS * R.BS;
  double pg[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) pg[v] = prims_guess[v * N + cell];
  double prev[2];
  srmhd::guess_from_prims(pg, aux_guess[cell], prev);
  double Z = prev[1], vsq = prev[0];
  int it = 0;
  bool ok = false;
  if (guess_mode == 1 && zguess) {
    Z = zguess[cell];
    ok = newton_srmhd(R.D, R.tau, BS2, R.Bsq, R.Ssq, g.gamma, Z, vsq, it);
    if (!ok) {
      tl.fb_prev += 1;
      Z = prev[1];
    }
  }
  if (!ok) ok = newton_srmhd(R.D, R.tau, BS2, R.Bsq, R.Ssq, g.gamma, Z, vsq, it);
  double x[2] = {vsq, Z};
  if (!ok) {
    tl.fb_hybrd += 1;
    const HybrdOut res = hybrd2_fallback(R, prev[0], prev[1]);
    x[0] = res.x0;
    x[1] = res.x1;
    it += res.nfev;
    if (res.info != 1) tl.bad += 1;
  }
  tl.its += it;
  double p[8], a[13];
  from_solution_fast(c, x, g.gamma, R.BS, R.Bsq, R.Ssq, p, a);
  if constexpr (LEAN) {
#pragma unroll
    for (int v = 1; v < 8; ++v) prims[v * N + cell] = p[v];
    aux[N + cell] = a[1];
#pragma unroll
    for (int v = 4; v < 9; ++v) aux[v * N + cell] = a[v];
  } else {
    solution[cell] = x[0];
    solution[N + cell] = x[1];
#pragma unroll
    for (int v = 0; v < 8; ++v) prims[v * N + cell] = p[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) aux[v * N + cell] = a[v];
  }
}

__device__ __forceinline__ void tally_flush(NewtonTally tl, bool active, long long* counters) {
  const unsigned mask = __ballot_sync(0xffffffffu, active);
  for (int o = 16; o > 0; o >>= 1) {
    tl.its += __shfl_down_sync(0xffffffffu, tl.its, o);
    tl.fb_prev += __shfl_down_sync(0xffffffffu, tl.fb_prev, o);
    tl.fb_hybrd += __shfl_down_sync(0xffffffffu, tl.fb_hybrd, o);
    tl.bad += __shfl_down_sync(0xffffffffu, tl.bad, o);
  }
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&counters[1], (unsigned long long)tl.its);
    if (tl.bad) {
      atomicAdd((unsigned long long*)&counters[2], (unsigned long long)tl.bad);
    }
    if (tl.fb_prev) atomicAdd((unsigned long long*)&counters[8], (unsigned long long)tl.fb_prev);
    if (tl.fb_hybrd) atomicAdd((unsigned long long*)&counters[9], (unsigned long long)tl.fb_hybrd);
  }
}

// Minimum resident CTAs the register allocation of the solver kernels is
// sized for.  Capping registers doubles the warps that hide the FP64 latency
// of the Newton iterations; the values that no longer fit go to local memory,
// and the net is faster: OT 1024^2 0.107 -> 0.090 ms per C2P launch, SSP2
// 512x1024 stages 5-15%.  With the Powell-hybrid fallback out of line the
// SRMHD Newton kernels spill 80 bytes instead of 700 (0.083 -> 0.076 ms).
constexpr int kNewtonMinBlocks = 8;     // 128 threads x 8 CTAs -> 64 registers

template <bool LEAN>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_c2p_newton_srmhd(Grid g, int guess_mode, const double* __restrict__ cons,
                       const double* prims_guess, const double* aux_guess, double* prims,
                       double* aux, double* __restrict__ solution, C2PWork w,
                       const double* __restrict__ zguess, long long t0, long long t_end) {
  const long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  NewtonTally tl;
  if (t < t_end) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    c2p_srmhd_newton_cell<LEAN>(g, cell_id(g, i, j, k), guess_mode, cons, prims_guess, aux_guess,
                                prims, aux, solution, zguess, tl);
  }
  tally_flush(tl, t < t_end, w.counters);
}

// Mixed-form SRRMHD recovery of one cell (Newton in Z, secant fallback).
// LEAN writes only what the stage's flux, source and next implicit solve read
// back (prims 1-4; aux 4-8 and 10): the recovered SSP2 stage states (and the
// RK2 predictor state) feed nothing else.
template <bool LEAN>
__device__ __forceinline__ void c2p_srrmhd_newton_cell(const Grid& g, long long cell,
                                                       const double* __restrict__ cons,
                                                       const double* aux_guess, double* prims,
                                                       double* aux, NewtonTally& tl,
                                                       long long* counters,
                                                       const double* zseed = nullptr) {
  const long long N = g.Ntot;
  double c[14], p[11], a[17];
#pragma unroll
  for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
  const double gm = g.gamma;
  p[5] = c[5]; p[6] = c[6]; p[7] = c[7];
  p[8] = c[8]; p[9] = c[9]; p[10] = c[10];
  a[7] = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  a[8] = c[8] * c[8] + c[9] * c[9] + c[10] * c[10];
  a[12] = c[1] - (c[9] * c[7] - c[10] * c[6]);
  a[13] = c[2] - (c[10] * c[5] - c[8] * c[7]);
  a[14] = c[3] - (c[8] * c[6] - c[9] * c[5]);
  a[15] = a[12] * a[12] + a[13] * a[13] + a[14] * a[14];
  a[16] = c[4] - 0.5 * (a[7] + a[8]);
  double Z = zseed ? zseed[cell] : aux_guess[10 * N + cell];
  int it = 0;
  bool ok = newton_srrmhd(a[15], c[0], a[16], gm, Z, it);
  if (!ok && zseed) {  // the network's Z failed: the previous state's, as without it
    tl.fb_prev += 1;
    Z = aux_guess[10 * N + cell];
    ok = newton_srrmhd(a[15], c[0], a[16], gm, Z, it);
  }
  bool bad = false;
  if (!ok) {
    tl.fb_hybrd += 1;
    Z = aux_guess[10 * N + cell];
    ok = srrmhd::z_secant(Z, a[15], c[0], a[16], gm, it);
    if (!ok) bad = true;
  }
  tl.its += it;
  // srrmhd.cc:283-301 with reciprocals: W = 1/sqrt(1 - v^2), rho = D/W,
  // h = Z/(rho W^2) = Z/(D W), c_s^2 = e gamma (gamma - 1)/h = (h - 1)(gamma - 1)/h
  a[10] = Z;
  const double iZ = 1 / Z;
  a[9] = a[15] * iZ * iZ;
  const double om = 1 - a[9];
  a[1] = rsqrt(om);
  const double iW = om * a[1];
  p[0] = c[0] * iW;
  a[0] = Z * iW / c[0];
  a[2] = (a[0] - 1) / gm;
  a[3] = sqrt((a[0] - 1) * (gm - 1) / a[0]);
  p[4] = p[0] * a[2] * (gm - 1);
  p[1] = a[12] * iZ;
  p[2] = a[13] * iZ;
  p[3] = a[14] * iZ;
  a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
  const double sg = sigma_of(g, c[0]);
  a[4] = c[13] * p[1] + a[1] * sg * (c[8] + (p[2] * c[7] - p[3] * c[6]) - a[11] * p[1]);
  a[5] = c[13] * p[2] + a[1] * sg * (c[9] + (p[3] * c[5] - p[1] * c[7]) - a[11] * p[2]);
  a[6] = c[13] * p[3] + a[1] * sg * (c[10] + (p[1] * c[6] - p[2] * c[5]) - a[11] * p[3]);
  if (bad) {
    tl.bad += 1;
    atomicOr((unsigned long long*)&counters[3], (unsigned long long)ERR_C2P);
  } else if constexpr (LEAN) {
#pragma unroll
    for (int v = 1; v < 5; ++v) prims[v * N + cell] = p[v];
#pragma unroll
    for (int v = 4; v < 9; ++v) aux[v * N + cell] = a[v];
    aux[10 * N + cell] = a[10];
  } else {
#pragma unroll
    for (int v = 0; v < 11; ++v) prims[v * N + cell] = p[v];
#pragma unroll
    for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
  }
}

// Mixed-form recovery of the Hybrid model (hybrid.cc:354-436): SRRMHD's
// Newton recovery where the conductivity is below sigmaCrossOver, else
// SRMHD's Newton recovery of the ideal variables (Powell-hybrid fallback)
// started from the previous velocity and enthalpy, converted back to the
// resistive prims and aux as Hybrid::getPrimitiveVarsSingleCell does.  A
// cell neither solver recovers raises ERR_C2P (the reference throws).
__global__ void __launch_bounds__(128)
    k_c2p_newton_hybrid(Grid g, const double* __restrict__ cons, const double* prims_guess,
                        const double* aux_guess, double* prims, double* aux, C2PWork w) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = t < n_interior(g);
  NewtonTally tl;
  if (active) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long N = g.Ntot, cell = cell_id(g, i, j, k);
    const double D = cons[cell];
    if (sigma_of(g, D) < g.sigma_cross) {
      c2p_srrmhd_newton_cell<false>(g, cell, cons, aux_guess, prims, aux, tl, w.counters);
    } else {
      double c[14];
#pragma unroll
      for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
      double ic[9];
#pragma unroll
      for (int v = 0; v < 8; ++v) ic[v] = c[v];
      ic[8] = c[12];
      srmhd::Residual R = srmhd::residual_args(ic, g.gamma);
      const double BS2 = R.BS * R.BS;
      double pg[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) pg[v] = prims_guess[v * N + cell];
      double prev[2];
      srmhd::guess_from_prims(pg, aux_guess[cell], prev);
      double Z = prev[1], vsq = prev[0];
      int it = 0;
      bool ok = newton_srmhd(R.D, R.tau, BS2, R.Bsq, R.Ssq, g.gamma, Z, vsq, it);
      double x[2] = {vsq, Z};
      if (!ok) {
        tl.fb_hybrd += 1;
        const HybrdOut res = hybrd2_fallback(R, prev[0], prev[1]);
        x[0] = res.x0;
        x[1] = res.x1;
        it += res.nfev;
        ok = res.info == 1;
      }
      tl.its += it;
      if (!ok) {
        tl.bad += 1;
        atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_C2P);
      } else {
        double ip[8], ia[13], p[11], a[17];
        from_solution_fast(ic, x, g.gamma, R.BS, R.Bsq, R.Ssq, ip, ia);
#pragma unroll
        for (int v = 0; v < 8; ++v) p[v] = ip[v];
        p[8] = c[8]; p[9] = c[9]; p[10] = c[10];
        a[0] = ia[0]; a[1] = ia[1]; a[2] = ia[2]; a[3] = ia[3];
        a[4] = 0; a[5] = 0; a[6] = 0; a[7] = ia[11];
        a[8] = c[8] * c[8] + c[9] * c[9] + c[10] * c[10];
        a[9] = ia[9];
        a[10] = p[0] * a[0] * a[1] * a[1];
        a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
        a[12] = a[10] * p[1];
        a[13] = a[10] * p[2];
        a[14] = a[10] * p[3];
        a[15] = a[12] * a[12] + a[13] * a[13] + a[14] * a[14];
        a[16] = a[10] - p[4] - c[0];
#pragma unroll
        for (int v = 0; v < 11; ++v) prims[v * N + cell] = p[v];
#pragma unroll
        for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
      }
    }
  }
  tally_flush(tl, active, w.counters);
}

template <bool LEAN>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_c2p_newton_srrmhd(Grid g, const double* __restrict__ cons, const double* aux_guess,
                        double* prims, double* aux, C2PWork w, const double* zseed, long long t0,
                        long long t_end) {
  const long long t = t0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  NewtonTally tl;
  if (t < t_end) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    c2p_srrmhd_newton_cell<LEAN>(g, cell_id(g, i, j, k), cons, aux_guess, prims, aux, tl,
                                 w.counters, zseed);
  }
  tally_flush(tl, t < t_end, w.counters);
}

// Batched SRMHD primitive recovery for independent cells.
__global__ void __launch_bounds__(128)
    k_c2p_batch_srmhd(long long n, double gamma, int method, int guess,
                      const double* __restrict__ cons, double* prims, double* aux,
                      const double* __restrict__ zguess, long long* counters) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long its = 0, bad = 0, fb = 0;
  if (q < n) {
    double c[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) c[v] = cons[v * n + q];
    srmhd::Residual R = srmhd::residual_args(c, gamma);
    double prev[2];
    {
      double pg[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) pg[v] = prims[v * n + q];
      srmhd::guess_from_prims(pg, aux[q], prev);
    }
    double x0[2];
    if (guess == 1) {
      x0[0] = zguess[n + q];
      x0[1] = zguess[q];
    } else if (guess == 2) {
      const double E = R.tau + R.D;
      x0[1] = fmax(E, sqrt(R.Ssq) * 1.0000001);
      x0[0] = fmin(R.Ssq / (x0[1] * x0[1]), 0.999999);
    } else {
      x0[0] = prev[0];
      x0[1] = prev[1];
    }
    double x[2] = {x0[0], x0[1]}, fv[2];
    int it = 0;
    bool ok = false;
    if (method == 1) {
      double Z = x0[1], vsq = x0[0];
      ok = newton_srmhd(R.D, R.tau, R.BS * R.BS, R.Bsq, R.Ssq, gamma, Z, vsq, it);
      if (!ok && guess != 0) {
        fb = 1;
        Z = prev[1];
        ok = newton_srmhd(R.D, R.tau, R.BS * R.BS, R.Bsq, R.Ssq, gamma, Z, vsq, it);
      }
      if (ok) {
        x[0] = vsq;
        x[1] = Z;
      } else {
        fb = 1;
        x[0] = prev[0];
        x[1] = prev[1];
        HybrdResult r = Hybrd<2>::solve(R, x, fv, 1.49011612e-7);
        it += r.nfev;
        ok = r.info == 1;
      }
    } else {
      HybrdResult r = Hybrd<2>::solve(R, x, fv, 1.49011612e-7);
      it = r.nfev;
      ok = r.info == 1;
    }
    bad = ok ? 0 : 1;
    its = it;
    double p[8], a[13];
    srmhd::from_solution(c, x, gamma, R.BS, R.Bsq, R.Ssq, p, a);
#pragma unroll
    for (int v = 0; v < 8; ++v) prims[v * n + q] = p[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) aux[v * n + q] = a[v];
  }
  for (int o = 16; o > 0; o >>= 1) {
    its += __shfl_down_sync(0xffffffffu, its, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
    fb += __shfl_down_sync(0xffffffffu, fb, o);
  }
  const unsigned mask = __ballot_sync(0xffffffffu, q < n);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&counters[1], (unsigned long long)its);
    if (bad) atomicAdd((unsigned long long*)&counters[2], (unsigned long long)bad);
    if (fb) atomicAdd((unsigned long long*)&counters[3], (unsigned long long)fb);
  }
}

// SSP2 implicit stage of the mixed form (SRRMHD).  Both stages solve
//   x = c + a S(x),  a = dt * gam,
// with c = U^n (stage 1) or U^n - dt (flux1 - om2gam source1) (stage 2),
// the residuals of SSP2.cc:194-264 rearranged.  Only E, psi, phi have
// sources (srrmhd.cc:194-206): phi and psi are linear and solved in closed
// form, charge and the other variables equal c, and E solves
//   R(E) = E - c_E + a J(E),  J = q v + W sigma (E + v x B - (v.E) v),
// by Newton steps with the Jacobian of the stiff term at frozen velocity,
// (1 + a W sigma) I - a W sigma v v^T, inverted by Sherman-Morrison.  Every
// residual runs the 1D Newton primitive recovery in Z.  A cell that does not
// converge is queued for the reference Powell-hybrid stage kernel.
constexpr double kGam = 0.2928932188134525;
constexpr double kOm2Gam = 0.4142135623730950;
constexpr double kHmGam = 0.2071067811865475;

__device__ __forceinline__ bool srrmhd_prims_newton(const double* x, double g, double& Z,
                                                    double* v, double& W, int& its) {
  const double Sb0 = x[1] - (x[9] * x[7] - x[10] * x[6]);
  const double Sb1 = x[2] - (x[10] * x[5] - x[8] * x[7]);
  const double Sb2 = x[3] - (x[8] * x[6] - x[9] * x[5]);
  const double Sbsq = Sb0 * Sb0 + Sb1 * Sb1 + Sb2 * Sb2;
  const double Bsq = x[5] * x[5] + x[6] * x[6] + x[7] * x[7];
  const double Esq = x[8] * x[8] + x[9] * x[9] + x[10] * x[10];
  const double tauB = x[4] - 0.5 * (Bsq + Esq);
  if (!newton_srrmhd(Sbsq, x[0], tauB, g, Z, its)) return false;
  const double iZ = 1 / Z;
  const double vsq = Sbsq * iZ * iZ;
  W = rsqrt(1 - vsq);
  v[0] = Sb0 * iZ;
  v[1] = Sb1 * iZ;
  v[2] = Sb2 * iZ;
  return true;
}

// One cell of the mixed-form implicit stage; returns false when Newton on E
// did not converge (out then holds the last iterate).
// One implicit stage x = c + a S(x) in the mixed form.  FORM selects c and a
// from the stage's residual (srrmhd::ImexResidual forms): 1, 2 = SSP2 stages
// and SSP3 stages 1, 2 (a = dt gam); 3 = SSP3 stage 3,
// c = U - dt (F1 + F2) / 4 + dt hmgam S1; 4, 5, 6 = SSP2322 stages (a = dt / 2)
// with c = U, U - dt S1 / 2, U - dt (F2 - S2 / 2).  psi and phi have closed
// forms; E is Newton-iterated with the stiff Jacobian inverted by
// Sherman-Morrison (v frozen per step).  The final Z goes to zout[10] when
// zout is given (the seed of the stage's recovery).
template <int FORM>
__device__ __forceinline__ bool imex_fast_form(const Grid& g, long long cell,
                                               const double* __restrict__ cons,
                                               const double* __restrict__ aux_guess,
                                               const double* __restrict__ flux1,
                                               const double* __restrict__ flux2,
                                               const double* __restrict__ source1,
                                               const double* __restrict__ source2,
                                               double* __restrict__ out, double* zout, double dt,
                                               int& its, const double* zseed = nullptr) {
  const long long N = g.Ntot;
  double c[14], x[14];
#pragma unroll
  for (int v = 0; v < 14; ++v) {
    const long long o = v * N + cell;
    const double u = cons[o];
    if (FORM == 1 || FORM == 4) c[v] = u;
    else if (FORM == 2) c[v] = u - dt * (flux1[o] - kOm2Gam * source1[o]);
    else if (FORM == 3) c[v] = u - dt * (flux1[o] + flux2[o]) / 4.0 + dt * kHmGam * source1[o];
    else if (FORM == 5) c[v] = u - 0.5 * dt * source1[o];
    else c[v] = u - dt * (flux2[o] - 0.5 * source2[o]);
    x[v] = c[v];
  }
  // D has no source: x[0] = c[0] throughout, so the conductivity is fixed per cell
  const double a = FORM <= 3 ? dt * kGam : 0.5 * dt, cp2 = g.cp * g.cp, sg = sigma_of(g, c[0]);
  x[12] = c[12] / (1 + a / cp2);
  x[11] = (c[11] + a * c[13]) / (1 + a / cp2);
  // the inner recovery's Z: the network's guess for the stage's first
  // iterate when given (the previous state's Z is its fallback), else that Z
  double Z = zseed ? zseed[cell] : aux_guess[10 * N + cell];
  bool ok = false;
  for (int it = 0; it < 50; ++it) {
    double v[3], W;
    if (!srrmhd_prims_newton(x, g.gamma, Z, v, W, its)) {
      if (it > 0 || !zseed) break;
      Z = aux_guess[10 * N + cell];
      if (!srrmhd_prims_newton(x, g.gamma, Z, v, W, its)) break;
    }
    const double q = x[13];
    const double vE = v[0] * x[8] + v[1] * x[9] + v[2] * x[10];
    const double vxB0 = v[1] * x[7] - v[2] * x[6];
    const double vxB1 = v[2] * x[5] - v[0] * x[7];
    const double vxB2 = v[0] * x[6] - v[1] * x[5];
    const double Ws = W * sg;
    double R[3];
    R[0] = x[8] - c[8] + a * (q * v[0] + Ws * (x[8] + vxB0 - vE * v[0]));
    R[1] = x[9] - c[9] + a * (q * v[1] + Ws * (x[9] + vxB1 - vE * v[1]));
    R[2] = x[10] - c[10] + a * (q * v[2] + Ws * (x[10] + vxB2 - vE * v[2]));
    // (alpha I - beta v v^T)^-1 R, alpha = 1 + a W sigma, beta = a W sigma
    const double beta = a * Ws, alpha = 1 + beta;
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double vR = v[0] * R[0] + v[1] * R[1] + v[2] * R[2];
    const double iA = 1 / alpha;
    const double f = beta * vR * iA / (alpha - beta * vv);
    double dE[3];
    dE[0] = -(R[0] * iA + f * v[0]);
    dE[1] = -(R[1] * iA + f * v[1]);
    dE[2] = -(R[2] * iA + f * v[2]);
    x[8] += dE[0];
    x[9] += dE[1];
    x[10] += dE[2];
    const double en = fabs(x[8]) + fabs(x[9]) + fabs(x[10]);
    const double dn = fabs(dE[0]) + fabs(dE[1]) + fabs(dE[2]);
    if (dn <= 1e-14 * en + 1e-300) {
      ok = true;
      break;
    }
  }
#pragma unroll
  for (int v = 0; v < 14; ++v) out[v * N + cell] = x[v];
  if (zout) zout[10 * N + cell] = Z;
  return ok;
}

// SSP2 stages (forms 1, 2).
template <int STAGE>
__device__ __forceinline__ bool imex_fast_cell(const Grid& g, long long cell,
                                               const double* __restrict__ cons,
                                               const double* __restrict__ aux_guess,
                                               const double* __restrict__ flux1,
                                               const double* __restrict__ source1,
                                               double* __restrict__ out, double dt, int& its,
                                               const double* zseed = nullptr) {
  return imex_fast_form<STAGE>(g, cell, cons, aux_guess, flux1, nullptr, source1, nullptr, out,
                               nullptr, dt, its, zseed);
}

// The first iterate of SSP2 implicit stage STAGE (the stage's explicit part
// c, SSP2.cc:194-264) of every interior cell, into `out`: the state the
// guess network reads for that stage (stage 1's is U^n itself).
template <int STAGE>
__global__ void __launch_bounds__(128)
    k_imex_explicit_part(Grid g, const double* __restrict__ cons,
                         const double* __restrict__ flux1, const double* __restrict__ source1,
                         double* __restrict__ out, double dt) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
#pragma unroll
  for (int v = 0; v < 14; ++v) {
    const long long o = v * g.Ntot + cell;
    out[o] = STAGE == 1 ? cons[o] : cons[o] - dt * (flux1[o] - kOm2Gam * source1[o]);
  }
}

// SSP3 / SSP2322 stages in the mixed form; failures queued for the exact solve.
template <int FORM>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_imex_fast_form(Grid g, const double* __restrict__ cons, const double* zaux,
                     const double* __restrict__ flux1, const double* __restrict__ flux2,
                     const double* __restrict__ source1, const double* __restrict__ source2,
                     double* __restrict__ out, double* zout, double dt, C2PWork w) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long its_total = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long cell = cell_id(g, i, j, k);
    int its = 0;
    if (!imex_fast_form<FORM>(g, cell, cons, zaux, flux1, flux2, source1, source2, out, zout, dt,
                              its)) {
      const int slot = atomicAdd(w.fail_count, 1);
      w.fail_list[slot] = (int)cell;
    }
    its_total = its;
  }
  const unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) its_total += __shfl_down_sync(0xffffffffu, its_total, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)its_total);
  }
}

template <int STAGE>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_imex_fast(Grid g, const double* __restrict__ cons, const double* __restrict__ aux_guess,
                const double* __restrict__ u1, const double* __restrict__ flux1,
                const double* __restrict__ source1, double* __restrict__ out, double dt,
                C2PWork w, const double* zseed) {
  (void)u1;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long its_total = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long cell = cell_id(g, i, j, k);
    int its = 0;
    if (!imex_fast_cell<STAGE>(g, cell, cons, aux_guess, flux1, source1, out, dt, its,
                               zseed)) {
      const int slot = atomicAdd(w.fail_count, 1);
      w.fail_list[slot] = (int)cell;
    }
    its_total = its;
  }
  const unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) its_total += __shfl_down_sync(0xffffffffu, its_total, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)its_total);
  }
}

// ---------------------------------------------------------------------------
// Ensemble kernels (mixed form).
template <class M, int ORDER, int TI>
__global__ void __launch_bounds__(32 * TI, (fvs2d_min_blocks<M, float, ORDER, TI>()))
    k_ens_fvs_fp32(const Member* __restrict__ mem, const Item* __restrict__ items, int n_items,
                   int ic, int ip, int ia, int iu0, int iout, int mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    fvs2d_tile<M, float, ORDER, TI>(g, d.a[ic], d.a[ip], d.a[ia], iu0 >= 0 ? d.a[iu0] : nullptr,
                                    d.a[iout], d.dt, mode, w.a, w.b, smem_raw,
                                    StageTail{d.a[EA_F1], d.a[EA_S1], g.cp});
    __syncthreads();
  }
}

// One model's members per launch (the work list holds one model's cells), so
// each instantiation carries one recovery method's registers.
template <int MODEL, bool LEAN>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_ens_c2p_newton(const Member* __restrict__ mem, const Item* __restrict__ items, int n_items,
                     int guess_mode, int ic, int ipg, int iag, int ip, int ia) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    const long long t = w.a + threadIdx.x;
    const bool act = t < n_interior(g);
    NewtonTally tl;
    if (act) {
      int i, j, k;
      interior_ijk(g, t, i, j, k);
      const long long cell = cell_id(g, i, j, k);
      if (MODEL == MODEL_SRMHD)
        c2p_srmhd_newton_cell<LEAN>(g, cell, guess_mode, d.a[ic], d.a[ipg], d.a[iag], d.a[ip],
                                    d.a[ia], d.a[EA_SOL], guess_mode ? d.a[EA_ZG] : nullptr, tl);
      else
        c2p_srrmhd_newton_cell<LEAN>(g, cell, d.a[ic], d.a[iag], d.a[ip], d.a[ia], tl,
                                     d.counters, guess_mode ? d.a[EA_ZG] : nullptr);
    }
    tally_flush(tl, act, d.counters);
  }
}

// SSP2 stage STAGE's explicit part of every SRRMHD member into EA_U2 (the
// state the guess network reads for stage 2; stage 1 reads EA_CONS).
__global__ void __launch_bounds__(128)
    k_ens_imex_explicit_part2(const Member* __restrict__ mem, const Item* __restrict__ items,
                              int n_items) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    const long long t = w.a + threadIdx.x;
    if (t >= n_interior(g)) continue;
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long cell = cell_id(g, i, j, k);
#pragma unroll
    for (int v = 0; v < 14; ++v) {
      const long long o = v * g.Ntot + cell;
      d.a[EA_U2][o] = d.a[EA_CONS][o] - d.dt * (d.a[EA_F1][o] - kOm2Gam * d.a[EA_S1][o]);
    }
  }
}

template <int STAGE>
__global__ void __launch_bounds__(128, kNewtonMinBlocks)
    k_ens_imex_fast(const Member* __restrict__ mem, const Item* __restrict__ items, int n_items,
                    int guess_mode) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    const long long t = w.a + threadIdx.x;
    const bool act = t < n_interior(g);
    long long its_total = 0;
    if (act) {
      int i, j, k;
      interior_ijk(g, t, i, j, k);
      int its = 0;
      const long long cell = cell_id(g, i, j, k);
      const bool ok = imex_fast_cell<STAGE>(g, cell, d.a[EA_CONS], d.a[EA_AUX], d.a[EA_F1],
                                            d.a[EA_S1], d.a[STAGE == 1 ? EA_U1 : EA_U2], d.dt,
                                            its, guess_mode ? d.a[EA_ZG] : nullptr);
      its_total = its;
      if (!ok) {  // queued for the reference solve (ens_imex_queued)
        const int slot = atomicAdd(d.fail_count, 1);
        d.fail_list[slot] = (int)cell;
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, act);
    for (int o = 16; o > 0; o >>= 1) its_total += __shfl_down_sync(0xffffffffu, its_total, o);
    if ((threadIdx.x & 31) == 0 && mask) {
      atomicAdd((unsigned long long*)&d.counters[4], (unsigned long long)__popc(mask));
      atomicAdd((unsigned long long*)&d.counters[5], (unsigned long long)its_total);
    }
  }
}

template <class M, int ORDER, int TI>
cudaError_t ens_fvs_fp32_instance(const Member* mem, const Item* items, int n, int ic, int ip,
                                  int ia, int iu0, int iout, int mode, int grid,
                                  cudaStream_t st) {
  using S = Fvs2dSmem<M, float, ORDER, TI>;
  auto kern = k_ens_fvs_fp32<M, ORDER, TI>;
  static int cap = 0;  // resident CTAs of this instance on the device
  if (!cap) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::bytes);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * TI, S::bytes);
    cap = std::max(1, occ) * std::max(1, sms);
  }
  grid = std::min(grid, cap);
  kern<<<grid, dim3(32, TI), S::bytes, st>>>(mem, items, n, ic, ip, ia, iu0, iout, mode);
  return cudaGetLastError();
}

template <class M, int ORDER, int TI>
cudaError_t fvs2d_fp32_instance(const Grid& g, const double* cons, const double* prims,
                                const double* aux, const double* u0, double* out, double dt,
                                int mode, StageTail tail, cudaStream_t st, int ti0, int nti) {
  using S = Fvs2dSmem<M, float, ORDER, TI>;
  auto kern = k_fvs2d<M, float, ORDER, TI>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (e != cudaSuccess) return e;
  const int rows = (g.ie - g.is + TI - 1) / TI;
  if (nti < 0) nti = rows - ti0;
  if (nti <= 0) return cudaSuccess;
  dim3 grid((g.je - g.js + 31) / 32, nti);
  dim3 block(32, TI);
  kern<<<grid, block, S::bytes, st>>>(g, cons, prims, aux, u0, out, dt, mode, tail, ti0);
  return cudaGetLastError();
}

}  // namespace

cudaError_t ens_fvs_fp32(const Member* mem, const Item* items, int n, int model, int order,
                         int TI, int ic, int ip, int ia, int iu0, int iout, int mode, int grid,
                         cudaStream_t st) {
#define ENS_FVS(MM, O, T) \
  return ens_fvs_fp32_instance<MM, O, T>(mem, items, n, ic, ip, ia, iu0, iout, mode, grid, st)
  if (model == MODEL_SRMHD) {
    if (order == 3) {
      if (TI == 4) ENS_FVS(SRMHD, 3, 4);
      if (TI == 16) ENS_FVS(SRMHD, 3, 16);
      ENS_FVS(SRMHD, 3, 8);
    }
    if (TI == 4) ENS_FVS(SRMHD, 5, 4);
    if (TI == 16) ENS_FVS(SRMHD, 5, 16);
    ENS_FVS(SRMHD, 5, 8);
  }
  if (order == 3) {
    if (TI == 4) ENS_FVS(SRRMHD, 3, 4);
    if (TI == 16) ENS_FVS(SRRMHD, 3, 16);
    ENS_FVS(SRRMHD, 3, 8);
  }
  if (TI == 4) ENS_FVS(SRRMHD, 5, 4);
  if (TI == 16) ENS_FVS(SRRMHD, 5, 16);
  ENS_FVS(SRRMHD, 5, 8);
#undef ENS_FVS
}

cudaError_t ens_c2p_newton(const Member* mem, const Item* items, int n, int model,
                           int guess_mode, int ic, int ipg, int iag, int ip, int ia, bool lean,
                           int grid, cudaStream_t st) {
  if (model == MODEL_SRMHD && lean)
    k_ens_c2p_newton<MODEL_SRMHD, true><<<grid, 128, 0, st>>>(mem, items, n, guess_mode, ic, ipg,
                                                              iag, ip, ia);
  else if (model == MODEL_SRMHD)
    k_ens_c2p_newton<MODEL_SRMHD, false><<<grid, 128, 0, st>>>(mem, items, n, guess_mode, ic, ipg,
                                                               iag, ip, ia);
  else if (lean)
    k_ens_c2p_newton<MODEL_SRRMHD, true><<<grid, 128, 0, st>>>(mem, items, n, guess_mode, ic,
                                                               ipg, iag, ip, ia);
  else
    k_ens_c2p_newton<MODEL_SRRMHD, false><<<grid, 128, 0, st>>>(mem, items, n, guess_mode, ic,
                                                                ipg, iag, ip, ia);
  return cudaGetLastError();
}

cudaError_t ens_imex_explicit_part2(const Member* mem, const Item* items, int n, int grid,
                                    cudaStream_t st) {
  k_ens_imex_explicit_part2<<<grid, 128, 0, st>>>(mem, items, n);
  return cudaGetLastError();
}

cudaError_t ens_imex_fast(const Member* mem, const Item* items, int n, int stage, int grid,
                          cudaStream_t st, int guess_mode) {
  if (stage == 1)
    k_ens_imex_fast<1><<<grid, 128, 0, st>>>(mem, items, n, guess_mode);
  else
    k_ens_imex_fast<2><<<grid, 128, 0, st>>>(mem, items, n, guess_mode);
  return cudaGetLastError();
}


cudaError_t launch_fvs2d_fp32(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st,
                              StageTail tail, int ti0, int nti) {
#define FVS32(MM, O) \
  return fvs2d_fp32_instance<MM, O, 8>(g, cons, prims, aux, u0, out, dt, mode, tail, st, ti0, nti)
  if (model == MODEL_SRMHD) {
    switch (order) {
      case 3: FVS32(SRMHD, 3);
      case 5: FVS32(SRMHD, 5);
      case 7: FVS32(SRMHD, 7);
      case 9: FVS32(SRMHD, 9);
      default: FVS32(SRMHD, 11);
    }
  }
  if (model == MODEL_HYBRID) {  // WENO3 / WENO5; higher orders take the generic path
    if (order == 3) FVS32(HYBRID, 3);
    if (order == 5) FVS32(HYBRID, 5);
    return cudaErrorInvalidValue;
  }
  switch (order) {
    case 3: FVS32(SRRMHD, 3);
    case 5: FVS32(SRRMHD, 5);
    case 7: FVS32(SRRMHD, 7);
    case 9: FVS32(SRRMHD, 9);
    default: FVS32(SRRMHD, 11);
  }
#undef FVS32
}

cudaError_t launch_c2p_batch(long long n, double gamma, int method, int guess,
                             const double* cons, double* prims, double* aux,
                             const double* zguess, long long* counters, cudaStream_t st) {
  k_c2p_batch_srmhd<<<(int)((n + 127) / 128), 128, 0, st>>>(n, gamma, method, guess, cons, prims,
                                                              aux, zguess, counters);
  return cudaGetLastError();
}

cudaError_t launch_c2p_mixed(const Grid& g, int model, int guess, const double* cons,
                             const double* prims_guess, const double* aux_guess, double* prims,
                             double* aux, double* solution, C2PWork w, const MixedWork& mw,
                             bool lean, cudaStream_t st, long long t0, long long nt) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  if (nt < 0) nt = nI - t0;
  const long long t_end = t0 + nt;
  const int blocks = (int)((nt + 127) / 128);
  if (nt <= 0) return cudaSuccess;
  if (model == MODEL_SRMHD && guess == 1 && mw.has_mlp) {
    cudaError_t e = mlp::launch_zguess(g, nI, false, cons, mw.mlp_params, mw.feat_stats,
                                       mw.zguess, st, MODEL_SRMHD, w.counters + 3);
    if (e != cudaSuccess) return e;
  }
  if (model == MODEL_SRMHD) {
    const int gm = (guess == 1 && mw.has_mlp) ? 1 : 0;
    if (lean)
      k_c2p_newton_srmhd<true><<<blocks, 128, 0, st>>>(g, gm, cons, prims_guess, aux_guess, prims,
                                                       aux, solution, w, mw.zguess, t0, t_end);
    else
      k_c2p_newton_srmhd<false><<<blocks, 128, 0, st>>>(g, gm, cons, prims_guess, aux_guess, prims,
                                                        aux, solution, w, mw.zguess, t0, t_end);
  } else {
    const double* zseed = nullptr;
    if (guess == 1 && mw.has_mlp) {
      cudaError_t e = mlp::launch_zguess(g, nI, false, cons, mw.mlp_params, mw.feat_stats,
                                         mw.zguess, st, MODEL_SRRMHD, w.counters + 3);
      if (e != cudaSuccess) return e;
      zseed = mw.zguess;
    }
    if (lean)
      k_c2p_newton_srrmhd<true><<<blocks, 128, 0, st>>>(g, cons, aux_guess, prims, aux, w, zseed,
                                                        t0, t_end);
    else
      k_c2p_newton_srrmhd<false><<<blocks, 128, 0, st>>>(g, cons, aux_guess, prims, aux, w,
                                                         zseed, t0, t_end);
  }
  return cudaGetLastError();
}

cudaError_t launch_c2p_hybrid_mixed(const Grid& g, const double* cons, const double* prims_guess,
                                    const double* aux_guess, double* prims, double* aux,
                                    C2PWork w, cudaStream_t st) {
  const long long nI = n_interior_host(g);
  k_c2p_newton_hybrid<<<(int)((nI + 127) / 128), 128, 0, st>>>(g, cons, prims_guess, aux_guess,
                                                               prims, aux, w);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_hybrid_finalise(g, const_cast<double*>(cons), prims, st);
}

cudaError_t launch_imex_fast(const Grid& g, int stage, const double* cons,
                             const double* aux_guess, const double* u1, const double* flux1,
                             const double* source1, double* out, double dt, C2PWork w,
                             cudaStream_t st, const MixedWork* mw) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  const int blocks = (int)((nI + 127) / 128);
  const double* zseed = nullptr;
  if (mw && mw->has_mlp) {
    // the network's Z for the stage's first iterate, its explicit part: U^n
    // itself for stage 1; for stage 2 staged in `out` (which the stage then
    // overwrites)
    if (stage == 2)
      k_imex_explicit_part<2><<<blocks, 128, 0, st>>>(g, cons, flux1, source1, out, dt);
    cudaError_t e = mlp::launch_zguess(g, nI, false, stage == 1 ? cons : out, mw->mlp_params,
                                       mw->feat_stats, mw->zguess, st, MODEL_SRRMHD,
                                       w.counters + 3);
    if (e != cudaSuccess) return e;
    zseed = mw->zguess;
  }
  if (stage == 1)
    k_imex_fast<1><<<blocks, 128, 0, st>>>(g, cons, aux_guess, u1, flux1, source1, out, dt, w,
                                           zseed);
  else
    k_imex_fast<2><<<blocks, 128, 0, st>>>(g, cons, aux_guess, u1, flux1, source1, out, dt, w,
                                           zseed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // cells the fast solve could not converge: the reference stage solve
  return launch_imex_stage_queued(g, stage, cons, aux_guess, u1, flux1, source1, out, dt, w, st);
}

cudaError_t launch_imex_fast_form(const Grid& g, int form, const double* cons,
                                  const double* zaux, const double* u1, const double* u2,
                                  const double* flux1, const double* flux2,
                                  const double* source1, const double* source2, double* out,
                                  double* zout, double dt, C2PWork w, cudaStream_t st) {
  const int blocks = (int)((n_interior_host(g) + 127) / 128);
#define FAST(F)                                                                          \
  k_imex_fast_form<F><<<blocks, 128, 0, st>>>(g, cons, zaux, flux1, flux2, source1, source2, \
                                              out, zout, dt, w)
  switch (form) {
    case 1: FAST(1); break;
    case 2: FAST(2); break;
    case 3: FAST(3); break;
    case 4: FAST(4); break;
    case 5: FAST(5); break;
    case 6: FAST(6); break;
    default: return cudaErrorInvalidValue;
  }
#undef FAST
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // cells the fast solve could not converge: the reference stage solve
  return launch_imex_sweep_queued(g, form, cons, zaux, u1, u2, flux1, flux2, source1, source2,
                                  out, zout, dt, w, st);
}

cudaError_t mixed_init(MixedWork* w, const Grid& g, int model, cudaStream_t st) {
  (void)model;
  cudaError_t e = cudaMalloc(&w->mlp_params, sizeof(float) * MLP_NPARAM);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->mlp_params, 0, sizeof(float) * MLP_NPARAM, st);
  if (e == cudaSuccess) e = cudaMalloc(&w->feat_stats, sizeof(float) * 32);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->feat_stats, 0, sizeof(float) * 32, st);
  if (e == cudaSuccess) e = cudaMalloc(&w->zguess, sizeof(double) * 2 * g.Ntot);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->zguess, 0, sizeof(double) * 2 * g.Ntot, st);
  if (e == cudaSuccess) e = mlp::configure();
  w->has_mlp = 0;
  return e;
}

void mixed_free(MixedWork* w) {
  if (w->mlp_params) cudaFree(w->mlp_params);
  if (w->feat_stats) cudaFree(w->feat_stats);
  if (w->zguess) cudaFree(w->zguess);
  w->mlp_params = nullptr;
  w->feat_stats = nullptr;
  w->zguess = nullptr;
  w->has_mlp = 0;
}

}  // namespace mth
