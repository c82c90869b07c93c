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

#include "common.cuh"
#include "fvs2d.cuh"
#include "launch.h"
#include "minpack.cuh"
#include "mixed.h"
#include "srmhd.cuh"
#include "srrmhd.cuh"

namespace mth {

namespace {

__device__ __forceinline__ void interior_ijk(const Grid& g, long long t, int& i, int& j, int& k) {
  const int nk = g.ke - g.ks, nj = g.je - g.js;
  k = g.ks + (int)(t % nk);
  t /= nk;
  j = g.js + (int)(t % nj);
  i = g.is + (int)(t / nj);
}

__device__ __forceinline__ long long n_interior(const Grid& g) {
  return (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
}

// Newton in Z for SRMHD.  On success Z and vsq hold the root.
__device__ __forceinline__ bool newton_srmhd(double D, double tau, double BS2, double Bsq,
                                             double Ssq, double g, double& Z, double& vsq,
                                             int& iters) {
  const double k = (g - 1) / g;
  double Zc = Z;
  if (!(Zc > 0) || !isfinite(Zc)) return false;
  for (int it = 0; it < 60; ++it) {
    ++iters;
    const double Z2 = Zc * Zc, ZB = Zc + Bsq;
    const double N = fma(Ssq, Z2, (2 * Zc + Bsq) * BS2);
    const double Dn = Z2 * ZB * ZB;
    const double v2 = N / Dn;
    if (!(v2 < 1.0)) {  // Z below the physical range: v^2(Z) decreases with Z
      Zc *= 2;
      continue;
    }
    const double om = 1 - v2;
    const double s = sqrt(om);
    const double rho = D * s;
    const double p = k * (Zc * om - rho);
    const double gv = Zc + Bsq - p - 0.5 * Bsq * om - BS2 / (2 * Z2) - D - tau;
    const double dv2 = (fma(2 * Ssq, Zc, 2 * BS2) - v2 * (2 * Zc * ZB * (2 * Zc + Bsq))) / Dn;
    const double dp = k * (om - Zc * dv2 + D * dv2 / (2 * s));
    const double dg = 1 - dp + 0.5 * Bsq * dv2 + BS2 / (Z2 * Zc);
    double Zn = Zc - gv / dg;
    if (!(Zn > 0) || !isfinite(Zn)) Zn = 0.5 * Zc;
    if (fabs(Zn - Zc) <= 1e-13 * Zn) {
      const double Z2n = Zn * Zn, ZBn = Zn + Bsq;
      const double v2n = fma(Ssq, Z2n, (2 * Zn + Bsq) * BS2) / (Z2n * ZBn * ZBn);
      if (!(v2n < 1.0)) return false;
      const double rn = D * sqrt(1 - v2n);
      const double pn = k * (Zn * (1 - v2n) - rn);
      if (pn < 0 || rn < 0) return false;
      Z = Zn;
      vsq = v2n;
      return true;
    }
    Zc = Zn;
  }
  return false;
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
    const double q = Sb2 / Z2;
    const double s = sqrt(1 - q);
    const double r = Zc - k * (Zc - Sb2 / Zc) + (k * s - 1) * D - tauT;
    const double dr = 1 - k * (1 + q) + k * D * (q / Zc) / s;
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

__global__ void __launch_bounds__(128)
    k_c2p_newton_srmhd(Grid g, int guess_mode, const double* __restrict__ cons,
                       const double* prims_guess, const double* aux_guess, double* prims,
                       double* aux, double* __restrict__ solution, C2PWork w,
                       const double* __restrict__ zguess) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long its = 0, fb_prev = 0, fb_hybrd = 0, bad = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long N = g.Ntot, cell = cell_id(g, i, j, k);
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
        fb_prev = 1;
        Z = prev[1];
      }
    }
    if (!ok) ok = newton_srmhd(R.D, R.tau, BS2, R.Bsq, R.Ssq, g.gamma, Z, vsq, it);
    double x[2] = {vsq, Z};
    if (!ok) {
      fb_hybrd = 1;
      x[0] = prev[0];
      x[1] = prev[1];
      double fv[2];
      HybrdResult res = Hybrd<2>::solve(R, x, fv, 1.49011612e-7);
      it += res.nfev;
      if (res.info != 1) bad = 1;
    }
    its = it;
    solution[cell] = x[0];
    solution[N + cell] = x[1];
    double p[8], a[13];
    srmhd::from_solution(c, x, g.gamma, R.BS, R.Bsq, R.Ssq, p, a);
#pragma unroll
    for (int v = 0; v < 8; ++v) prims[v * N + cell] = p[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) aux[v * N + cell] = a[v];
  }
  unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) {
    its += __shfl_down_sync(0xffffffffu, its, o);
    fb_prev += __shfl_down_sync(0xffffffffu, fb_prev, o);
    fb_hybrd += __shfl_down_sync(0xffffffffu, fb_hybrd, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)its);
    if (bad) atomicAdd((unsigned long long*)&w.counters[2], (unsigned long long)bad);
    if (fb_prev) atomicAdd((unsigned long long*)&w.counters[8], (unsigned long long)fb_prev);
    if (fb_hybrd) atomicAdd((unsigned long long*)&w.counters[9], (unsigned long long)fb_hybrd);
  }
}

__global__ void __launch_bounds__(128)
    k_c2p_newton_srrmhd(Grid g, const double* __restrict__ cons, const double* aux_guess,
                        double* prims, double* aux, C2PWork w) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long its = 0, fb = 0, bad = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long N = g.Ntot, cell = cell_id(g, i, j, k);
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
    double Z = aux_guess[10 * N + cell];
    int it = 0;
    bool ok = newton_srrmhd(a[15], c[0], a[16], gm, Z, it);
    if (!ok) {
      fb = 1;
      Z = aux_guess[10 * N + cell];
      ok = srrmhd::z_secant(Z, a[15], c[0], a[16], gm, it);
      if (!ok) bad = 1;
    }
    its = it;
    a[10] = Z;
    a[9] = a[15] / (a[10] * a[10]);
    a[1] = 1.0 / sqrt(1 - a[9]);
    p[0] = c[0] / a[1];
    a[0] = a[10] / (p[0] * a[1] * a[1]);
    a[2] = (a[0] - 1) / gm;
    a[3] = sqrt((a[2] * gm * (gm - 1)) / a[0]);
    p[4] = p[0] * a[2] * (gm - 1);
    p[1] = a[12] / a[10];
    p[2] = a[13] / a[10];
    p[3] = a[14] / a[10];
    a[11] = p[1] * c[8] + p[2] * c[9] + p[3] * c[10];
    const double sg = g.sigma;
    a[4] = c[13] * p[1] + a[1] * sg * (c[8] + (p[2] * c[7] - p[3] * c[6]) - a[11] * p[1]);
    a[5] = c[13] * p[2] + a[1] * sg * (c[9] + (p[3] * c[5] - p[1] * c[7]) - a[11] * p[2]);
    a[6] = c[13] * p[3] + a[1] * sg * (c[10] + (p[1] * c[6] - p[2] * c[5]) - a[11] * p[3]);
    if (!bad) {
#pragma unroll
      for (int v = 0; v < 11; ++v) prims[v * N + cell] = p[v];
#pragma unroll
      for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
    }
  }
  unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) {
    its += __shfl_down_sync(0xffffffffu, its, o);
    fb += __shfl_down_sync(0xffffffffu, fb, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)its);
    if (fb) atomicAdd((unsigned long long*)&w.counters[9], (unsigned long long)fb);
    if (bad) {
      atomicAdd((unsigned long long*)&w.counters[2], (unsigned long long)bad);
      atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_C2P);
    }
  }
}

template <class M, int ORDER, int TI>
cudaError_t fvs2d_fp32_instance(const Grid& g, const double* cons, const double* prims,
                                const double* aux, const double* u0, double* out, double dt,
                                int mode, cudaStream_t st) {
  using S = Fvs2dSmem<M, float, ORDER, TI>;
  auto kern = k_fvs2d<M, float, ORDER, TI>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (e != cudaSuccess) return e;
  dim3 grid((g.je - g.js + 31) / 32, (g.ie - g.is + TI - 1) / TI);
  dim3 block(32, TI);
  kern<<<grid, block, S::bytes, st>>>(g, cons, prims, aux, u0, out, dt, mode);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fvs2d_fp32(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st) {
  if (model == MODEL_SRMHD) {
    if (order == 3)
      return fvs2d_fp32_instance<SRMHD, 3, 8>(g, cons, prims, aux, u0, out, dt, mode, st);
    return fvs2d_fp32_instance<SRMHD, 5, 8>(g, cons, prims, aux, u0, out, dt, mode, st);
  }
  if (order == 3)
    return fvs2d_fp32_instance<SRRMHD, 3, 8>(g, cons, prims, aux, u0, out, dt, mode, st);
  return fvs2d_fp32_instance<SRRMHD, 5, 8>(g, cons, prims, aux, u0, out, dt, mode, st);
}

cudaError_t launch_c2p_mixed(const Grid& g, int model, int guess, const double* cons,
                             const double* prims_guess, const double* aux_guess, double* prims,
                             double* aux, double* solution, C2PWork w, const MixedWork& mw,
                             cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  const int blocks = (int)((nI + 127) / 128);
  if (model == MODEL_SRMHD) {
    k_c2p_newton_srmhd<<<blocks, 128, 0, st>>>(
        g, (guess == 1 && mw.has_mlp) ? 1 : 0, cons, prims_guess, aux_guess, prims, aux, solution,
        w, mw.zguess);
  } else {
    k_c2p_newton_srrmhd<<<blocks, 128, 0, st>>>(g, cons, aux_guess, prims, aux, w);
  }
  return cudaGetLastError();
}

cudaError_t mixed_init(MixedWork* w, const Grid& g, int model, cudaStream_t st) {
  (void)g;
  (void)model;
  cudaError_t e = cudaMalloc(&w->mlp_params, sizeof(__nv_bfloat16) * MLP_NPARAM);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w->mlp_params, 0, sizeof(__nv_bfloat16) * MLP_NPARAM, st);
  if (e != cudaSuccess) return e;
  e = cudaMalloc(&w->feat_stats, sizeof(float) * 32);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w->feat_stats, 0, sizeof(float) * 32, st);
  w->has_mlp = 0;
  return e;
}

void mixed_free(MixedWork* w) {
  if (w->mlp_params) cudaFree(w->mlp_params);
  if (w->feat_stats) cudaFree(w->feat_stats);
  w->mlp_params = nullptr;
  w->feat_stats = nullptr;
  w->has_mlp = 0;
}

}  // namespace mth
