// The Hybrid model (hybrid.cc): SRRMHD's variables, with the ideal (SRMHD)
// and resistive (SRRMHD) fluxes, sources and initial data blended by a
// penalty weight of the local conductivity, the recovery switching between
// the two models per cell, and optionally the REGIME source on the ideal
// part.  Every expression keeps the reference's order and the unit is
// compiled without FMA contraction, so the plain path is the reference's bit
// for bit.  Generic (materialised-ghost) path, any dimension.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"
#include "minpack.cuh"
#include "srmhd.cuh"
#include "srrmhd.cuh"
#include "hybrid.cuh"

namespace mth {
namespace {

constexpr int kThreads = 128;
inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void load_cell(const Grid& g, const double* cons, const double* prims,
                                          const double* aux, long long cell, double* c, double* p,
                                          double* a) {
  const long long N = g.Ntot;
  for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
  for (int v = 0; v < 11; ++v) p[v] = prims[v * N + cell];
  for (int v = 0; v < 17; ++v) a[v] = aux[v * N + cell];
}

// Hybrid::fluxVector (hybrid.cc:210-259) along `dir` and the Lax-Friedrichs
// split of FVS::fluxReconstruction, every cell: f = (1 - w) f_resistive,
// then + w f_ideal on D, S, tau, B and + w f_ideal(phi) on phi.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_split(Grid g, const double* __restrict__ cons, const double* __restrict__ prims,
                   const double* __restrict__ aux, int dir, double* __restrict__ fplus,
                   double* __restrict__ fminus) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  double c[14], p[11], a[17];
  load_cell(g, cons, prims, aux, cell, c, p, a);
  double f[14];
  hybrid_flux<double>(g, c, p, a, dir, f);
  const long long N = g.Ntot;
  for (int v = 0; v < 14; ++v) {
    fplus[v * N + cell] = 0.5 * (f[v] + 1.0 * c[v]);
    fminus[v * N + cell] = 0.5 * (f[v] - 1.0 * c[v]);
  }
}

// Hybrid::getPrimitiveVars (hybrid.cc:354-436) on interior cells: B and E
// taken from cons, then the resistive recovery where the conductivity is
// below sigmaCrossOver, else SRMHD's single-cell recovery (hybrd1, tol 1.4e-8,
// srmhd.cc:297-377) of the ideal variables and its conversion back.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_c2p(Grid g, const double* __restrict__ cons, const double* prims_guess,
                 const double* aux_guess, double* prims, double* aux, C2PWork w) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  double c[14], p[11], a[17];
  for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
  for (int v = 5; v < 11; ++v) p[v] = c[v];
  bool ok;
  long long evals = 0;
  // Each branch reads only the guesses its recovery uses: the secant on Z
  // its aux[10] (and it writes all of prims and aux), SRMHD's hybrd1 the
  // velocity, density and enthalpy of the ideal variables, which
  // Hybrid::setIdealCPAs copies from the resistive prims[0..3] and aux[0].
  if (sigma_of(g, c[0]) < g.sigma_cross) {
    a[10] = aux_guess[10 * N + cell];
    int ev = 0;
    ok = srrmhd::c2p_cell(c, g.gamma, sigma_of(g, c[0]), p, a, ev);
    evals = ev;
  } else {
    double ic[9], ip[8], ia[13];
    for (int v = 0; v < 8; ++v) ic[v] = c[v];
    ic[8] = c[12];
    for (int v = 0; v < 4; ++v) ip[v] = prims_guess[v * N + cell];
    ia[0] = aux_guess[cell];
    srmhd::Residual R = srmhd::residual_args(ic, g.gamma);
    double x[2], fv[2];
    srmhd::guess_from_prims(ip, ia[0], x);
    const HybrdResult res = Hybrd<2>::solve(R, x, fv, 1.4e-8);
    evals = res.nfev;
    ok = res.info == 1;
    if (ok) {
      srmhd::from_solution(ic, x, g.gamma, R.BS, R.Bsq, R.Ssq, ip, ia);
      for (int v = 0; v < 8; ++v) p[v] = ip[v];
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
    }
  }
  atomicAdd((unsigned long long*)&w.counters[0], 1ull);
  atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)evals);
  if (!ok) {
    atomicAdd((unsigned long long*)&w.counters[2], 1ull);
    atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_C2P);
    return;
  }
  for (int v = 0; v < 11; ++v) prims[v * N + cell] = p[v];
  for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
}

// Hybrid::finalise (hybrid.cc:474-503) on interior cells (the boundary
// conditions that follow overwrite the ghosts): E blended towards -v x B.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_finalise(Grid g, double* cons, double* prims) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  const double iW = ideal_weight(g, sigma_of(g, cons[cell]));
  const double p1 = prims[1 * N + cell], p2 = prims[2 * N + cell], p3 = prims[3 * N + cell];
  const double p5 = prims[5 * N + cell], p6 = prims[6 * N + cell], p7 = prims[7 * N + cell];
  const double iE[3] = {-(p2 * p7 - p3 * p6), -(p3 * p5 - p1 * p7), -(p1 * p6 - p2 * p5)};
  for (int v = 0; v < 3; ++v) {
    double e = cons[(8 + v) * N + cell];
    e *= (1 - iW);
    e += iW * iE[v];
    cons[(8 + v) * N + cell] = e;
    prims[(8 + v) * N + cell] = e;
  }
}

// Hybrid::sourceTermSingleCell (hybrid.cc:261-278) on interior cells.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_source(Grid g, const double* __restrict__ cons, const double* __restrict__ prims,
                    const double* __restrict__ aux, double* __restrict__ src) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  double c[14], p[11], a[17];
  load_cell(g, cons, prims, aux, cell, c, p, a);
  const double iW = ideal_weight(g, sigma_of(g, c[0]));
  double ic[9], ip[8], ia[13], is[9], rs[14];
  ideal_cpas<double>(c, p, a, ic, ip, ia);
  srrmhd::source(c, a, g.cp, rs);
  srmhd::source(ic, g.cp, is);
  for (int v = 0; v < 8; ++v) src[v * N + cell] = iW * is[v] + (1 - iW) * rs[v];
  for (int v = 8; v < 14; ++v) src[v * N + cell] = (1 - iW) * rs[v];
}

// Data::sigmaFunc with cell indices (simData.cc:114-127) as Hybrid::setMasks
// calls it: a negative index reads the first cell's D, any other the flat
// index i Ny Nz + j Nz + k of the D plane (which, past the plane's end, runs
// on into the next variable's, as the reference's arrays do).
__device__ __forceinline__ double sigma_at(const Grid& g, const double* cons, int i, int j,
                                           int k) {
  if (!g.functional_sigma) return g.sigma;
  if (i < 0 || j < 0 || k < 0) return g.sigma * pow(cons[0], g.sigma_exp);
  return g.sigma * pow(cons[((long long)i * g.Ny + j) * g.Nz + k], g.sigma_exp);
}

// Hybrid::setMasks (hybrid.cc:505-560) and the REGIME contribution of
// Hybrid::sourceTerm (hybrid.cc:320-345) on interior cells: src += S_REGIME
// w mask, mask 1 where the cell and its 6^3 neighbourhood (offsets -3 .. 2
// in every direction, also across unused dimensions) are not too resistive.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_regime_add(Grid g, const double* __restrict__ cons, const double* __restrict__ ext,
                        double* __restrict__ src) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  const int ms = 3, mie = g.Nx - 3;
  const int mjs = g.dims < 2 ? 0 : 3, mje = g.dims < 2 ? 1 : g.Ny - 3;
  const int mks = g.dims < 3 ? 0 : 3, mke = g.dims < 3 ? 1 : g.Nz - 3;
  int mask = 0;
  if (i >= ms && i < mie && j >= mjs && j < mje && k >= mks && k < mke &&
      sigma_at(g, cons, i, j, k) > g.sigma_cross - g.sigma_span) {
    bool possible = true;
    for (int l = -3; l < 3; l++)
      for (int m = -3; m < 3; m++)
        for (int n = -3; n < 3; n++)
          if (sigma_at(g, cons, i + l, j + m, k + n) < g.sigma_cross - g.sigma_span)
            possible = false;
    if (possible) mask = 1;
  }
  const double iW = ideal_weight(g, sigma_of(g, cons[cell]));
  for (int v = 0; v < 9; ++v)
    src[v * N + cell] = src[v * N + cell] + ext[v * N + cell] * iW * mask;
}

// Hybrid::primsToAll's blend (hybrid.cc:438-472), every cell: the resistive
// cons / prims / aux (already from SRRMHD's primsToAll) weighted by 1 - w,
// plus w times the ideal ones (SRMHD's primsToAll of the first eight prims,
// in icons / iaux) on the first 9 / 8 / 13 variables.
__global__ void __launch_bounds__(kThreads)
    k_hybrid_blend(Grid g, double* cons, double* prims, double* aux,
                   const double* __restrict__ icons, const double* __restrict__ iaux) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  const double iW = ideal_weight(g, sigma_of(g, cons[cell]));
  for (int v = 0; v < 14; ++v) {
    double x = cons[v * N + cell];
    x *= (1 - iW);
    if (v < 9) x += iW * icons[v * N + cell];
    cons[v * N + cell] = x;
  }
  for (int v = 0; v < 11; ++v) {
    const double ip = prims[v * N + cell];
    double x = ip;
    x *= (1 - iW);
    if (v < 8) x += iW * ip;
    prims[v * N + cell] = x;
  }
  for (int v = 0; v < 17; ++v) {
    double x = aux[v * N + cell];
    x *= (1 - iW);
    if (v < 13) x += iW * iaux[v * N + cell];
    aux[v * N + cell] = x;
  }
}

// cons += h src on interior cells (rkSplit2ndOrder.cc:43-51, 57-65).
__global__ void __launch_bounds__(kThreads)
    k_add_scaled(Grid g, int nc, double* cons, const double* __restrict__ src, double h) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  for (int v = 0; v < nc; ++v) cons[v * N + cell] += h * src[v * N + cell];
}

}  // namespace

cudaError_t launch_hybrid_split(const Grid& g, const double* cons, const double* prims,
                                const double* aux, int dir, double* fplus, double* fminus,
                                cudaStream_t st) {
  k_hybrid_split<<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux, dir, fplus,
                                                          fminus);
  return cudaGetLastError();
}

cudaError_t launch_c2p_hybrid(const Grid& g, const double* cons, const double* prims_guess,
                              const double* aux_guess, double* prims, double* aux, C2PWork w,
                              cudaStream_t st) {
  k_hybrid_c2p<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, cons, prims_guess,
                                                                    aux_guess, prims, aux, w);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_hybrid_finalise<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, const_cast<double*>(cons),
                                                                         prims);
  return cudaGetLastError();
}

cudaError_t launch_hybrid_finalise(const Grid& g, double* cons, double* prims, cudaStream_t st) {
  k_hybrid_finalise<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, cons, prims);
  return cudaGetLastError();
}

cudaError_t launch_hybrid_source(const Grid& g, int order, const double* cons,
                                 const double* prims, const double* aux, double* src,
                                 const RegimeWork* regime, double* ext, bool mixed,
                                 cudaStream_t st) {
  const long long nI = n_interior_host(g);
  k_hybrid_source<<<blocks_for(nI), kThreads, 0, st>>>(g, cons, prims, aux, src);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !regime) return e;
  if ((e = launch_regime_ext(g, order, cons, prims, *regime, ext, mixed, st)) != cudaSuccess)
    return e;
  k_hybrid_regime_add<<<blocks_for(nI), kThreads, 0, st>>>(g, cons, ext, src);
  return cudaGetLastError();
}

cudaError_t launch_hybrid_blend(const Grid& g, double* cons, double* prims, double* aux,
                                const double* icons, const double* iaux, cudaStream_t st) {
  k_hybrid_blend<<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux, icons, iaux);
  return cudaGetLastError();
}

cudaError_t launch_add_scaled(const Grid& g, int nc, double* cons, const double* src, double h,
                              cudaStream_t st) {
  k_add_scaled<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, nc, cons, src, h);
  return cudaGetLastError();
}

}  // namespace mth
