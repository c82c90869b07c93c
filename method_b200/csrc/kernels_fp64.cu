// Plain FP64 kernels.  This translation unit is compiled with -fmad=false
// (and IEEE division / square root, the nvcc defaults) so that every
// expression rounds exactly like the reference's x86-64 build, which has no
// FMA contraction at the default -march.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "ensemble.h"
#include "fvs2d.cuh"
#include "fvs2d_group.cuh"
#include "hybrid.cuh"
#include "launch.h"
#include "minpack.cuh"
#include "srmhd.cuh"
#include "srrmhd.cuh"

namespace mth {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// primsToAll over every cell (srmhd.cc:573-673, srrmhd.cc:358-510).
__global__ void k_prims_to_all_srmhd(Grid g, const double* __restrict__ prims,
                                     double* __restrict__ cons, double* __restrict__ aux) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  double p[8], c[9], a[13];
#pragma unroll
  for (int v = 0; v < 8; ++v) p[v] = prims[v * N + cell];
  srmhd::prims_to_all(p, g.gamma, c, a);
#pragma unroll
  for (int v = 0; v < 9; ++v) cons[v * N + cell] = c[v];
#pragma unroll
  for (int v = 0; v < 13; ++v) aux[v * N + cell] = a[v];
}

// ---------------------------------------------------------------------------
// Boundary conditions: every ghost cell receives the interior value it maps
// to.  Sources are always interior cells, so one pass is race free.
__global__ void k_apply_bcs(Grid g, double* __restrict__ arr, int nvars) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  int k = (int)(cell % g.Nz);
  long long t = cell / g.Nz;
  int j = (int)(t % g.Ny);
  int i = (int)(t / g.Ny);
  bool ghost = (i < g.is || i >= g.ie) || (g.dims > 1 && (j < g.js || j >= g.je)) ||
               (g.dims > 2 && (k < g.ks || k >= g.ke));
  if (!ghost) return;
  long long src = mapped_cell(g, i, j, k);
  for (int v = 0; v < nvars; ++v) arr[v * g.Ntot + cell] = arr[v * g.Ntot + src];
}

// ---------------------------------------------------------------------------
// Generic flux path, one direction at a time, on materialised ghosts.  Mirrors
// FVS::fluxReconstruction and FVS::F (fluxVectorSplitting.cc:4-131).
// Flux vector and Lax-Friedrichs split of one direction over every cell.
template <class M>
__global__ void k_split_dir_full(Grid g, const double* __restrict__ cons,
                                 const double* __restrict__ prims,
                                 const double* __restrict__ aux, int dir,
                                 double* __restrict__ fplus, double* __restrict__ fminus) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  double c[M::NC], p[M::NP], a[M::NA], f[M::NC];
  M::template load_flux_inputs<double>(cons, prims, aux, g.Ntot, cell, c, p, a);
  M::template flux<double>(c, p, a, dir, f);
#pragma unroll
  for (int v = 0; v < M::NC; ++v) {
    fplus[v * g.Ntot + cell] = 0.5 * (f[v] + 1.0 * c[v]);
    fminus[v * g.Ntot + cell] = 0.5 * (f[v] - 1.0 * c[v]);
  }
}

template <int ORDER>
__global__ void k_weno_dir(Grid g, int nc, int dir, const double* __restrict__ fplus,
                           const double* __restrict__ fminus, double* __restrict__ frecon) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  int k = (int)(cell % g.Nz);
  long long t = cell / g.Nz;
  int j = (int)(t % g.Ny);
  int i = (int)(t / g.Ny);
  constexpr int shift = (ORDER + 1) / 2;
  int idx = dir == 0 ? i : (dir == 1 ? j : k);
  int n = dir == 0 ? g.Nx : (dir == 1 ? g.Ny : g.Nz);
  long long stride = dir == 0 ? (long long)g.Ny * g.Nz : (dir == 1 ? g.Nz : 1);
  const bool inside = idx >= shift && idx < n - shift;
  for (int v = 0; v < nc; ++v) {
    double r = 0.0;  // the reference zero-initialises its reconstruction arrays
    if (inside) {
      const double* P = fplus + v * g.Ntot + cell;
      const double* Mm = fminus + v * g.Ntot + cell;
      double up, dn;
      if constexpr (ORDER == 3) {
        up = weno3_exact(P[-2 * stride], P[-1 * stride], P[0]);
        dn = weno3_exact(Mm[1 * stride], Mm[0], Mm[-1 * stride]);
      } else if constexpr (ORDER == 5) {
        up = weno5_exact(P[-3 * stride], P[-2 * stride], P[-1 * stride], P[0], P[1 * stride]);
        dn = weno5_exact(Mm[2 * stride], Mm[1 * stride], Mm[0], Mm[-1 * stride],
                         Mm[-2 * stride]);
      } else {
        // upwind i-shift .. i-shift+order-1, downwind i+shift-1 .. i+shift-order
        const int s = (int)stride;
        up = weno_point<ORDER, double>(P - shift * stride, s);
        dn = weno_point<ORDER, double>(Mm + (shift - 1) * stride, -s);
      }
      r = up + dn;
    } else {
      r = 0.0 + 0.0;
    }
    frecon[v * g.Ntot + cell] = r;
  }
}

// k_weno_dir for a runtime order.
void weno_dir_launch(const Grid& g, int nc, int order, int dir, const double* fplus,
                     const double* fminus, double* frecon, cudaStream_t st) {
  const int b = (int)((g.Ntot + kThreads - 1) / kThreads);
  switch (order) {
    case 3: k_weno_dir<3><<<b, kThreads, 0, st>>>(g, nc, dir, fplus, fminus, frecon); break;
    case 5: k_weno_dir<5><<<b, kThreads, 0, st>>>(g, nc, dir, fplus, fminus, frecon); break;
    case 7: k_weno_dir<7><<<b, kThreads, 0, st>>>(g, nc, dir, fplus, fminus, frecon); break;
    case 9: k_weno_dir<9><<<b, kThreads, 0, st>>>(g, nc, dir, fplus, fminus, frecon); break;
    default: k_weno_dir<11><<<b, kThreads, 0, st>>>(g, nc, dir, fplus, fminus, frecon); break;
  }
}

__global__ void k_fnet_dir(Grid g, int nc, int dir, int first, const double* __restrict__ frecon,
                           double* __restrict__ fnet) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
  const long long nb = dir == 0 ? cell_id(g, i + 1, j, k)
                                : (dir == 1 ? cell_id(g, i, j + 1, k) : cell_id(g, i, j, k + 1));
  const double d = dir == 0 ? g.dx : (dir == 1 ? g.dy : g.dz);
  for (int v = 0; v < nc; ++v) {
    const double* F = frecon + v * g.Ntot;
    double val = F[nb] / d - F[cell] / d;
    fnet[v * g.Ntot + cell] = first ? val : fnet[v * g.Ntot + cell] + val;
  }
}

__global__ void k_stage_update(Grid g, int nc, int mode, const double* u0,
                               const double* in, const double* __restrict__ fnet, double dt,
                               double* out) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
  for (int v = 0; v < nc; ++v) {
    const long long o = v * g.Ntot + cell;
    if (mode == STAGE_EULER) out[o] = in[o] - dt * fnet[o];
    else if (mode == STAGE_RK2_CORR) out[o] = 0.5 * (u0[o] + in[o] - dt * fnet[o]);
    else out[o] = fnet[o];
  }
}

// ---------------------------------------------------------------------------
// SRMHD primitive recovery (srmhd.cc:390-562): one Powell-hybrid solve per
// interior cell from the previous state's guess; cells that fail are queued
// for the neighbour-average retry.
constexpr double kSrmhdTol = 1.49011612e-7;

// One interior cell: returns the residual evaluations; a failure is queued.
__device__ __forceinline__ long long c2p_srmhd_hybrd_cell(const Grid& g, long long cell,
                                                          const double* __restrict__ cons,
                                                          const double* prims_guess,
                                                          const double* aux_guess,
                                                          double* prims, double* aux,
                                                          double* __restrict__ solution,
                                                          int* fail_list, int* fail_count) {
  const long long N = g.Ntot;
  double c[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
  double pg[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) pg[v] = prims_guess[v * N + cell];
  double hg = aux_guess[cell];
  srmhd::Residual R = srmhd::residual_args(c, g.gamma);
  double x[2], fv[2];
  srmhd::guess_from_prims(pg, hg, x);
  HybrdResult res = Hybrd<2>::solve(R, x, fv, kSrmhdTol);
  if (res.info == 1) {
    solution[cell] = x[0];
    solution[N + cell] = x[1];
    double p[8], a[13];
    srmhd::from_solution(c, x, g.gamma, R.BS, R.Bsq, R.Ssq, p, a);
#pragma unroll
    for (int v = 0; v < 8; ++v) prims[v * N + cell] = p[v];
#pragma unroll
    for (int v = 0; v < 13; ++v) aux[v * N + cell] = a[v];
  } else {
    prims[5 * N + cell] = c[5];
    prims[6 * N + cell] = c[6];
    prims[7 * N + cell] = c[7];
    aux[10 * N + cell] = R.BS;
    aux[11 * N + cell] = R.Bsq;
    aux[12 * N + cell] = R.Ssq;
    int slot = atomicAdd(fail_count, 1);
    fail_list[slot] = (int)cell;
  }
  return res.nfev;
}

// Registers capped at 64 (8 resident CTAs of 128 threads): twice the warps
// outweigh the local-memory spills this causes (twice the DRAM writes at
// 768^2), OT 1024^2 0.415 -> 0.377 ms per launch.  Register allocation
// changes no result.
__global__ void __launch_bounds__(128, 8)
    k_c2p_srmhd(Grid g, const double* __restrict__ cons, const double* prims_guess,
                const double* aux_guess, double* prims, double* aux,
                double* __restrict__ solution, C2PWork w) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nfev = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    nfev = c2p_srmhd_hybrd_cell(g, cell_id(g, i, j, k), cons, prims_guess, aux_guess, prims, aux,
                                solution, w.fail_list, w.fail_count);
  }
  // one atomic per warp for the statistics
  unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) nfev += __shfl_down_sync(0xffffffffu, nfev, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)nfev);
  }
}

// Neighbour-average retry of failed cells (srmhd.cc:458-507), processed one
// at a time in (i, j, k) order as the reference does.  The reference solves
// the retry with the residual arguments left over from the last interior cell
// of the first pass; that behaviour is kept so that results stay identical.
__device__ void c2p_retry_body(const Grid& g, const double* __restrict__ cons, double* prims,
                               double* aux, double* solution, int* fail_list, int* fail_count,
                               long long* counters) {
  const int n = *fail_count;
  if (n == 0) return;
  int* L = fail_list;
  // heap sort of the failed cell ids (ascending = the reference's loop order)
  for (int s = n / 2 - 1; s >= 0; --s) {
    for (int r = s;;) {
      int ch = 2 * r + 1;
      if (ch >= n) break;
      if (ch + 1 < n && L[ch + 1] > L[ch]) ++ch;
      if (L[r] >= L[ch]) break;
      int tmp = L[r]; L[r] = L[ch]; L[ch] = tmp;
      r = ch;
    }
  }
  for (int end = n - 1; end > 0; --end) {
    int tmp = L[0]; L[0] = L[end]; L[end] = tmp;
    for (int r = 0;;) {
      int ch = 2 * r + 1;
      if (ch >= end) break;
      if (ch + 1 < end && L[ch + 1] > L[ch]) ++ch;
      if (L[r] >= L[ch]) break;
      int t2 = L[r]; L[r] = L[ch]; L[ch] = t2;
      r = ch;
    }
  }
  const long long N = g.Ntot;
  double cl[9];
  const long long last = cell_id(g, g.ie - 1, g.je - 1, g.ke - 1);
  for (int v = 0; v < 9; ++v) cl[v] = cons[v * N + last];
  srmhd::Residual R = srmhd::residual_args(cl, g.gamma);
  long long still = 0, nfev = 0;
  for (int f = 0; f < n; ++f) {
    const long long cell = L[f];
    const int z = (int)(cell % g.Nz);
    const int y = (int)((cell / g.Nz) % g.Ny);
    const int x = (int)(cell / ((long long)g.Nz * g.Ny));
    long long nb[6];
    int cnt = 0;
    if (x > 0) nb[cnt++] = cell_id(g, x - 1, y, z);
    if (y > 0) nb[cnt++] = cell_id(g, x, y - 1, z);
    if (z > 0) nb[cnt++] = cell_id(g, x, y, z - 1);
    if (x < g.Nx - 1) nb[cnt++] = cell_id(g, x + 1, y, z);
    if (y < g.Ny - 1) nb[cnt++] = cell_id(g, x, y + 1, z);
    if (z < g.Nz - 1) nb[cnt++] = cell_id(g, x, y, z + 1);
    double s[2] = {0, 0};
    for (int q = 0; q < cnt; ++q) {
      s[0] += solution[nb[q]];
      s[1] += solution[N + nb[q]];
    }
    s[0] /= (double)cnt;
    s[1] /= (double)cnt;
    double fv[2];
    HybrdResult res = Hybrd<2>::solve(R, s, fv, kSrmhdTol);
    nfev += res.nfev;
    if (res.info != 1) ++still;
    solution[cell] = s[0];
    solution[N + cell] = s[1];
    double c[9];
    for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
    double p[8], a[13];
    srmhd::from_solution(c, s, g.gamma, aux[10 * N + cell], aux[11 * N + cell],
                         aux[12 * N + cell], p, a);
    for (int v = 0; v < 8; ++v) prims[v * N + cell] = p[v];
    for (int v = 0; v < 13; ++v) aux[v * N + cell] = a[v];
  }
  counters[1] += nfev;
  counters[2] += still;
  *fail_count = 0;
}

__global__ void k_c2p_retry_srmhd(Grid g, const double* __restrict__ cons, double* prims,
                                  double* aux, double* solution, C2PWork w) {
  if (threadIdx.x != 0) return;
  c2p_retry_body(g, cons, prims, aux, solution, w.fail_list, w.fail_count, w.counters);
}

// RKSplit source step: target += dt * S(cons) on the interior (rkSplit.cc:31-53).
template <int MODEL>
__global__ void k_source_add(Grid g, const double* __restrict__ cons,
                             const double* __restrict__ prims, const double* __restrict__ aux,
                             double* target, double dt) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  if (MODEL == MODEL_SRMHD) {
    double c[9], s[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
    srmhd::source(c, g.cp, s);
#pragma unroll
    for (int v = 0; v < 9; ++v) target[v * N + cell] = target[v * N + cell] + dt * s[v];
  } else {
    double c[14], a[17], s[14];
#pragma unroll
    for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
#pragma unroll
    for (int v = 0; v < 17; ++v) a[v] = aux[v * N + cell];
    srrmhd::source(c, a, g.cp, s);
#pragma unroll
    for (int v = 0; v < 14; ++v) target[v * N + cell] = target[v * N + cell] + dt * s[v];
  }
}

// ---------------------------------------------------------------------------
// SRRMHD primsToAll with the 4th-order central-difference charge density
// (srrmhd.cc:358-510); the stencil reads the input primitives of neighbours.
__global__ void k_prims_to_all_srrmhd(Grid g, const double* __restrict__ prims,
                                      double* __restrict__ cons, double* __restrict__ aux) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  const int k = (int)(cell % g.Nz);
  const int j = (int)((cell / g.Nz) % g.Ny);
  const int i = (int)(cell / ((long long)g.Nz * g.Ny));
  double p[11], c[14], a[17];
#pragma unroll
  for (int v = 0; v < 11; ++v) p[v] = prims[v * N + cell];
  auto P = [&](int v, int ii, int jj, int kk) { return prims[v * N + cell_id(g, ii, jj, kk)]; };
  bool qfd = true;
  double divE = 0.0;
  if (i > 1 && j > 1 && k > 1 && i < g.Nx - 2 && j < g.Ny - 2 && k < g.Nz - 2) {
    divE = (-P(8, i + 2, j, k) + 8 * P(8, i + 1, j, k) - 8 * P(8, i - 1, j, k) + P(8, i - 2, j, k)) /
               (12 * g.dx) +
           (-P(9, i, j + 2, k) + 8 * P(9, i, j + 1, k) - 8 * P(9, i, j - 1, k) + P(9, i, j - 2, k)) /
               (12 * g.dy) +
           (-P(10, i, j, k + 2) + 8 * P(10, i, j, k + 1) - 8 * P(10, i, j, k - 1) +
            P(10, i, j, k - 2)) /
               (12 * g.dz);
  } else if (i > 1 && j > 1 && i < g.Nx - 2 && j < g.Ny - 2 && g.nz == 0) {
    divE = (-P(8, i + 2, j, k) + 8 * P(8, i + 1, j, k) - 8 * P(8, i - 1, j, k) + P(8, i - 2, j, k)) /
               (12 * g.dx) +
           (-P(9, i, j + 2, k) + 8 * P(9, i, j + 1, k) - 8 * P(9, i, j - 1, k) + P(9, i, j - 2, k)) /
               (12 * g.dy);
  } else if (i > 1 && i < g.Nx - 2 && g.ny == 0) {
    divE = (-P(8, i + 2, j, k) + 8 * P(8, i + 1, j, k) - 8 * P(8, i - 1, j, k) + P(8, i - 2, j, k)) /
           (12 * g.dx);
  } else {
    qfd = false;
  }
  srrmhd::prims_to_all(p, g.gamma, g.sigma, g.sigma_exp, g.functional_sigma, qfd, divE, c, a);
#pragma unroll
  for (int v = 0; v < 14; ++v) cons[v * N + cell] = c[v];
#pragma unroll
  for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
}

// SRRMHD grid primitive recovery (srrmhd.cc:314-356): secant on Z per
// interior cell, seeded from the guess array's aux[10].
__global__ void __launch_bounds__(128)
    k_c2p_srrmhd(Grid g, const double* __restrict__ cons, const double* aux_guess, double* prims,
                 double* aux, C2PWork w) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long evals = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long N = g.Ntot, cell = cell_id(g, i, j, k);
    double c[14], p[11], a[17];
#pragma unroll
    for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
    a[10] = aux_guess[10 * N + cell];
    int ev = 0;
    bool ok = srrmhd::c2p_cell(c, g.gamma, sigma_of(g, c[0]), p, a, ev);
    evals = ev;
    if (ok) {
#pragma unroll
      for (int v = 0; v < 11; ++v) prims[v * N + cell] = p[v];
#pragma unroll
      for (int v = 0; v < 17; ++v) aux[v * N + cell] = a[v];
    } else {
      atomicAdd((unsigned long long*)&w.counters[2], 1ull);
      atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_C2P);
    }
  }
  unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) evals += __shfl_down_sync(0xffffffffu, evals, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)evals);
  }
}

// Model::sourceTerm into an array, over the interior (ALL = false) or every
// cell (ALL = true, the reference's sourceTerm loops, srmhd.cc:226-250).
template <int MODEL, bool ALL>
__global__ void k_source(Grid g, const double* __restrict__ cons, const double* __restrict__ aux,
                         double* __restrict__ out) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long cell;
  if (ALL) {
    if (t >= g.Ntot) return;
    cell = t;
  } else {
    if (t >= n_interior(g)) return;
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    cell = cell_id(g, i, j, k);
  }
  const long long N = g.Ntot;
  if (MODEL == MODEL_SRMHD) {
    double c[9], s[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
    srmhd::source(c, g.cp, s);
#pragma unroll
    for (int v = 0; v < 9; ++v) out[v * N + cell] = s[v];
  } else {
    double c[14], a[17], s[14];
#pragma unroll
    for (int v = 0; v < 14; ++v) c[v] = cons[v * N + cell];
#pragma unroll
    for (int v = 0; v < 17; ++v) a[v] = aux[v * N + cell];
    srrmhd::source(c, a, g.cp, s);
#pragma unroll
    for (int v = 0; v < 14; ++v) out[v * N + cell] = s[v];
  }
}

// One implicit SSP2(222) stage per interior cell: a 14-unknown Powell-hybrid
// solve whose residual runs the secant C2P and the source (SSP2.cc:72-148).
constexpr double kImexTol = 0.000000149011612;
// The reference's SSP2 assigns IMEX2Arguments(data) to its member, but
// IMEX2Arguments::operator= (IMEX2Args.cc:34-63) does not copy gam / om2gam,
// so the constants in effect are those of the default constructor
// (IMEX2Args.h:35-37): om2gam = 0.4142135623730950, one ulp above the
// parameterised constructor's 0.4142135623730949.
constexpr double kImexGam = 0.2928932188134525;
constexpr double kImexOm2Gam = 0.4142135623730950;

// One cell of the implicit stage; returns the residual evaluations and sets
// the error flag when hybrd1 did not converge.
template <int STAGE>
__device__ __forceinline__ long long imex_cell(const Grid& g, long long cell,
                                               const double* __restrict__ cons,
                                               const double* __restrict__ aux_guess,
                                               const double* __restrict__ u1,
                                               const double* __restrict__ flux1,
                                               const double* __restrict__ source1,
                                               double* __restrict__ out, double dt, C2PWork w) {
  const long long N = g.Ntot;
  double u[14], f1[14], s1[14], x[14], fv[14];
#pragma unroll
  for (int v = 0; v < 14; ++v) u[v] = cons[v * N + cell];
  if (STAGE == 1) {
#pragma unroll
    for (int v = 0; v < 14; ++v) x[v] = u[v];
  } else {
#pragma unroll
    for (int v = 0; v < 14; ++v) {
      f1[v] = flux1[v * N + cell];
      s1[v] = source1[v * N + cell];
      x[v] = 0.5 * (u[v] + u1[v * N + cell] - dt * f1[v]);
    }
  }
  srrmhd::ImexResidual R;
  R.u = u;
  R.flux1 = f1;
  R.source1 = s1;
  R.flux2 = nullptr;
  R.source2 = nullptr;
  R.hmgam = 0.0;
  R.dt = dt;
  R.gam = kImexGam;
  R.om2gam = kImexOm2Gam;
  R.g = g.gamma;
  R.sigma = g.sigma;
  R.sigma_exp = g.sigma_exp;
  R.functional = g.functional_sigma;
  R.cp = g.cp;
  R.Z = aux_guess[10 * N + cell];
  R.stage = STAGE;
  R.evals = 0;
  HybrdResult res = Hybrd<14>::solve(R, x, fv, kImexTol);
#pragma unroll
  for (int v = 0; v < 14; ++v) out[v * N + cell] = x[v];
  if (res.info != 1) {
    atomicAdd((unsigned long long*)&w.counters[2], 1ull);
    atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_IMPLICIT);
  }
  return res.nfev;
}

template <int STAGE>
__global__ void __launch_bounds__(64)
    k_imex_stage(Grid g, const double* __restrict__ cons, const double* __restrict__ aux_guess,
                 const double* __restrict__ u1, const double* __restrict__ flux1,
                 const double* __restrict__ source1, double* __restrict__ out, double dt,
                 C2PWork w) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long evals = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    evals = imex_cell<STAGE>(g, cell_id(g, i, j, k), cons, aux_guess, u1, flux1, source1, out,
                             dt, w);
  }
  unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) evals += __shfl_down_sync(0xffffffffu, evals, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)evals);
  }
}

// The same solve for the cells of a queue (mixed-form fallback).  One block
// of 64 threads strides over the queue; the count is reset at the end by the
// block after all threads finished reading it.
template <int STAGE>
__global__ void __launch_bounds__(64)
    k_imex_stage_queued(Grid g, const double* __restrict__ cons,
                        const double* __restrict__ aux_guess, const double* __restrict__ u1,
                        const double* __restrict__ flux1, const double* __restrict__ source1,
                        double* __restrict__ out, double dt, C2PWork w) {
  const int n = *w.fail_count;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    imex_cell<STAGE>(g, w.fail_list[q], cons, aux_guess, u1, flux1, source1, out, dt, w);
    atomicAdd((unsigned long long*)&w.counters[3 + 5], 1ull);  // fallbacks (counters[8])
  }
}

__global__ void k_reset_count(int* c) { *c = 0; }

// SSP3(332) / SSP2(322) implicit stages.  FORM is the residual form of
// srrmhd::ImexResidual (1, 2, 3: SSP3 stages; 4, 5, 6: SSP2322 stages);
// XFORM the initial guess: 0 U^n, 1 U1 (SSP3.cc:114), 2 U2 + dt (F1 + F2) / 4
// (SSP3.cc:149-150), 3 (U^n + U2 - dt F2) / 2 (SSP2322.cc:169-171).  The Z
// guess comes from zaux[10]; as the reference copies args.aux back into
// tempaux after each cell's solve, the last evaluation's Z goes to zout[10],
// which then seeds that stage's recovery.
constexpr double kSsp3Tol = 0.0000000149011612;
constexpr double kSsp2322Tol = 1.48e-8;
constexpr double kImexHmGam = 0.2071067811865475;

template <int FORM, int XFORM>
__device__ __forceinline__ long long imex_sweep_cell(
    const Grid& g, long long cell, const double* __restrict__ cons, const double* zaux,
    const double* __restrict__ u1, const double* __restrict__ u2,
    const double* __restrict__ flux1, const double* __restrict__ flux2,
    const double* __restrict__ source1, const double* __restrict__ source2,
    double* __restrict__ out, double* zout, double dt, C2PWork w) {
  const long long N = g.Ntot;
  double u[14], f1[14], f2[14], s1[14], s2[14], x[14], fv[14];
#pragma unroll
  for (int v = 0; v < 14; ++v) {
    const long long o = v * N + cell;
    u[v] = cons[o];
    f1[v] = (FORM == 2 || FORM == 3) ? flux1[o] : 0.0;
    s1[v] = (FORM == 2 || FORM == 3 || FORM == 5) ? source1[o] : 0.0;
    f2[v] = (FORM == 3 || FORM == 6) ? flux2[o] : 0.0;
    s2[v] = (FORM == 6) ? source2[o] : 0.0;
    if (XFORM == 0) x[v] = u[v];
    else if (XFORM == 1) x[v] = u1[o];
    else if (XFORM == 2) x[v] = u2[o] + dt * (f1[v] + f2[v]) / 4.0;
    else x[v] = 0.5 * (u[v] + u2[o] - dt * f2[v]);
  }
  srrmhd::ImexResidual R;
  R.u = u;
  R.flux1 = f1;
  R.source1 = s1;
  R.flux2 = f2;
  R.source2 = s2;
  R.dt = dt;
  R.gam = kImexGam;
  R.om2gam = kImexOm2Gam;
  R.hmgam = kImexHmGam;
  R.g = g.gamma;
  R.sigma = g.sigma;
  R.sigma_exp = g.sigma_exp;
  R.functional = g.functional_sigma;
  R.cp = g.cp;
  R.Z = zaux[10 * N + cell];
  R.stage = FORM;
  R.evals = 0;
  HybrdResult res = Hybrd<14>::solve(R, x, fv, FORM <= 3 ? kSsp3Tol : kSsp2322Tol);
#pragma unroll
  for (int v = 0; v < 14; ++v) out[v * N + cell] = x[v];
  zout[10 * N + cell] = R.Z;
  if (res.info != 1) {
    atomicAdd((unsigned long long*)&w.counters[2], 1ull);
    atomicOr((unsigned long long*)&w.counters[3], (unsigned long long)ERR_IMPLICIT);
  }
  return res.nfev;
}

template <int FORM, int XFORM>
__global__ void __launch_bounds__(64)
    k_imex_sweep(Grid g, const double* __restrict__ cons, const double* zaux,
                 const double* __restrict__ u1, const double* __restrict__ u2,
                 const double* __restrict__ flux1, const double* __restrict__ flux2,
                 const double* __restrict__ source1, const double* __restrict__ source2,
                 double* __restrict__ out, double* zout, double dt, C2PWork w) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long evals = 0;
  if (t < n_interior(g)) {
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    evals = imex_sweep_cell<FORM, XFORM>(g, cell_id(g, i, j, k), cons, zaux, u1, u2, flux1,
                                         flux2, source1, source2, out, zout, dt, w);
  }
  const unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
  for (int o = 16; o > 0; o >>= 1) evals += __shfl_down_sync(0xffffffffu, evals, o);
  if ((threadIdx.x & 31) == 0 && mask) {
    atomicAdd((unsigned long long*)&w.counters[0], (unsigned long long)__popc(mask));
    atomicAdd((unsigned long long*)&w.counters[1], (unsigned long long)evals);
  }
}

// The same solve for the cells the mixed-form stage queued (grid stride over
// the queue; the count is cleared afterwards by k_reset_count).
template <int FORM, int XFORM>
__global__ void __launch_bounds__(64)
    k_imex_sweep_queued(Grid g, const double* __restrict__ cons, const double* zaux,
                        const double* __restrict__ u1, const double* __restrict__ u2,
                        const double* __restrict__ flux1, const double* __restrict__ flux2,
                        const double* __restrict__ source1, const double* __restrict__ source2,
                        double* __restrict__ out, double* zout, double dt, C2PWork w) {
  const int n = *w.fail_count;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    imex_sweep_cell<FORM, XFORM>(g, w.fail_list[q], cons, zaux, u1, u2, flux1, flux2, source1,
                                 source2, out, zout, dt, w);
    atomicAdd((unsigned long long*)&w.counters[8], 1ull);  // fallbacks
  }
}

// SSP3(332) combination (SSP3.cc:204-214).
__global__ void k_ssp3_combine(Grid g, double* cons, const double* __restrict__ f1,
                               const double* __restrict__ f2, const double* __restrict__ f3,
                               const double* __restrict__ s1, const double* __restrict__ s2,
                               const double* __restrict__ s3, double dt) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
  for (int v = 0; v < 14; ++v) {
    const long long o = v * g.Ntot + cell;
    cons[o] = cons[o] - dt * (f1[o] + f2[o] + 4 * f3[o]) / 6.0 +
              dt * (s1[o] + s2[o] + 4 * s3[o]) / 6.0;
  }
}

// SSP2(322) combination (SSP2322.cc:224-234).
__global__ void k_ssp2322_combine(Grid g, double* cons, const double* __restrict__ f2,
                                  const double* __restrict__ f3, const double* __restrict__ s2,
                                  const double* __restrict__ s3, double dt) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
  for (int v = 0; v < 14; ++v) {
    const long long o = v * g.Ntot + cell;
    cons[o] = cons[o] - dt * 0.5 * (f2[o] + f3[o] - s2[o] - s3[o]);
  }
}

// SSP2 combination U += -0.5 dt (flux1 + flux2 - source1 - source2)
// (SSP2.cc:155-166).
__global__ void k_ssp2_combine(Grid g, int nc, double* cons, const double* __restrict__ flux1,
                               const double* __restrict__ flux2,
                               const double* __restrict__ source1,
                               const double* __restrict__ source2, double dt) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long cell = cell_id(g, i, j, k);
  for (int v = 0; v < nc; ++v) {
    const long long o = v * g.Ntot + cell;
    cons[o] += -0.5 * dt * (flux1[o] + flux2[o] - source1[o] - source2[o]);
  }
}

// Model::fluxVector over every cell (srmhd.cc:72-206, srrmhd.cc:65-192).
template <class M>
__global__ void k_flux_vector(Grid g, const double* __restrict__ cons,
                              const double* __restrict__ prims, const double* __restrict__ aux,
                              int dir, double* __restrict__ f) {
  long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  double c[M::NC], p[M::NP], a[M::NA], fv[M::NC];
  M::template load_flux_inputs<double>(cons, prims, aux, g.Ntot, cell, c, p, a);
  M::template flux<double>(c, p, a, dir, fv);
#pragma unroll
  for (int v = 0; v < M::NC; ++v) f[v * g.Ntot + cell] = fv[v];
}

// SRMHD::getPrimitiveVarsSingleCell (srmhd.cc:297-377) on n independent
// cells, variable-major with stride n.
__global__ void __launch_bounds__(128)
    k_c2p_cells_srmhd(long long n, double gamma, double tol, const double* __restrict__ cons,
                      double* prims, double* aux, int* flag) {
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  double c[9], pg[4];
#pragma unroll
  for (int v = 0; v < 9; ++v) c[v] = cons[v * n + q];
#pragma unroll
  for (int v = 0; v < 4; ++v) pg[v] = prims[v * n + q];
  srmhd::Residual R = srmhd::residual_args(c, gamma);
  double x[2], fv[2];
  srmhd::guess_from_prims(pg, aux[q], x);
  HybrdResult res = Hybrd<2>::solve(R, x, fv, tol);
  if (res.info != 1) {
    atomicOr(flag, 1);
    return;
  }
  double p[8], a[13];
  srmhd::from_solution(c, x, gamma, R.BS, R.Bsq, R.Ssq, p, a);
#pragma unroll
  for (int v = 0; v < 8; ++v) prims[v * n + q] = p[v];
#pragma unroll
  for (int v = 0; v < 13; ++v) aux[v * n + q] = a[v];
}

// SRRMHD::getPrimitiveVarsSingleCell (srrmhd.cc:256-312) on n cells.
__global__ void __launch_bounds__(128)
    k_c2p_cells_srrmhd(long long n, double gamma, double sigma, const double* __restrict__ cons,
                       double* prims, double* aux, int* flag) {
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  double c[14], p[11], a[17];
#pragma unroll
  for (int v = 0; v < 14; ++v) c[v] = cons[v * n + q];
  a[10] = aux[10 * n + q];
  int ev = 0;
  if (!srrmhd::c2p_cell(c, gamma, sigma, p, a, ev)) {
    aux[10 * n + q] = a[10];
    atomicOr(flag, 1);
    return;
  }
#pragma unroll
  for (int v = 0; v < 11; ++v) prims[v * n + q] = p[v];
#pragma unroll
  for (int v = 0; v < 17; ++v) aux[v * n + q] = a[v];
}

// The plain tile runs in passes of kFp64Group variables (fvs2d_group.cuh)
// with registers sized for kFp64Blocks CTAs per SM: WENO3/5 4 CTAs (64
// registers, a few spilled), WENO7 3, WENO9/11 2.  OT 1024^2 WENO5: two
// passes of 5 + 4 variables 0.515 ms per launch, three of 3 0.549 ms (0.600
// at 3 CTAs per SM), the one-pass tile 0.66 ms.
// Grids of fewer than two tiles per SM keep the one-pass tile: there the
// passes only lengthen each CTA (KH 64 x 128: 0.145 against 0.131 ms per
// step).  Both forms give the same bits.
template <class M>
constexpr int kFp64Group = 5;
template <int ORDER>
constexpr int kFp64Blocks = ORDER <= 5 ? 4 : ORDER <= 7 ? 3 : 2;

int device_sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return sms;
}

template <class M, int ORDER, int TI>
cudaError_t fvs2d_instance(const Grid& g, const double* cons, const double* prims,
                           const double* aux, const double* u0, double* out, double dt, int mode,
                           StageTail tail, cudaStream_t st) {
  dim3 grid((g.je - g.js + 31) / 32, (g.ie - g.is + TI - 1) / TI);
  dim3 block(32, TI);
  if ((long long)grid.x * grid.y >= 2LL * device_sm_count()) {
    using S = Fvs2dGroupSmem<M, ORDER, TI, kFp64Group<M>>;
    auto kern = k_fvs2d_group<M, ORDER, TI, kFp64Group<M>, kFp64Blocks<ORDER>>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::bytes);
    if (e != cudaSuccess) return e;
    kern<<<grid, block, S::bytes, st>>>(g, cons, prims, aux, u0, out, dt, mode, tail);
  } else {
    using S = Fvs2dSmem<M, double, ORDER, TI>;
    auto kern = k_fvs2d<M, double, ORDER, TI>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::bytes);
    if (e != cudaSuccess) return e;
    kern<<<grid, block, S::bytes, st>>>(g, cons, prims, aux, u0, out, dt, mode, tail, 0);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Ensemble kernels: CTAs stride over a work list covering every member.
template <class M, int ORDER, int TI>
__global__ void __launch_bounds__(32 * TI)
    k_ens_fvs_fp64(const Member* __restrict__ mem, const Item* __restrict__ items, int n_items,
                   int ic, int ip, int ia, int iu0, int iout, int mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    fvs2d_tile<M, double, ORDER, TI>(g, d.a[ic], d.a[ip], d.a[ia], iu0 >= 0 ? d.a[iu0] : nullptr,
                                     d.a[iout], d.dt, mode, w.a, w.b, smem_raw,
                                     StageTail{d.a[EA_F1], d.a[EA_S1], g.cp});
    __syncthreads();
  }
}

__global__ void __launch_bounds__(128, 8)
    k_ens_c2p_srmhd_hybrd(const Member* __restrict__ mem, const Item* __restrict__ items,
                          int n_items, int ic, int ipg, int iag, int ip, int ia) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    const long long t = w.a + threadIdx.x;
    long long nfev = 0;
    if (t < n_interior(g)) {
      int i, j, k;
      interior_ijk(g, t, i, j, k);
      nfev = c2p_srmhd_hybrd_cell(g, cell_id(g, i, j, k), d.a[ic], d.a[ipg], d.a[iag], d.a[ip],
                                  d.a[ia], d.a[EA_SOL], d.fail_list, d.fail_count);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, t < n_interior(g));
    for (int o = 16; o > 0; o >>= 1) nfev += __shfl_down_sync(0xffffffffu, nfev, o);
    if ((threadIdx.x & 31) == 0 && mask) {
      atomicAdd((unsigned long long*)&d.counters[0], (unsigned long long)__popc(mask));
      atomicAdd((unsigned long long*)&d.counters[1], (unsigned long long)nfev);
    }
  }
}

// One CTA per member: the member's neighbour-average retry.
__global__ void k_ens_c2p_retry(const Member* __restrict__ mem, int ic, int ip, int ia) {
  if (threadIdx.x != 0) return;
  const Member& d = mem[blockIdx.x];
  if (d.model != MODEL_SRMHD) return;
  const Grid g = d.g;
  c2p_retry_body(g, d.a[ic], d.a[ip], d.a[ia], d.a[EA_SOL], d.fail_list, d.fail_count,
                 d.counters);
}

// One CTA per SRRMHD member: the cells of the member's queue that the
// mixed-form implicit solve left unconverged, solved as the reference does
// (the ensemble counterpart of k_imex_stage_queued).
template <int STAGE>
__global__ void __launch_bounds__(64) k_ens_imex_queued(const Member* __restrict__ mem) {
  const Member& d = mem[blockIdx.x];
  if (d.model != MODEL_SRRMHD) return;
  const Grid g = d.g;
  const C2PWork w{d.fail_list, d.fail_count, d.counters + 4};
  const int n = *d.fail_count;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    imex_cell<STAGE>(g, d.fail_list[q], d.a[EA_CONS], d.a[EA_AUX], d.a[EA_U1], d.a[EA_F1],
                     d.a[EA_S1], d.a[STAGE == 1 ? EA_U1 : EA_U2], d.dt, w);
    atomicAdd((unsigned long long*)&w.counters[8], 1ull);  // implicit fallbacks
  }
  __syncthreads();
  if (threadIdx.x == 0) *d.fail_count = 0;
}

// SRRMHD source of the interior cells of every SRRMHD member (srrmhd.cc:194-206);
// here, without contraction, so that members match k_source bit for bit.
__global__ void __launch_bounds__(128)
    k_ens_source(const Member* __restrict__ mem, const Item* __restrict__ items, int n_items,
                 int ic, int ia, int iout) {
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid g = d.g;
    const long long t = w.a + threadIdx.x;
    if (t >= n_interior(g)) continue;
    int i, j, k;
    interior_ijk(g, t, i, j, k);
    const long long N = g.Ntot, cell = cell_id(g, i, j, k);
    double c[14], a[17], s[14];
#pragma unroll
    for (int v = 0; v < 14; ++v) c[v] = d.a[ic][v * N + cell];
#pragma unroll
    for (int v = 0; v < 17; ++v) a[v] = d.a[ia][v * N + cell];
    srrmhd::source(c, a, g.cp, s);
#pragma unroll
    for (int v = 0; v < 14; ++v) d.a[iout][v * N + cell] = s[v];
  }
}

// Simulation::updateTime's dt for every member (simulation.cc:113-124); the
// expression is the host's, compiled without contraction.
__global__ void k_ens_dt(Member* mem, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  Member& d = mem[m];
  const Grid& g = d.g;
  double dtX(d.cfl * g.dx / (1.0 * sqrt((double)g.dims)));
  double dtY(d.cfl * g.dy / (1.0 * sqrt((double)g.dims)));
  double dtZ(d.cfl * g.dz / (1.0 * sqrt((double)g.dims)));
  double dt = (dtX <= dtY && dtX <= dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
  if (d.iters < 15) dt *= 0.1;
  if (d.iters >= 15 && d.iters < 30) dt *= 0.25;
  if (d.t + dt > d.endTime) dt = d.endTime - d.t;
  d.dt = dt;
}

__global__ void k_ens_advance(Member* mem, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  mem[m].t += mem[m].dt;
  mem[m].iters++;
}

template <class M, int ORDER, int TI>
cudaError_t ens_fvs_fp64_instance(const Member* mem, const Item* items, int n, int ic, int ip,
                                  int ia, int iu0, int iout, int mode, int grid,
                                  cudaStream_t st) {
  using S = Fvs2dSmem<M, double, ORDER, TI>;
  auto kern = k_ens_fvs_fp64<M, ORDER, TI>;
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

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t launch_prims_to_all(const Grid& g, int model, const double* prims, double* cons,
                                double* aux, cudaStream_t st) {
  if (model == MODEL_SRMHD) {
    k_prims_to_all_srmhd<<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, prims, cons, aux);
    return cudaGetLastError();
  }
  return launch_prims_to_all_srrmhd(g, prims, cons, aux, st);
}

cudaError_t launch_apply_bcs(const Grid& g, double* arr, int nvars, cudaStream_t st) {
  k_apply_bcs<<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, arr, nvars);
  return cudaGetLastError();
}

// The ghost cells of x-rows [r0, r1) only (k_apply_bcs on a row range).
__global__ void k_apply_bcs_rows(Grid g, double* __restrict__ arr, int nvars, int r0, int r1) {
  const long long plane = (long long)g.Ny * g.Nz;
  const long long cell = r0 * plane + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= r1 * plane) return;
  const int k = (int)(cell % g.Nz);
  const long long t = cell / g.Nz;
  const int j = (int)(t % g.Ny);
  const int i = (int)(t / g.Ny);
  const bool ghost = (i < g.is || i >= g.ie) || (g.dims > 1 && (j < g.js || j >= g.je)) ||
                     (g.dims > 2 && (k < g.ks || k >= g.ke));
  if (!ghost) return;
  const long long src = mapped_cell(g, i, j, k);
  for (int v = 0; v < nvars; ++v) arr[v * g.Ntot + cell] = arr[v * g.Ntot + src];
}

cudaError_t launch_apply_bcs_rows(const Grid& g, double* arr, int nvars, int r0, int r1,
                                  cudaStream_t st) {
  const long long n = (long long)(r1 - r0) * g.Ny * g.Nz;
  if (n <= 0) return cudaSuccess;
  k_apply_bcs_rows<<<blocks_for(n), kThreads, 0, st>>>(g, arr, nvars, r0, r1);
  return cudaGetLastError();
}

cudaError_t launch_fvs2d_fp64(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st,
                              StageTail tail) {
#define FVS64(MM, O) return fvs2d_instance<MM, O, 8>(g, cons, prims, aux, u0, out, dt, mode, tail, st)
  if (model == MODEL_SRMHD) {
    switch (order) {
      case 3: FVS64(SRMHD, 3);
      case 5: FVS64(SRMHD, 5);
      case 7: FVS64(SRMHD, 7);
      case 9: FVS64(SRMHD, 9);
      default: FVS64(SRMHD, 11);
    }
  }
  if (model == MODEL_HYBRID) {  // WENO3 / WENO5; higher orders take the generic path
    if (order == 3) FVS64(HYBRID, 3);
    if (order == 5) FVS64(HYBRID, 5);
    return cudaErrorInvalidValue;
  }
  switch (order) {
    case 3: FVS64(SRRMHD, 3);
    case 5: FVS64(SRRMHD, 5);
    case 7: FVS64(SRRMHD, 7);
    case 9: FVS64(SRRMHD, 9);
    default: FVS64(SRRMHD, 11);
  }
#undef FVS64
}

cudaError_t launch_weno_dir(const Grid& g, int nc, int order, int dir, const double* fplus,
                            const double* fminus, double* frecon, cudaStream_t st) {
  weno_dir_launch(g, nc, order, dir, fplus, fminus, frecon, st);
  return cudaGetLastError();
}

cudaError_t launch_fvs_generic(const Grid& g, int model, int order, double* cons, double* prims,
                               double* aux, double* fplus, double* fminus, double* frecon,
                               double* fnet, cudaStream_t st) {
  const int nc = model == MODEL_SRMHD ? 9 : 14;
  const int np = model == MODEL_SRMHD ? 8 : 11;
  const int na = model == MODEL_SRMHD ? 13 : 17;
  cudaError_t e;
  if ((e = launch_apply_bcs(g, cons, nc, st)) != cudaSuccess) return e;
  if ((e = launch_apply_bcs(g, prims, np, st)) != cudaSuccess) return e;
  if ((e = launch_apply_bcs(g, aux, na, st)) != cudaSuccess) return e;
  return launch_fvs_generic_raw(g, model, order, cons, prims, aux, fplus, fminus, frecon, fnet,
                                st);
}

cudaError_t launch_fvs_generic_raw(const Grid& g, int model, int order, const double* cons,
                                   const double* prims, const double* aux, double* fplus,
                                   double* fminus, double* frecon, double* fnet,
                                   cudaStream_t st) {
  const int nc = model == MODEL_SRMHD ? 9 : 14;
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  for (int dir = 0; dir < g.dims; ++dir) {
    if (model == MODEL_SRMHD) {
      k_split_dir_full<SRMHD><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux, dir,
                                                                        fplus, fminus);
    } else if (model == MODEL_HYBRID) {
      cudaError_t e = launch_hybrid_split(g, cons, prims, aux, dir, fplus, fminus, st);
      if (e != cudaSuccess) return e;
    } else {
      k_split_dir_full<SRRMHD><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux,
                                                                         dir, fplus, fminus);
    }
    weno_dir_launch(g, nc, order, dir, fplus, fminus, frecon, st);
    k_fnet_dir<<<blocks_for(nI), kThreads, 0, st>>>(g, nc, dir, dir == 0, frecon, fnet);
  }
  return cudaGetLastError();
}

cudaError_t launch_stage_update(const Grid& g, int nc, int mode, const double* u0,
                                const double* in, const double* fnet, double dt, double* out,
                                cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  k_stage_update<<<blocks_for(nI), kThreads, 0, st>>>(g, nc, mode, u0, in, fnet, dt, out);
  return cudaGetLastError();
}

cudaError_t launch_c2p_srmhd(const Grid& g, const double* cons, const double* prims_guess,
                             const double* aux_guess, double* prims, double* aux,
                             double* solution, C2PWork w, cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  k_c2p_srmhd<<<blocks_for(nI, 128), 128, 0, st>>>(g, cons, prims_guess, aux_guess, prims, aux,
                                                    solution, w);
  k_c2p_retry_srmhd<<<1, 32, 0, st>>>(g, cons, prims, aux, solution, w);
  return cudaGetLastError();
}

cudaError_t launch_prims_to_all_srrmhd(const Grid& g, const double* prims, double* cons,
                                       double* aux, cudaStream_t st) {
  k_prims_to_all_srrmhd<<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, prims, cons, aux);
  return cudaGetLastError();
}

cudaError_t launch_c2p_srrmhd(const Grid& g, const double* cons, const double* aux_guess,
                              double* prims, double* aux, C2PWork w, cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  k_c2p_srrmhd<<<blocks_for(nI, 128), 128, 0, st>>>(g, cons, aux_guess, prims, aux, w);
  return cudaGetLastError();
}

cudaError_t launch_source(const Grid& g, int model, const double* cons, const double* aux,
                          double* out, cudaStream_t st, bool all_cells) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  if (all_cells) {
    if (model == MODEL_SRMHD)
      k_source<MODEL_SRMHD, true><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, aux, out);
    else
      k_source<MODEL_SRRMHD, true><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, aux, out);
  } else if (model == MODEL_SRMHD) {
    k_source<MODEL_SRMHD, false><<<blocks_for(nI), kThreads, 0, st>>>(g, cons, aux, out);
  } else {
    k_source<MODEL_SRRMHD, false><<<blocks_for(nI), kThreads, 0, st>>>(g, cons, aux, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_flux_vector(const Grid& g, int model, const double* cons, const double* prims,
                               const double* aux, int dir, double* f, cudaStream_t st) {
  if (model == MODEL_SRMHD)
    k_flux_vector<SRMHD><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux, dir, f);
  else
    k_flux_vector<SRRMHD><<<blocks_for(g.Ntot), kThreads, 0, st>>>(g, cons, prims, aux, dir, f);
  return cudaGetLastError();
}

cudaError_t launch_c2p_cells(int model, double gamma, double sigma, long long n,
                             const double* cons, double* prims, double* aux, double tol,
                             int* flag, cudaStream_t st) {
  if (model == MODEL_SRMHD)
    k_c2p_cells_srmhd<<<blocks_for(n, 128), 128, 0, st>>>(n, gamma, tol, cons, prims, aux, flag);
  else
    k_c2p_cells_srrmhd<<<blocks_for(n, 128), 128, 0, st>>>(n, gamma, sigma, cons, prims, aux,
                                                            flag);
  return cudaGetLastError();
}

cudaError_t launch_imex_stage(const Grid& g, int stage, const double* cons,
                              const double* aux_guess, const double* u1, const double* flux1,
                              const double* source1, double* out, double dt, C2PWork w,
                              cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  if (stage == 1)
    k_imex_stage<1><<<blocks_for(nI, 64), 64, 0, st>>>(g, cons, aux_guess, u1, flux1, source1,
                                                        out, dt, w);
  else
    k_imex_stage<2><<<blocks_for(nI, 64), 64, 0, st>>>(g, cons, aux_guess, u1, flux1, source1,
                                                        out, dt, w);
  return cudaGetLastError();
}

cudaError_t launch_imex_stage_queued(const Grid& g, int stage, const double* cons,
                                     const double* aux_guess, const double* u1,
                                     const double* flux1, const double* source1, double* out,
                                     double dt, C2PWork w, cudaStream_t st) {
  if (stage == 1)
    k_imex_stage_queued<1><<<148, 64, 0, st>>>(g, cons, aux_guess, u1, flux1, source1, out, dt, w);
  else
    k_imex_stage_queued<2><<<148, 64, 0, st>>>(g, cons, aux_guess, u1, flux1, source1, out, dt, w);
  k_reset_count<<<1, 1, 0, st>>>(w.fail_count);
  return cudaGetLastError();
}

cudaError_t launch_imex_sweep(const Grid& g, int form, const double* cons, const double* zaux,
                              const double* u1, const double* u2, const double* flux1,
                              const double* flux2, const double* source1, const double* source2,
                              double* out, double* zout, double dt, C2PWork w, cudaStream_t st) {
  const long long nI = n_interior_host(g);
  const int b = blocks_for(nI, 64);
#define SWEEP(F, X)                                                                        \
  k_imex_sweep<F, X><<<b, 64, 0, st>>>(g, cons, zaux, u1, u2, flux1, flux2, source1, source2, \
                                       out, zout, dt, w)
  switch (form) {
    case 1: SWEEP(1, 0); break;  // SSP3 stage 1
    case 2: SWEEP(2, 1); break;  // SSP3 stage 2
    case 3: SWEEP(3, 2); break;  // SSP3 stage 3
    case 4: SWEEP(4, 0); break;  // SSP2322 stage 1
    case 5: SWEEP(5, 0); break;  // SSP2322 stage 2
    case 6: SWEEP(6, 3); break;  // SSP2322 stage 3
    default: return cudaErrorInvalidValue;
  }
#undef SWEEP
  return cudaGetLastError();
}

cudaError_t launch_imex_sweep_queued(const Grid& g, int form, const double* cons,
                                     const double* zaux, const double* u1, const double* u2,
                                     const double* flux1, const double* flux2,
                                     const double* source1, const double* source2, double* out,
                                     double* zout, double dt, C2PWork w, cudaStream_t st) {
#define QSWEEP(F, X)                                                                     \
  k_imex_sweep_queued<F, X><<<148, 64, 0, st>>>(g, cons, zaux, u1, u2, flux1, flux2, source1, \
                                                source2, out, zout, dt, w)
  switch (form) {
    case 1: QSWEEP(1, 0); break;
    case 2: QSWEEP(2, 1); break;
    case 3: QSWEEP(3, 2); break;
    case 4: QSWEEP(4, 0); break;
    case 5: QSWEEP(5, 0); break;
    case 6: QSWEEP(6, 3); break;
    default: return cudaErrorInvalidValue;
  }
#undef QSWEEP
  k_reset_count<<<1, 1, 0, st>>>(w.fail_count);
  return cudaGetLastError();
}

cudaError_t launch_ssp3_combine(const Grid& g, double* cons, const double* f1, const double* f2,
                                const double* f3, const double* s1, const double* s2,
                                const double* s3, double dt, cudaStream_t st) {
  k_ssp3_combine<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, cons, f1, f2, f3, s1, s2,
                                                                      s3, dt);
  return cudaGetLastError();
}

cudaError_t launch_ssp2322_combine(const Grid& g, double* cons, const double* f2,
                                   const double* f3, const double* s2, const double* s3,
                                   double dt, cudaStream_t st) {
  k_ssp2322_combine<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, cons, f2, f3, s2, s3,
                                                                         dt);
  return cudaGetLastError();
}

cudaError_t launch_ssp2_combine(const Grid& g, int nc, double* cons, const double* flux1,
                                const double* flux2, const double* source1,
                                const double* source2, double dt, cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  k_ssp2_combine<<<blocks_for(nI), kThreads, 0, st>>>(g, nc, cons, flux1, flux2, source1, source2,
                                                      dt);
  return cudaGetLastError();
}

cudaError_t ens_fvs_fp64(const Member* mem, const Item* items, int n, int model, int order,
                         int TI, int ic, int ip, int ia, int iu0, int iout, int mode, int grid,
                         cudaStream_t st) {
#define ENS_FVS(MM, O, T) \
  return ens_fvs_fp64_instance<MM, O, T>(mem, items, n, ic, ip, ia, iu0, iout, mode, grid, st)
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
  return cudaErrorInvalidValue;  // plain-form ensembles are SRMHD
#undef ENS_FVS
}

cudaError_t ens_c2p_srmhd_hybrd(const Member* mem, const Item* items, int n, int ic, int ipg,
                                int iag, int ip, int ia, int grid, cudaStream_t st) {
  k_ens_c2p_srmhd_hybrd<<<grid, 128, 0, st>>>(mem, items, n, ic, ipg, iag, ip, ia);
  return cudaGetLastError();
}

cudaError_t ens_c2p_retry(const Member* mem, int n_members, int ic, int ip, int ia,
                          cudaStream_t st) {
  k_ens_c2p_retry<<<n_members, 32, 0, st>>>(mem, ic, ip, ia);
  return cudaGetLastError();
}

cudaError_t ens_imex_queued(const Member* mem, int n_members, int stage, cudaStream_t st) {
  if (stage == 1)
    k_ens_imex_queued<1><<<n_members, 64, 0, st>>>(mem);
  else
    k_ens_imex_queued<2><<<n_members, 64, 0, st>>>(mem);
  return cudaGetLastError();
}

cudaError_t ens_source(const Member* mem, const Item* items, int n, int ic, int ia, int iout,
                       int grid, cudaStream_t st) {
  k_ens_source<<<grid, 128, 0, st>>>(mem, items, n, ic, ia, iout);
  return cudaGetLastError();
}


cudaError_t ens_dt(Member* mem, int n, cudaStream_t st) {
  k_ens_dt<<<(n + 127) / 128, 128, 0, st>>>(mem, n);
  return cudaGetLastError();
}

cudaError_t ens_advance(Member* mem, int n, cudaStream_t st) {
  k_ens_advance<<<(n + 127) / 128, 128, 0, st>>>(mem, n);
  return cudaGetLastError();
}

cudaError_t launch_source_add(const Grid& g, int model, const double* cons, const double* prims,
                              const double* aux, double* target, double dt, cudaStream_t st) {
  const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  if (model == MODEL_SRMHD)
    k_source_add<MODEL_SRMHD><<<blocks_for(nI), kThreads, 0, st>>>(g, cons, prims, aux, target, dt);
  else
    k_source_add<MODEL_SRRMHD><<<blocks_for(nI), kThreads, 0, st>>>(g, cons, prims, aux, target,
                                                                     dt);
  return cudaGetLastError();
}

}  // namespace mth
