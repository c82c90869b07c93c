// REGIME: the resistive extension of ideal SRMHD by a diffusive source term
// (Wright & Hawke 2019, "A resistive extension to ideal MHD"; REGIME.cc), as
// RKSplit's model extension (rkSplit.cc:6-53):
//   S_ext = d/dx^i D^i,  D^i = M^i K,  M^i = -(df^i/dw) (ds-bar/dw)^-1,
//   K = d f-bar^j / dx^j (the stiff, electric-field fluxes, reconstructed
//   by the flux method's WENO).
// Computed as the reference does, over the whole ghost-inclusive arrays (the
// state's ghosts are filled by the boundary conditions first), with its loop
// ranges and its zero-initialised arrays: the charge density q keeps zero
// where its fourth-order stencil does not fit, reconstructed stiff fluxes are
// zero outside [shift, N - shift), K and the diffusion vectors start from
// zero.  Every expression keeps the reference's association order and the
// unit is compiled without FMA contraction, so the results are the
// reference's bit for bit.  One and two dimensions.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"
#include "srmhd.cuh"

namespace mth {
namespace {

constexpr int kThreads = 256;
inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void ijk_of(const Grid& g, long long cell, int& i, int& j, int& k) {
  k = (int)(cell % g.Nz);
  const long long t = cell / g.Nz;
  j = (int)(t % g.Ny);
  i = (int)(t / g.Ny);
}

// E = -v x B of every cell (REGIME.cc:151-153).
__global__ void k_regime_e(Grid g, const double* __restrict__ prims, double* __restrict__ E) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  const double p1 = prims[1 * N + cell], p2 = prims[2 * N + cell], p3 = prims[3 * N + cell];
  const double p5 = prims[5 * N + cell], p6 = prims[6 * N + cell], p7 = prims[7 * N + cell];
  E[0 * N + cell] = -(p2 * p7 - p3 * p6);
  E[1 * N + cell] = -(p3 * p5 - p1 * p7);
  E[2 * N + cell] = -(p1 * p6 - p2 * p5);
}

// Charge density q = div E by fourth-order central differences on cells
// 2 .. N-3 of each direction (REGIME.cc:180-205); other cells keep q = 0.
__global__ void k_regime_q(Grid g, const double* __restrict__ E, double* __restrict__ q) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  int i, j, k;
  ijk_of(g, cell, i, j, k);
  if (i < 2 || i >= g.Nx - 2) return;
  const long long N = g.Ntot, sx = (long long)g.Ny * g.Nz, sy = g.Nz;
  const double* Ex = E;
  double qx = (-Ex[cell + 2 * sx] + 8 * Ex[cell + sx] - 8 * Ex[cell - sx] + Ex[cell - 2 * sx]) /
              (12 * g.dx);
  if (g.dims == 1) {
    q[cell] = qx;
    return;
  }
  if (j < 2 || j >= g.Ny - 2) return;
  const double* Ey = E + N;
  q[cell] = qx + (-Ey[cell + 2 * sy] + 8 * Ey[cell + sy] - 8 * Ey[cell - sy] + Ey[cell - 2 * sy]) /
                     (12 * g.dy);
}

// Lax-Friedrichs split of the stiff fluxes along `dir` (REGIME.cc:302-304,
// 327-329; fluxVectorSplitting.cc:22-33): f-bar_x = (0, Bz, -By),
// f-bar_y = (-Bz, 0, Bx), the "conserved" variables being E.
__global__ void k_regime_split(Grid g, int dir, const double* __restrict__ prims,
                               const double* __restrict__ E, double* __restrict__ fp,
                               double* __restrict__ fm) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  const double p5 = prims[5 * N + cell], p6 = prims[6 * N + cell], p7 = prims[7 * N + cell];
  double fb[3];
  if (dir == 0) {
    fb[0] = 0;
    fb[1] = p7;
    fb[2] = -p6;
  } else {
    fb[0] = -p7;
    fb[1] = 0;
    fb[2] = p5;
  }
  const double alpha = 1;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    const double e = E[v * N + cell];
    fp[v * N + cell] = 0.5 * (fb[v] + alpha * e);
    fm[v * N + cell] = 0.5 * (fb[v] - alpha * e);
  }
}

// K: central differences of the reconstructed stiff face fluxes, x over cells
// 1 .. Nx-2, then y over 1 .. Ny-2 (REGIME.cc:309-318, 334-343).
__global__ void k_regime_k(Grid g, const double* __restrict__ frx, const double* __restrict__ fry,
                           double* __restrict__ K) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  int i, j, k;
  ijk_of(g, cell, i, j, k);
  const long long N = g.Ntot, sx = (long long)g.Ny * g.Nz, sy = g.Nz;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    double kv = 0.0;
    if (i >= 1 && i < g.Nx - 1)
      kv += frx[v * N + cell + sx] / (2 * g.dx) - frx[v * N + cell - sx] / (2 * g.dx);
    if (g.dims > 1 && j >= 1 && j < g.Ny - 1)
      kv += fry[v * N + cell + sy] / (2 * g.dy) - fry[v * N + cell - sy] / (2 * g.dy);
    K[v * N + cell] = kv;
  }
}

// The diffusion vectors D^x (and D^y) = M K, M = -dfdw . dwdsb, of every
// cell (REGIME.cc:223-291, 514-688): M's rows 0 and 4 from column 1 (x) or
// 2 (y) of dfdw and two rows from dwdsb's C block first, then rows 1-4 over
// dfdw's columns 5-10 in order, zero entries included, as the reference
// accumulates them; D from zero over m.
__global__ void k_regime_diffu(Grid g, const double* __restrict__ cons,
                               const double* __restrict__ prims, const double* __restrict__ E,
                               const double* __restrict__ q, const double* __restrict__ Karr,
                               double* __restrict__ DX, double* __restrict__ DY) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  double p[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) p[v] = prims[v * N + cell];
  const double E0 = E[cell], E1 = E[N + cell], E2 = E[2 * N + cell];
  const double K[3] = {Karr[cell], Karr[N + cell], Karr[2 * N + cell]};
  const double sigma = sigma_of(g, cons[cell]);
  const double qch = q[cell];
  // prefactor (REGIME.cc:212-213) and dwdsb (REGIME.cc:230-289)
  const double alpha = 1 / ((qch * qch + sigma * sigma) *
                            ((qch * qch + sigma * sigma) +
                             sigma * sigma * (p[5] * p[5] + p[6] * p[6] + p[7] * p[7])));
  const double qsigsq = qch * qch + sigma * sigma;
  const double sigcu = sigma * sigma * sigma;
  double w[11][3];
  w[0][0] = w[0][1] = w[0][2] = w[4][0] = w[4][1] = w[4][2] = 0.0;
  w[1][0] = -qch * (qch * qch + sigma * sigma * (1 + p[5] * p[5]));
  w[1][1] = -sigma * (p[5] * p[6] * qch * sigma - p[7] * qsigsq);
  w[1][2] = -sigma * (p[5] * p[7] * qch * sigma + p[6] * qsigsq);
  w[2][0] = -sigma * (p[5] * p[6] * qch * sigma + p[7] * qsigsq);
  w[2][1] = -qch * (qch * qch + sigma * sigma * (1 + p[6] * p[6]));
  w[2][2] = -sigma * (p[6] * p[7] * qch * sigma - p[5] * qsigsq);
  w[3][0] = -sigma * (p[5] * p[7] * qch * sigma - p[6] * qsigsq);
  w[3][1] = -sigma * (p[6] * p[7] * qch * sigma + p[5] * qsigsq);
  w[3][2] = -qch * (qch * qch + sigma * sigma * (1 + p[7] * p[7]));
  w[5][0] = -p[5] * sigcu * E0;
  w[5][1] = -p[6] * sigcu * E0 - sigma * qsigsq * p[3];
  w[5][2] = -p[7] * sigcu * E0 + sigma * qsigsq * p[2];
  w[6][0] = -p[5] * sigcu * E1 + sigma * qsigsq * p[3];
  w[6][1] = -p[6] * sigcu * E1;
  w[6][2] = -p[7] * sigcu * E1 - sigma * qsigsq * p[1];
  w[7][0] = -p[5] * sigcu * E2 - sigma * qsigsq * p[2];
  w[7][1] = -p[6] * sigcu * E2 + sigma * qsigsq * p[1];
  w[7][2] = -p[7] * sigcu * E2;
  w[8][0] = -p[5] * p[5] * sigcu - sigma * qsigsq;
  w[8][1] = -p[5] * p[6] * sigcu;
  w[8][2] = -p[5] * p[7] * sigcu;
  w[9][0] = -p[6] * p[5] * sigcu;
  w[9][1] = -p[6] * p[6] * sigcu - sigma * qsigsq;
  w[9][2] = -p[6] * p[7] * sigcu;
  w[10][0] = -p[7] * p[5] * sigcu;
  w[10][1] = -p[7] * p[6] * sigcu;
  w[10][2] = -p[7] * p[7] * sigcu - sigma * qsigsq;
#pragma unroll
  for (int l = 1; l < 11; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) w[l][m] *= alpha;
  const double gp = g.gamma * p[4] / (g.gamma - 1);

  // x (REGIME.cc:527-597): dfxdw rows 1-4, columns 5-10
  {
    const double fd[5][6] = {{0, 0, 0, 0, 0, 0},
                             {-p[5], p[6], p[7], -E0, E1, E2},
                             {-p[6], -p[5], 0, -E1, -E0, 0},
                             {-p[7], 0, -p[5], -E2, 0, -E0},
                             {0, -E2, E1, 0, p[7], -p[6]}};
    double M[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m) M[l][m] = 0.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) M[0][m] -= (p[0] * w[1][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[4][m] -= (gp * w[1][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[6][m] -= (-w[10][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[7][m] -= (w[9][m]);
#pragma unroll
    for (int l = 1; l < 5; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 5; n < 11; ++n) M[l][m] -= fd[l][n - 5] * w[n][m];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      double d = 0.0;
#pragma unroll
      for (int m = 0; m < 3; ++m) d += M[l][m] * K[m];
      DX[l * N + cell] = d;
    }
  }
  if (g.dims < 2) return;
  // y (REGIME.cc:616-687): dfydw rows 1-4, columns 5-10
  {
    const double fd[5][6] = {{0, 0, 0, 0, 0, 0},
                             {-p[6], -p[5], 0, -E1, -E0, 0},
                             {p[5], -p[6], p[7], E0, -E1, E2},
                             {0, -p[7], -p[6], 0, -E2, -E1},
                             {E2, 0, -E0, -p[7], 0, p[5]}};
    double M[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m) M[l][m] = 0.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) M[0][m] -= (p[0] * w[2][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[4][m] -= (gp * w[2][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[5][m] -= (w[10][m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) M[7][m] -= (-w[8][m]);
#pragma unroll
    for (int l = 1; l < 5; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 5; n < 11; ++n) M[l][m] -= fd[l][n - 5] * w[n][m];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      double d = 0.0;
#pragma unroll
      for (int m = 0; m < 3; ++m) d += M[l][m] * K[m];
      DY[l * N + cell] = d;
    }
  }
}

// RKSplit's source step with the extension (rkSplit.cc:6-53): on interior
// cells, source = S(U) + S_ext with S_ext the central differences of the
// diffusion vectors (REGIME.cc:99-133; phi's entry stays zero), then
// U += dt source.
__global__ void k_regime_source_add(Grid g, const double* __restrict__ cons,
                                    const double* __restrict__ DX, const double* __restrict__ DY,
                                    double* target, double dt) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  const long long sx = (long long)g.Ny * g.Nz, sy = g.Nz;
  double c[9], s[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) c[v] = cons[v * N + cell];
  srmhd::source(c, g.cp, s);
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    double ext = 0.0;
    if (v < 8) {
      ext = (DX[v * N + cell + sx] - DX[v * N + cell - sx]) / (2 * g.dx);
      if (g.dims > 1) ext += (DY[v * N + cell + sy] - DY[v * N + cell - sy]) / (2 * g.dy);
    }
    const double src = s[v] + ext;
    target[v * N + cell] = target[v * N + cell] + dt * src;
  }
}

}  // namespace

// cons (interior) += dt (S(cons) + S_REGIME) with cons and prims' ghosts
// filled by the boundary conditions; w's arrays hold Ntot doubles per
// variable (E 3, q 1 (zero at creation, kept between calls), fp/fm 3 each,
// frx/fry 3 each, K 3, DX/DY 8 each).
cudaError_t launch_regime_source_add(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     const RegimeWork& w, cudaStream_t st) {
  const int b = blocks_for(g.Ntot);
  k_regime_e<<<b, kThreads, 0, st>>>(g, prims, w.E);
  k_regime_q<<<b, kThreads, 0, st>>>(g, w.E, w.q);
  cudaError_t e;
  k_regime_split<<<b, kThreads, 0, st>>>(g, 0, prims, w.E, w.fp, w.fm);
  if ((e = launch_weno_dir(g, 3, order, 0, w.fp, w.fm, w.frx, st)) != cudaSuccess) return e;
  if (g.dims > 1) {
    k_regime_split<<<b, kThreads, 0, st>>>(g, 1, prims, w.E, w.fp, w.fm);
    if ((e = launch_weno_dir(g, 3, order, 1, w.fp, w.fm, w.fry, st)) != cudaSuccess) return e;
  }
  k_regime_k<<<b, kThreads, 0, st>>>(g, w.frx, w.fry, w.K);
  k_regime_diffu<<<b, kThreads, 0, st>>>(g, cons, prims, w.E, w.q, w.K, w.DX, w.DY);
  const long long nI = n_interior_host(g);
  k_regime_source_add<<<blocks_for(nI), kThreads, 0, st>>>(g, cons, w.DX, w.DY, target, dt);
  return cudaGetLastError();
}

}  // namespace mth
