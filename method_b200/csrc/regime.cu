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
#include "regime_tile.cuh"
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

// E of every cell.
__global__ void k_regime_e(Grid g, const double* __restrict__ prims, double* __restrict__ E) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  double e[3];
  regime_e_cell(prims, N, cell, e);
#pragma unroll
  for (int v = 0; v < 3; ++v) E[v * N + cell] = e[v];
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

// The split of every cell along `dir`.
__global__ void k_regime_split(Grid g, int dir, const double* __restrict__ prims,
                               const double* __restrict__ E, double* __restrict__ fp,
                               double* __restrict__ fm) {
  const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (cell >= g.Ntot) return;
  const long long N = g.Ntot;
  const double e[3] = {E[cell], E[N + cell], E[2 * N + cell]};
  double p[3], m[3];
  regime_split_cell(dir, e, prims[5 * N + cell], prims[6 * N + cell], prims[7 * N + cell], p, m);
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    fp[v * N + cell] = p[v];
    fm[v * N + cell] = m[v];
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
  const double K[3] = {Karr[cell], Karr[N + cell], Karr[2 * N + cell]};
  double dx[8], dy[8];
  regime_diffu_cell(g, p, E[cell], E[N + cell], E[2 * N + cell], K, sigma_of(g, cons[cell]),
                    q[cell], dx, dy);
#pragma unroll
  for (int l = 0; l < 8; ++l) DX[l * N + cell] = dx[l];
  if (g.dims < 2) return;
#pragma unroll
  for (int l = 0; l < 8; ++l) DY[l * N + cell] = dy[l];
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

// REGIME::sourceExtension's result alone (REGIME.cc:97-133) on interior
// cells: the central differences of the diffusion vectors; phi's entry 0.
__global__ void k_regime_ext(Grid g, const double* __restrict__ DX,
                             const double* __restrict__ DY, double* __restrict__ ext) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_interior(g)) return;
  int i, j, k;
  interior_ijk(g, t, i, j, k);
  const long long N = g.Ntot, cell = cell_id(g, i, j, k);
  const long long sx = (long long)g.Ny * g.Nz, sy = g.Nz;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    double e = (DX[v * N + cell + sx] - DX[v * N + cell - sx]) / (2 * g.dx);
    if (g.dims > 1) e += (DY[v * N + cell + sy] - DY[v * N + cell - sy]) / (2 * g.dy);
    ext[v * N + cell] = e;
  }
  ext[8 * N + cell] = 0.0;
}

// E, q, the split stiff fluxes and their faces, K and the diffusion vectors
// of every cell into w (the per-array chain).
cudaError_t regime_chain(const Grid& g, int order, const double* cons, const double* prims,
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
  return cudaGetLastError();
}

}  // namespace

// cons (interior) += dt (S(cons) + S_REGIME) with cons and prims' ghosts
// filled by the boundary conditions; w's arrays hold Ntot doubles per
// variable (E 3, q 1 (zero at creation, kept between calls), fp/fm 3 each,
// frx/fry 3 each, K 3, DX/DY 8 each).
cudaError_t launch_regime_source_add(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     const RegimeWork& w, bool mixed, cudaStream_t st) {
  if (regime_tile_applies(g)) {
    if (mixed) return launch_regime_tile_mixed(g, order, cons, prims, target, dt, st);
    return launch_regime_tile_order<double>(g, order, cons, prims, target, dt, st);
  }
  cudaError_t e = regime_chain(g, order, cons, prims, w, st);
  if (e != cudaSuccess) return e;
  const long long nI = n_interior_host(g);
  k_regime_source_add<<<blocks_for(nI), kThreads, 0, st>>>(g, cons, w.DX, w.DY, target, dt);
  return cudaGetLastError();
}

cudaError_t launch_regime_ext(const Grid& g, int order, const double* cons, const double* prims,
                              const RegimeWork& w, double* ext, bool mixed, cudaStream_t st) {
  if (regime_tile_applies(g)) {
    if (mixed) return launch_regime_tile_mixed(g, order, cons, prims, ext, 0.0, st, true);
    return launch_regime_tile_order<double>(g, order, cons, prims, ext, 0.0, st, true);
  }
  cudaError_t e = regime_chain(g, order, cons, prims, w, st);
  if (e != cudaSuccess) return e;
  k_regime_ext<<<blocks_for(n_interior_host(g)), kThreads, 0, st>>>(g, w.DX, w.DY, ext);
  return cudaGetLastError();
}

}  // namespace mth
