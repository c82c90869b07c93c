// REGIME per-cell formulas and the fused 2D tile of RKSplit's source step
// with the extension, shared by the plain unit (regime.cu, compiled without
// FMA contraction: bit-identical to the reference) and the mixed unit
// (regime_mixed.cu: FP32 stiff-flux reconstruction).
#pragma once
#include "common.cuh"
#include "fvs2d.cuh"
#include "srmhd.cuh"

namespace mth {
namespace {

// E = -v x B of one cell (REGIME.cc:151-153) from its primitives.
__device__ __forceinline__ void regime_e_cell(const double* __restrict__ prims, long long N,
                                              long long cell, double* E) {
  const double p1 = prims[1 * N + cell], p2 = prims[2 * N + cell], p3 = prims[3 * N + cell];
  const double p5 = prims[5 * N + cell], p6 = prims[6 * N + cell], p7 = prims[7 * N + cell];
  E[0] = -(p2 * p7 - p3 * p6);
  E[1] = -(p3 * p5 - p1 * p7);
  E[2] = -(p1 * p6 - p2 * p5);
}

// Lax-Friedrichs split of the stiff fluxes along `dir` (REGIME.cc:302-304,
// 327-329; fluxVectorSplitting.cc:22-33): f-bar_x = (0, Bz, -By),
// f-bar_y = (-Bz, 0, Bx), the "conserved" variables being E.
// R = double: the reference's expressions; R = float: the same in FP32
// (the mixed form's reconstruction inputs).
template <typename R>
__device__ __forceinline__ void regime_split_cell(int dir, const double* E, double p5, double p6,
                                                  double p7, R* fp, R* fm) {
  R fb[3];
  if (dir == 0) {
    fb[0] = 0;
    fb[1] = R(p7);
    fb[2] = -R(p6);
  } else {
    fb[0] = -R(p7);
    fb[1] = 0;
    fb[2] = R(p5);
  }
  const R alpha = 1;
#pragma unroll
  for (int v = 0; v < 3; ++v) {
    fp[v] = R(0.5) * (fb[v] + alpha * R(E[v]));
    fm[v] = R(0.5) * (fb[v] - alpha * R(E[v]));
  }
}

// Column m of dwdsb (REGIME.cc:230-289) times the prefactor alpha
// (REGIME.cc:212-213): w[1..10] (w[0] and w[4] are zero and unused).
template <int m>
__device__ __forceinline__ void regime_w_col(const double* p, double E0, double E1, double E2,
                                             double qch, double sigma, double qsigsq,
                                             double sigcu, double alpha, double* w) {
  if constexpr (m == 0) {
    w[1] = -qch * (qch * qch + sigma * sigma * (1 + p[5] * p[5]));
    w[2] = -sigma * (p[5] * p[6] * qch * sigma + p[7] * qsigsq);
    w[3] = -sigma * (p[5] * p[7] * qch * sigma - p[6] * qsigsq);
    w[5] = -p[5] * sigcu * E0;
    w[6] = -p[5] * sigcu * E1 + sigma * qsigsq * p[3];
    w[7] = -p[5] * sigcu * E2 - sigma * qsigsq * p[2];
    w[8] = -p[5] * p[5] * sigcu - sigma * qsigsq;
    w[9] = -p[6] * p[5] * sigcu;
    w[10] = -p[7] * p[5] * sigcu;
  } else if constexpr (m == 1) {
    w[1] = -sigma * (p[5] * p[6] * qch * sigma - p[7] * qsigsq);
    w[2] = -qch * (qch * qch + sigma * sigma * (1 + p[6] * p[6]));
    w[3] = -sigma * (p[6] * p[7] * qch * sigma + p[5] * qsigsq);
    w[5] = -p[6] * sigcu * E0 - sigma * qsigsq * p[3];
    w[6] = -p[6] * sigcu * E1;
    w[7] = -p[6] * sigcu * E2 + sigma * qsigsq * p[1];
    w[8] = -p[5] * p[6] * sigcu;
    w[9] = -p[6] * p[6] * sigcu - sigma * qsigsq;
    w[10] = -p[7] * p[6] * sigcu;
  } else {
    w[1] = -sigma * (p[5] * p[7] * qch * sigma + p[6] * qsigsq);
    w[2] = -sigma * (p[6] * p[7] * qch * sigma - p[5] * qsigsq);
    w[3] = -qch * (qch * qch + sigma * sigma * (1 + p[7] * p[7]));
    w[5] = -p[7] * sigcu * E0 + sigma * qsigsq * p[2];
    w[6] = -p[7] * sigcu * E1 - sigma * qsigsq * p[1];
    w[7] = -p[7] * sigcu * E2;
    w[8] = -p[5] * p[7] * sigcu;
    w[9] = -p[6] * p[7] * sigcu;
    w[10] = -p[7] * p[7] * sigcu - sigma * qsigsq;
  }
#pragma unroll
  for (int l = 1; l < 11; ++l)
    if (l != 4) w[l] *= alpha;
}

// Column m of M = -dfdw . dwdsb along x (DIR 0, REGIME.cc:527-597) or y
// (DIR 1, REGIME.cc:616-687): rows 0 and 4 from column 1 (x) or 2 (y) of
// dfdw and two rows from dwdsb's C block first, then rows 1-4 over dfdw's
// columns 5-10 in order, zero entries included, as the reference accumulates
// them; then D += M[:, m] K[m].
template <int DIR>
__device__ __forceinline__ void regime_d_col(const double* p, double gp, double E0, double E1,
                                             double E2, const double* w, double Km, double* D) {
  double fd[5][6];
  if constexpr (DIR == 0) {
    const double t[5][6] = {{0, 0, 0, 0, 0, 0},
                            {-p[5], p[6], p[7], -E0, E1, E2},
                            {-p[6], -p[5], 0, -E1, -E0, 0},
                            {-p[7], 0, -p[5], -E2, 0, -E0},
                            {0, -E2, E1, 0, p[7], -p[6]}};
#pragma unroll
    for (int l = 0; l < 5; ++l)
#pragma unroll
      for (int n = 0; n < 6; ++n) fd[l][n] = t[l][n];
  } else {
    const double t[5][6] = {{0, 0, 0, 0, 0, 0},
                            {-p[6], -p[5], 0, -E1, -E0, 0},
                            {p[5], -p[6], p[7], E0, -E1, E2},
                            {0, -p[7], -p[6], 0, -E2, -E1},
                            {E2, 0, -E0, -p[7], 0, p[5]}};
#pragma unroll
    for (int l = 0; l < 5; ++l)
#pragma unroll
      for (int n = 0; n < 6; ++n) fd[l][n] = t[l][n];
  }
  double M[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) M[l] = 0.0;
  if (DIR == 0) {
    M[0] -= (p[0] * w[1]);
    M[4] -= (gp * w[1]);
    M[6] -= (-w[10]);
    M[7] -= (w[9]);
  } else {
    M[0] -= (p[0] * w[2]);
    M[4] -= (gp * w[2]);
    M[5] -= (w[10]);
    M[7] -= (-w[8]);
  }
#pragma unroll
  for (int l = 1; l < 5; ++l)
#pragma unroll
    for (int n = 5; n < 11; ++n) M[l] -= fd[l][n - 5] * w[n];
#pragma unroll
  for (int l = 0; l < 8; ++l) D[l] += M[l] * Km;
}

// The diffusion vectors D^x (and D^y, dims > 1) = M K of one cell
// (REGIME.cc:223-291, 514-688), D from zero over m = 0, 1, 2.  Computed a
// column of M at a time: each entry is the same sum in the same order as
// the full matrices, with fewer values live at once.
__device__ __forceinline__ void regime_diffu_cell(const Grid& g, const double* p, double E0,
                                                  double E1, double E2, const double* K,
                                                  double sigma, double qch, double* DXo,
                                                  double* DYo) {
  const double alpha = 1 / ((qch * qch + sigma * sigma) *
                            ((qch * qch + sigma * sigma) +
                             sigma * sigma * (p[5] * p[5] + p[6] * p[6] + p[7] * p[7])));
  const double qsigsq = qch * qch + sigma * sigma;
  const double sigcu = sigma * sigma * sigma;
  const double gp = g.gamma * p[4] / (g.gamma - 1);
  const bool two_d = g.dims > 1;
#pragma unroll
  for (int l = 0; l < 8; ++l) DXo[l] = DYo[l] = 0.0;
  double w[11];
  regime_w_col<0>(p, E0, E1, E2, qch, sigma, qsigsq, sigcu, alpha, w);
  regime_d_col<0>(p, gp, E0, E1, E2, w, K[0], DXo);
  if (two_d) regime_d_col<1>(p, gp, E0, E1, E2, w, K[0], DYo);
  regime_w_col<1>(p, E0, E1, E2, qch, sigma, qsigsq, sigcu, alpha, w);
  regime_d_col<0>(p, gp, E0, E1, E2, w, K[1], DXo);
  if (two_d) regime_d_col<1>(p, gp, E0, E1, E2, w, K[1], DYo);
  regime_w_col<2>(p, E0, E1, E2, qch, sigma, qsigsq, sigcu, alpha, w);
  regime_d_col<0>(p, gp, E0, E1, E2, w, K[2], DXo);
  if (two_d) regime_d_col<1>(p, gp, E0, E1, E2, w, K[2], DYo);
}

// ---------------------------------------------------------------------------
// The same source step as one 2D tile kernel.  A CTA owns TI x TJ interior
// cells and forms, in shared memory, everything their update reads: E on the
// tile plus 3 cells, the split stiff fluxes and their WENO faces along x and
// then y, K and q on the tile plus one cell (R1), the diffusion vectors on R1,
// and finally the update of its own cells.  With R = double each value is
// the per-cell formula of the per-array kernels of regime.cu (the same device
// functions or expressions, the same zero-outside-range rules, on global
// indices), so the result is bit-identical to that chain; only the
// intermediate arrays stay on chip.  R = float is the mixed form: the split
// and WENO faces in FP32, everything from K's differences on in FP64.  With a
// conductivity that depends on the state (functionalSigma) the diffusion
// vectors of a halo cell would read cons[0] that a neighbouring CTA updates
// in place, so that case keeps the per-array chain.
template <int ORDER, typename R>
struct RegimeTile {
  static constexpr int TI = 8, TJ = 32, NT = TI * TJ, S = (ORDER + 1) / 2;
  static constexpr int R1I = TI + 2, R1J = TJ + 2, R1 = R1I * R1J;  // rows/cols -1 .. T
  static constexpr int RXI = TI + 3 + 2 * S, RX = RXI * R1J;        // x split: rows -2-S .. TI+S
  static constexpr int RYJ = TJ + 3 + 2 * S, RY = R1I * RYJ;        // y split: cols -2-S .. TJ+S
  static constexpr int RS = RX > RY ? RX : RY;
  static constexpr int FXI = TI + 4, FX = FXI * R1J;  // x faces: rows -2 .. TI+1, cols of R1
  static constexpr int FYJ = TJ + 4, FY = R1I * FYJ;  // y faces: rows of R1, cols -2 .. TJ+1
  static constexpr int EI = TI + 6, EJ = TJ + 6, EN = EI * EJ;  // E: rows/cols -3 .. T+2
  // bytes of the split and faces (R), later reused for the diffusion vectors (double)
  static constexpr size_t A0 = sizeof(R) * (size_t)(6 * RS + 3 * FX + 3 * FY);
  static constexpr size_t A = A0 > sizeof(double) * 16 * R1 ? A0 : sizeof(double) * 16 * R1;
  static constexpr size_t bytes = A + sizeof(double) * (size_t)(3 * EN + 4 * R1);
  static constexpr int MINB = ORDER <= 5 ? 3 : 2;
  static_assert(A % sizeof(double) == 0, "the FP64 arrays follow the split region");
};

__device__ __forceinline__ long long clamped_cell(const Grid& g, int i, int j) {
  i = min(max(i, 0), g.Nx - 1);
  j = min(max(j, 0), g.Ny - 1);
  return (long long)i * g.Ny + j;
}

template <int ORDER, typename R>
__global__ void __launch_bounds__(RegimeTile<ORDER, R>::NT, RegimeTile<ORDER, R>::MINB)
    k_regime_tile(Grid g, const double* __restrict__ cons, const double* __restrict__ prims,
                  double* target, double dt, bool ext_only) {
  using T = RegimeTile<ORDER, R>;
  constexpr int S = T::S, TJ = T::TJ, NT = T::NT, R1J = T::R1J, EJ = T::EJ;
  extern __shared__ __align__(16) unsigned char sh_raw[];
  R* spl = reinterpret_cast<R*>(sh_raw);            // f+ [3][RS], f- [3][RS]
  R* frx = spl + 6 * T::RS;                         // [3][FX]
  R* fry = frx + 3 * T::FX;                         // [3][FY]
  double* Dsh = reinterpret_cast<double*>(sh_raw);  // DX [8][R1], DY [8][R1], once the above are dead
  double* Esh = reinterpret_cast<double*>(sh_raw + T::A);  // [3][EN]
  double* KQ = Esh + 3 * T::EN;                     // K [3][R1], q [R1]
  const int tid = threadIdx.x;
  const int i0 = g.is + blockIdx.y * T::TI, j0 = g.js + blockIdx.x * TJ;
  const long long N = g.Ntot;
  // The plain form divides as the reference does; the mixed form multiplies
  // by reciprocals of the central-difference widths.
  constexpr bool kExact = sizeof(R) == sizeof(double);
  const double i2dx = 1.0 / (2 * g.dx), i2dy = 1.0 / (2 * g.dy);
  const double i12dx = 1.0 / (12 * g.dx), i12dy = 1.0 / (12 * g.dy);

  // E on rows/cols -3 .. T+2 of the tile; the x split on rows -2-S .. TI+S,
  // columns -1 .. TJ (indices outside the array are clamped: such values
  // only reach cells whose results are zero by the range rules or unused)
  for (int e = tid; e < T::EN; e += NT) {
    const int r = e / EJ, c = e - r * EJ;
    double E[3];
    regime_e_cell(prims, N, clamped_cell(g, i0 - 3 + r, j0 - 3 + c), E);
#pragma unroll
    for (int v = 0; v < 3; ++v) Esh[v * T::EN + e] = E[v];
  }
  for (int e = tid; e < T::RX; e += NT) {
    const int r = e / R1J, c = e - r * R1J;
    const long long cell = clamped_cell(g, i0 - 2 - S + r, j0 - 1 + c);
    double E[3];
    R fp[3], fm[3];
    regime_e_cell(prims, N, cell, E);
    regime_split_cell<R>(0, E, prims[5 * N + cell], prims[6 * N + cell], prims[7 * N + cell], fp, fm);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      spl[v * T::RS + e] = fp[v];
      spl[(3 + v) * T::RS + e] = fm[v];
    }
  }
  __syncthreads();
  // x faces on rows -2 .. TI+1 (zero outside [S, Nx - S), as k_weno_dir)
  for (int e = tid; e < 3 * T::FX; e += NT) {
    const int v = e / T::FX, f = e - v * T::FX, r = f / R1J, c = f - r * R1J;
    const int gi = i0 - 2 + r;
    R val;
    if (gi >= S && gi < g.Nx - S)
      val = weno_face<ORDER, R>(spl + v * T::RS + c, spl + (3 + v) * T::RS + c, R1J, r);
    else
      val = R(0.0) + R(0.0);
    frx[e] = val;
  }
  __syncthreads();
  // the y split on rows -1 .. TI, columns -2-S .. TJ+S
  for (int e = tid; e < T::RY; e += NT) {
    const int r = e / T::RYJ, c = e - r * T::RYJ;
    const long long cell = clamped_cell(g, i0 - 1 + r, j0 - 2 - S + c);
    double E[3];
    R fp[3], fm[3];
    regime_e_cell(prims, N, cell, E);
    regime_split_cell<R>(1, E, prims[5 * N + cell], prims[6 * N + cell], prims[7 * N + cell], fp, fm);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      spl[v * T::RS + e] = fp[v];
      spl[(3 + v) * T::RS + e] = fm[v];
    }
  }
  __syncthreads();
  // y faces on columns -2 .. TJ+1 (zero outside [S, Ny - S))
  for (int e = tid; e < 3 * T::FY; e += NT) {
    const int v = e / T::FY, f = e - v * T::FY, r = f / T::FYJ, c = f - r * T::FYJ;
    const int gj = j0 - 2 + c;
    R val;
    if (gj >= S && gj < g.Ny - S)
      val = weno_face<ORDER, R>(spl + v * T::RS + r * T::RYJ,
                                spl + (3 + v) * T::RS + r * T::RYJ, 1, c);
    else
      val = R(0.0) + R(0.0);
    fry[e] = val;
  }
  __syncthreads();
  // K and q on R1 (k_regime_k, k_regime_q)
  for (int e = tid; e < T::R1; e += NT) {
    const int r = e / R1J, c = e - r * R1J;
    const int gi = i0 - 1 + r, gj = j0 - 1 + c;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const R* fx = frx + v * T::FX + r * R1J + c;
      const R* fy = fry + v * T::FY + r * T::FYJ + c;
      double kv = 0.0;
      if constexpr (kExact) {
        if (gi >= 1 && gi < g.Nx - 1)
          kv += double(fx[2 * R1J]) / (2 * g.dx) - double(fx[0]) / (2 * g.dx);
        if (gj >= 1 && gj < g.Ny - 1)
          kv += double(fy[2]) / (2 * g.dy) - double(fy[0]) / (2 * g.dy);
      } else {
        if (gi >= 1 && gi < g.Nx - 1) kv += (double(fx[2 * R1J]) - double(fx[0])) * i2dx;
        if (gj >= 1 && gj < g.Ny - 1) kv += (double(fy[2]) - double(fy[0])) * i2dy;
      }
      KQ[v * T::R1 + e] = kv;
    }
    double qv = 0.0;
    if (gi >= 2 && gi < g.Nx - 2 && gj >= 2 && gj < g.Ny - 2) {
      const double* Ex = Esh + (r + 2) * EJ + (c + 2);
      const double* Ey = Ex + T::EN;
      if constexpr (kExact) {
        const double qx = (-Ex[2 * EJ] + 8 * Ex[EJ] - 8 * Ex[-EJ] + Ex[-2 * EJ]) / (12 * g.dx);
        qv = qx + (-Ey[2] + 8 * Ey[1] - 8 * Ey[-1] + Ey[-2]) / (12 * g.dy);
      } else {
        qv = (-Ex[2 * EJ] + 8 * Ex[EJ] - 8 * Ex[-EJ] + Ex[-2 * EJ]) * i12dx +
             (-Ey[2] + 8 * Ey[1] - 8 * Ey[-1] + Ey[-2]) * i12dy;
      }
    }
    KQ[3 * T::R1 + e] = qv;
  }
  __syncthreads();
  // diffusion vectors on R1 (k_regime_diffu), over the dead split and faces
  for (int e = tid; e < T::R1; e += NT) {
    const int r = e / R1J, c = e - r * R1J;
    const long long cell = clamped_cell(g, i0 - 1 + r, j0 - 1 + c);
    double p[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) p[v] = prims[v * N + cell];
    const double* E = Esh + (r + 2) * EJ + (c + 2);
    const double K[3] = {KQ[e], KQ[T::R1 + e], KQ[2 * T::R1 + e]};
    double dx[8], dy[8];
    regime_diffu_cell(g, p, E[0], E[T::EN], E[2 * T::EN], K, g.sigma, KQ[3 * T::R1 + e], dx, dy);
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      Dsh[l * T::R1 + e] = dx[l];
      Dsh[(8 + l) * T::R1 + e] = dy[l];
    }
  }
  __syncthreads();
  // the update of the tile's own cells (k_regime_source_add)
  const int ty = tid / TJ, tx = tid - ty * TJ;
  const int i = i0 + ty, j = j0 + tx;
  if (i >= g.ie || j >= g.je) return;
  const long long cell = (long long)i * g.Ny + j;
  const int e = (ty + 1) * R1J + tx + 1;
  // ext_only: the extension's source alone into target (REGIME::sourceExtension,
  // phi's entry 0), as the Hybrid model's source reads it
  double s[9];
  if (!ext_only) {
    double cv[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) cv[v] = cons[v * N + cell];
    srmhd::source(cv, g.cp, s);
  }
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    double ext = 0.0;
    if (v < 8) {
      const double ddx = Dsh[v * T::R1 + e + R1J] - Dsh[v * T::R1 + e - R1J];
      const double ddy = Dsh[(8 + v) * T::R1 + e + 1] - Dsh[(8 + v) * T::R1 + e - 1];
      if constexpr (kExact) {
        ext = ddx / (2 * g.dx);
        ext += ddy / (2 * g.dy);
      } else {
        ext = ddx * i2dx + ddy * i2dy;
      }
    }
    if (ext_only) {
      target[v * N + cell] = ext;
    } else {
      const double src = s[v] + ext;
      target[v * N + cell] = target[v * N + cell] + dt * src;
    }
  }
}

template <int ORDER, typename R>
cudaError_t launch_regime_tile(const Grid& g, const double* cons, const double* prims,
                               double* target, double dt, bool ext_only, cudaStream_t st) {
  using T = RegimeTile<ORDER, R>;
  auto kern = k_regime_tile<ORDER, R>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)T::bytes);
  if (e != cudaSuccess) return e;
  const dim3 grid((g.je - g.js + T::TJ - 1) / T::TJ, (g.ie - g.is + T::TI - 1) / T::TI);
  kern<<<grid, T::NT, T::bytes, st>>>(g, cons, prims, target, dt, ext_only);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_regime_tile_order(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     cudaStream_t st, bool ext_only = false) {
  switch (order) {
    case 3: return launch_regime_tile<3, R>(g, cons, prims, target, dt, ext_only, st);
    case 5: return launch_regime_tile<5, R>(g, cons, prims, target, dt, ext_only, st);
    case 7: return launch_regime_tile<7, R>(g, cons, prims, target, dt, ext_only, st);
    case 9: return launch_regime_tile<9, R>(g, cons, prims, target, dt, ext_only, st);
    case 11: return launch_regime_tile<11, R>(g, cons, prims, target, dt, ext_only, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace mth
