// Grid description, reference-layout indexing and in-kernel ghost mapping.
//
// State lives in HBM in METHOD's own layout, ID(var,i,j,k) =
// var*Nx*Ny*Nz + i*Ny*Nz + j*Nz + k (Project/CPU/Include/simData.h:10), with
// Ng ghost cells on each side of every active direction
// (Project/CPU/Src/simData.cc:65-97).  Kernels never read a ghost cell
// directly: a ghost index is mapped onto the interior cell that the
// reference's Bcs::apply would have copied into it (Outflow: nearest
// interior cell; Periodic: the opposite edge; Flow: periodic in x, outflow in
// y and z; Project/CPU/Src/boundaryConds.cc:5-145, 449-733).  Because every
// ghost value of the reference is an exact copy of an interior value, this
// mapping is bit-identical to materialising the ghosts.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mth {

enum BcKind : int { BC_OUTFLOW = 0, BC_PERIODIC = 1, BC_FLOW = 2 };
enum DimBc : int { DIM_NONE = 0, DIM_OUTFLOW = 1, DIM_PERIODIC = 2 };

enum StageMode : int {
  STAGE_FNET = 0,      // out = fnet (FVS::F)
  STAGE_EULER = 1,     // out = in - dt * fnet (RK2 predictor, RK2.cc:58-66)
  STAGE_RK2_CORR = 2,  // out = 0.5 * (u0 + in - dt * fnet) (RK2.cc:81-89)
  // SSP2's closing combination (SSP2.cc:155-166) fused into the stage-2 flux:
  // out = u0 + -0.5 dt (flux1 + fnet - source1 - S(in)), S(in) from the
  // stage state's own cons / aux in registers.
  STAGE_SSP2_FINAL = 3,
};

// Extra inputs of STAGE_SSP2_FINAL: the stage-1 flux and source and cp.
struct StageTail {
  const double* flux1;
  const double* source1;
  double cp;
};

struct Grid {
  int nx, ny, nz;        // interior cells (reference Data::nx..nz; 0 for inactive)
  int Nx, Ny, Nz;        // ghost-inclusive extents
  int Ng, dims;
  int is, ie, js, je, ks, ke;
  int bcx, bcy, bcz;     // DimBc per direction
  double dx, dy, dz;
  double gamma, sigma, cp;
  long long Ntot;        // Nx*Ny*Nz
  double sigma_exp;      // Data::gam, exponent of a functional conductivity
  int functional_sigma;  // Data::functionalSigma
  double sigma_cross;    // Hybrid::sigmaCrossOver
  double sigma_span;     // Hybrid::sigmaSpan
};

// Data::sigmaFunc (simData.cc:114-127): the conductivity of a cell whose
// conserved density is D -- sigma, or sigma * D^gam when it is functional.
__host__ __device__ inline double sigma_of(double sigma, double sigma_exp, int functional,
                                           double D) {
  return functional ? sigma * pow(D, sigma_exp) : sigma;
}
__host__ __device__ inline double sigma_of(const Grid& g, double D) {
  return sigma_of(g.sigma, g.sigma_exp, g.functional_sigma, D);
}

__host__ __device__ inline long long cell_id(const Grid& g, int i, int j, int k) {
  return ((long long)i * g.Ny + j) * g.Nz + k;
}

// Interior cell number t (k fastest) -> (i, j, k), and the interior count.
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

inline long long n_interior_host(const Grid& g) {
  return (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
}

// Maps an index of one direction onto the interior cell whose value the
// reference's boundary pass would have copied there.
__host__ __device__ inline int map_dim(int i, int n, int Ng, int kind) {
  if (kind == DIM_PERIODIC) {
    if (i < Ng) return i + n;
    if (i >= n + Ng) return i - n;
    return i;
  }
  if (kind == DIM_OUTFLOW) {
    if (i < Ng) return Ng;
    if (i > n + Ng - 1) return n + Ng - 1;
    return i;
  }
  return i;
}

__host__ __device__ inline long long mapped_cell(const Grid& g, int i, int j, int k) {
  return cell_id(g, map_dim(i, g.nx, g.Ng, g.bcx), map_dim(j, g.ny, g.Ng, g.bcy),
                 map_dim(k, g.nz, g.Ng, g.bcz));
}

#ifdef __CUDACC__
// Read-only input load: through the non-coherent path (`__ldg`, which the
// compiler keeps even when the value is unused), or as a plain load that it
// may drop when nothing uses the value.
template <bool LDG>
__device__ __forceinline__ double ld_in(const double* __restrict__ p) {
  if constexpr (LDG)
    return __ldg(p);
  else
    return *p;
}
#endif

}  // namespace mth
