// The Hybrid model's per-cell formulas (hybrid.cc) shared by the generic
// kernels (hybrid.cu) and the fused 2D flux tile (HYBRID below, used by
// kernels_fp64.cu).  Compiled without FMA contraction in both units.
#pragma once
#include "common.cuh"
#include "srmhd.cuh"
#include "srrmhd.cuh"

namespace mth {

// Hybrid::idealWeight (hybrid.cc:115-131): 0 below sigmaCrossOver -
// sigmaSpan, 1 above sigmaCrossOver + sigmaSpan, a tanh ramp between.
__device__ __forceinline__ double ideal_weight(const Grid& g, double sig) {
  return sig < g.sigma_cross - g.sigma_span
             ? 0
             : sig < g.sigma_cross + g.sigma_span
                   ? (tanh((sig - g.sigma_cross) / (g.sigma_span / 3)) + 1) / 2
                   : 1;
}

// Hybrid::setIdealCPAs (hybrid.cc:139-168): the SRMHD cons (9), prims (8) and
// aux (13) of one cell from its resistive cons (14), prims (11) and aux (17).
template <typename R>
__device__ __forceinline__ void ideal_cpas(const R* rc, const R* rp, const R* ra, R* c, R* p,
                                           R* a) {
  for (int v = 0; v < 8; ++v) c[v] = rc[v];
  c[8] = rc[12];
  for (int v = 0; v < 8; ++v) p[v] = rp[v];
  for (int v = 0; v < 4; ++v) a[v] = ra[v];
  const R b0 = ra[1] * (rp[5] * rp[1] + rp[6] * rp[2] + rp[7] * rp[3]);
  const R bx = rp[5] / ra[1] + b0 * rp[1];
  const R by = rp[6] / ra[1] + b0 * rp[2];
  const R bz = rp[7] / ra[1] + b0 * rp[3];
  const R bsq = (rp[5] * rp[5] + rp[6] * rp[6] + rp[7] * rp[7] + b0 * b0) / (ra[1] * ra[1]);
  const R BS = ra[1] * (rp[5] * rc[1] + rp[6] * rc[2] + rp[7] * rc[3]);
  const R Ssq = rc[1] * rc[1] + rc[2] * rc[2] + rc[3] * rc[3];
  a[4] = b0;
  a[5] = bx;
  a[6] = by;
  a[7] = bz;
  a[8] = bsq;
  a[9] = ra[9];
  a[10] = BS;
  a[11] = ra[7];
  a[12] = Ssq;
}

// Hybrid::fluxVector of one cell (hybrid.cc:210-259): f = (1 - w) f_resistive,
// then + w f_ideal on D, S, tau, B and + w f_ideal(phi) on phi.
// R = float: the mixed form's flux (the weight from the FP64 conductivity).
template <typename R>
__device__ __forceinline__ void hybrid_flux(const Grid& g, const R* c, const R* p, const R* a,
                                            int dir, R* f) {
  const R iW = R(ideal_weight(g, sigma_of(g, double(c[0]))));
  R ic[9], ip[8], ia[13], fi[9];
  ideal_cpas<R>(c, p, a, ic, ip, ia);
  srmhd::flux<R>(ic, ip, ia, dir, fi);
  srrmhd::flux<R>(c, p, a, dir, f);
  for (int v = 0; v < 14; ++v) f[v] = (1 - iW) * f[v];
  for (int v = 0; v < 8; ++v) f[v] += iW * fi[v];
  f[12] += iW * fi[8];
}

// The model interface of the fused flux tiles (fvs2d.cuh, fvs2d_group.cuh).
struct HYBRID {
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
    for (int v = 0; v < NP; ++v) p[v] = R(ld_in<LDG>(prims + v * N + cell));
#pragma unroll
    for (int v = 0; v < NA; ++v) a[v] = R(ld_in<LDG>(aux + v * N + cell));
  }
  template <typename R>
  __device__ __forceinline__ static void flux_g(const Grid& g, const R* c, const R* p, const R* a,
                                                int dir, R* f) {
    hybrid_flux<R>(g, c, p, a, dir, f);
  }
  // The SSP2 closing stage does not run with this model (RK2 and RKSplit2
  // only); the tile's stage epilogue still names a cell source.
  __device__ __forceinline__ static void cell_source(const double* __restrict__,
                                                     const double* __restrict__, long long,
                                                     long long, double, double* s) {
#pragma unroll
    for (int v = 0; v < NC; ++v) s[v] = 0.0;
  }
};

}  // namespace mth
