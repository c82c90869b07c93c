// Fused 2D flux stage, plain FP64 form, conserved variables in groups.
//
// The FP64 tile of fvs2d.cuh keeps f+ and f- of all NC variables of its
// tile-plus-halo region in shared memory (85 KB for SRMHD WENO5 at 8 x 32),
// which with its register count holds two CTAs, 16 warps, on an SM; its
// WENO chains (IEEE divisions, no FMA contraction, the reference's order)
// then wait on FP64 latency with too few warps to cover it.  This form runs
// the same tile as G-variable passes: each pass loads the region's flux
// inputs, evaluates the flux of only its G variables (the compiler drops
// the rest, loads included, as they are plain loads), splits, reconstructs
// and accumulates their x and then y differences in registers.  Shared memory
// shrinks by NC / G and the register cap admits more CTAs per SM.  Every
// value is computed by the same expression as in the one-pass tile, so the
// result is bit-identical to it and to the reference.
#pragma once
#include "fvs2d.cuh"

namespace mth {

template <class M, int ORDER, int TI, int G>
struct Fvs2dGroupSmem {
  using B = Fvs2dSmem<M, double, ORDER, TI>;
  static constexpr int NG = (M::NC + G - 1) / G;
  static constexpr size_t bytes = sizeof(double) * (size_t)G * (2 * B::RMAX + B::FMAX);
};

// Flux inputs of one cell by plain loads, its flux along `dir`, and the
// Lax-Friedrichs split of variables [V0, V0 + NV).
template <class M, int V0, int NV>
__device__ __forceinline__ void split_group(const Grid& g, const double* __restrict__ cons,
                                            const double* __restrict__ prims,
                                            const double* __restrict__ aux, long long cell,
                                            int dir, double* sp, double* sm, int stride) {
  double c[M::NC], p[M::NP], a[M::NA];
  M::template load_flux_inputs<double, false>(cons, prims, aux, g.Ntot, cell, c, p, a);
  double f[M::NC];
  M::template flux_g<double>(g, c, p, a, dir, f);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    sp[v * stride] = 0.5 * (f[V0 + v] + c[V0 + v]);
    sm[v * stride] = 0.5 * (f[V0 + v] - c[V0 + v]);
  }
}

// Pass Q: the x and y flux differences of variables [Q G, Q G + NV) into
// acc.  Ends with a barrier, so the next pass may reuse shared memory.
template <class M, int ORDER, int TI, int G, int Q>
__device__ __forceinline__ void group_pass(const Grid& g, const double* __restrict__ cons,
                                           const double* __restrict__ prims,
                                           const double* __restrict__ aux, int i0, int j0,
                                           double* acc, unsigned char* smem_raw) {
  using S = Fvs2dSmem<M, double, ORDER, TI>;
  constexpr int V0 = Q * G, NV = M::NC - V0 < G ? M::NC - V0 : G;
  constexpr int TJ = S::TJ, H = S::H, NT = 32 * TI, WY = TJ + 2 * H;
  double* sp = reinterpret_cast<double*>(smem_raw);
  double* sm = sp + G * S::RMAX;
  double* sr = sm + G * S::RMAX;
  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;

  // x direction: region rows i0-H .. i0+TI+H-1, faces as in fvs2d_tile
  for (int e = tid; e < S::RX; e += NT) {
    const int r = e / TJ, c = e - r * TJ;
    const int gi = min(i0 - H + r, g.ie - 1 + H);
    const int gj = min(j0 + c, g.je - 1);
    split_group<M, V0, NV>(g, cons, prims, aux, mapped_cell(g, gi, gj, 0), 0, sp + e, sm + e,
                           S::RX);
  }
  __syncthreads();
  for (int e = tid, v = 0, fi = ty; e < NV * S::FX; e += NT) {
    sr[e] = weno_face<ORDER, double>(sp + v * S::RX + lane, sm + v * S::RX + lane, TJ, fi);
    fi += TI;
    if (fi > TI) {
      fi -= TI + 1;
      ++v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NV; ++v)
    acc[V0 + v] = face_diff<double>(sr[v * S::FX + (ty + 1) * TJ + lane],
                                    sr[v * S::FX + ty * TJ + lane], g.dx);
  __syncthreads();

  // y direction: region columns j0-H .. j0+TJ+H-1
  for (int e = tid; e < S::RY; e += NT) {
    const int r = e / WY, c = e - r * WY;
    const int gi = min(i0 + r, g.ie - 1);
    const int gj = min(j0 - H + c, g.je - 1 + H);
    split_group<M, V0, NV>(g, cons, prims, aux, mapped_cell(g, gi, gj, 0), 1, sp + e, sm + e,
                           S::RY);
  }
  __syncthreads();
  {
    constexpr int RS = NT / (TJ + 1), FS = NT % (TJ + 1);
    int v = 0, r = tid / (TJ + 1), fj = tid % (TJ + 1);
    for (int e = tid; e < NV * S::FY; e += NT) {
      sr[e] = weno_face<ORDER, double>(sp + v * S::RY + r * WY, sm + v * S::RY + r * WY, 1, fj);
      fj += FS;
      r += RS;
      if (fj > TJ) {
        fj -= TJ + 1;
        ++r;
      }
      if (r >= TI) {
        r -= TI;
        ++v;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NV; ++v)
    acc[V0 + v] = acc[V0 + v] + face_diff<double>(sr[v * S::FY + ty * (TJ + 1) + lane + 1],
                                                  sr[v * S::FY + ty * (TJ + 1) + lane], g.dy);
  __syncthreads();
  if constexpr (Q + 1 < Fvs2dGroupSmem<M, ORDER, TI, G>::NG)
    group_pass<M, ORDER, TI, G, Q + 1>(g, cons, prims, aux, i0, j0, acc, smem_raw);
}

template <class M, int ORDER, int TI, int G, int MINB>
__global__ void __launch_bounds__(32 * TI, MINB)
    k_fvs2d_group(Grid g, const double* __restrict__ cons, const double* __restrict__ prims,
                  const double* __restrict__ aux, const double* u0, double* out, double dt,
                  int mode, StageTail tail) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int i0 = g.is + blockIdx.y * TI, j0 = g.js + blockIdx.x * 32;
  const int ci = i0 + threadIdx.y, cj = j0 + threadIdx.x;
  if (ci < g.ie && cj < g.je) prefetch_tail<M>(g, u0, mode, tail, cell_id(g, ci, cj, 0));
  double acc[M::NC];
  group_pass<M, ORDER, TI, G, 0>(g, cons, prims, aux, i0, j0, acc, smem_raw);
  if (ci < g.ie && cj < g.je)
    stage_update<M, double>(g, cons, aux, u0, out, dt, mode, tail, cell_id(g, ci, cj, 0), acc);
}

}  // namespace mth
