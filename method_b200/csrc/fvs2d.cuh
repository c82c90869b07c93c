// Fused 2D flux-vector-splitting stage kernel.
//
// One CTA owns a TI x 32 tile of interior cells (32 consecutive j per warp, the
// contiguous direction of METHOD's layout).  For each direction it
//   1. loads the tile plus a halo of H cells along that direction, mapping
//      ghost indices onto the interior (in-kernel boundary conditions),
//   2. evaluates Model::fluxVector and the Lax-Friedrichs split
//      f+- = 0.5 (f +- U) (Project/CPU/Src/fluxVectorSplitting.cc:22-33) into
//      shared memory,
//   3. reconstructs every face with WENO upwind(f+) + downwind(f-)
//      (fluxVectorSplitting.cc:36-49, weno.cc:123-228),
//   4. forms fnet = (fx[i+1]/dx - fx[i]/dx) + (fy[j+1]/dy - fy[j]/dy)
//      (fluxVectorSplitting.cc:105-111) in registers,
// and finally applies the Runge-Kutta stage update to its own cells, so a
// stage reads each state array once and writes the new conserved state once.
//
// `R` is the arithmetic type of flux, split and reconstruction: double in the
// plain form (compiled without FMA, bit-identical to the reference), float in
// the mixed form.  The conserved-state update is always FP64.
#pragma once
#include "common.cuh"
#include "weno.cuh"
#include "weno_hi.cuh"

namespace mth {

// The upwind point reconstruction of order ORDER (3 .. 11) on the values
// v[q * stride], q = 0 .. ORDER-1, walking forwards (dir = +1) or backwards.
template <int ORDER, typename R>
__device__ __forceinline__ R weno_point(const R* v, int stride) {
#define V(q) v[(q) * stride]
  if constexpr (sizeof(R) == 8) {
    if constexpr (ORDER == 7) return weno7_exact(V(0), V(1), V(2), V(3), V(4), V(5), V(6));
    if constexpr (ORDER == 9)
      return weno9_exact(V(0), V(1), V(2), V(3), V(4), V(5), V(6), V(7), V(8));
    if constexpr (ORDER == 11)
      return weno11_exact(V(0), V(1), V(2), V(3), V(4), V(5), V(6), V(7), V(8), V(9), V(10));
  } else {
    if constexpr (ORDER == 7) return weno7_fast(V(0), V(1), V(2), V(3), V(4), V(5), V(6));
    if constexpr (ORDER == 9)
      return weno9_fast(V(0), V(1), V(2), V(3), V(4), V(5), V(6), V(7), V(8));
    if constexpr (ORDER == 11)
      return weno11_fast(V(0), V(1), V(2), V(3), V(4), V(5), V(6), V(7), V(8), V(9), V(10));
  }
#undef V
  return R(0);
}

template <int ORDER, typename R>
__device__ __forceinline__ R weno_face(const R* p, const R* m, int stride, int base) {
  // p, m point at the first stencil cell of the region column; `base` is the
  // region index of cell i-H for face i (face between cells i-1 and i).
  if constexpr (ORDER >= 7) {
    // upwind cells i-H .. i-H+ORDER-1; downwind cells i+H-1 down to i+H-ORDER
    // (weno.cc:239-482): the region indices base .. base+ORDER-1 and
    // base+ORDER down to base+1
    return weno_point<ORDER, R>(p + base * stride, stride) +
           weno_point<ORDER, R>(m + (base + ORDER) * stride, -stride);
  } else if constexpr (ORDER == 3) {
    // upwind cells i-2, i-1, i ; downwind cells i+1, i, i-1 (weno.cc:123-164)
    if constexpr (sizeof(R) == 8) {
      return weno3_exact(p[(base + 0) * stride], p[(base + 1) * stride], p[(base + 2) * stride]) +
             weno3_exact(m[(base + 3) * stride], m[(base + 2) * stride], m[(base + 1) * stride]);
    } else {
      const float2 r = weno3_fast2(make_float2(p[(base + 0) * stride], m[(base + 3) * stride]),
                                   make_float2(p[(base + 1) * stride], m[(base + 2) * stride]),
                                   make_float2(p[(base + 2) * stride], m[(base + 1) * stride]));
      return r.x + r.y;
    }
  } else {
    // upwind cells i-3 .. i+1 ; downwind cells i+2 .. i-2 (weno.cc:175-228)
    if constexpr (sizeof(R) == 8) {
      return weno5_exact(p[(base + 0) * stride], p[(base + 1) * stride], p[(base + 2) * stride],
                         p[(base + 3) * stride], p[(base + 4) * stride]) +
             weno5_exact(m[(base + 5) * stride], m[(base + 4) * stride], m[(base + 3) * stride],
                         m[(base + 2) * stride], m[(base + 1) * stride]);
    } else {
      const float2 r = weno5_fast2(make_float2(p[(base + 0) * stride], m[(base + 5) * stride]),
                                   make_float2(p[(base + 1) * stride], m[(base + 4) * stride]),
                                   make_float2(p[(base + 2) * stride], m[(base + 3) * stride]),
                                   make_float2(p[(base + 3) * stride], m[(base + 2) * stride]),
                                   make_float2(p[(base + 4) * stride], m[(base + 1) * stride]));
      return r.x + r.y;
    }
  }
}

// Halo of a face reconstruction: the reference's WENO shift (order + 1) / 2.
template <int ORDER>
struct Halo {
  static constexpr int H = (ORDER + 1) / 2;
};

template <class M, typename R, int ORDER, int TI>
struct Fvs2dSmem {
  static constexpr int TJ = 32;
  static constexpr int H = Halo<ORDER>::H;
  static constexpr int RX = (TI + 2 * H) * TJ;
  static constexpr int RY = TI * (TJ + 2 * H);
  static constexpr int RMAX = RX > RY ? RX : RY;
  static constexpr int FX = (TI + 1) * TJ;
  static constexpr int FY = TI * (TJ + 1);
  static constexpr int FMAX = FX > FY ? FX : FY;
  static constexpr size_t bytes = sizeof(R) * (size_t)M::NC * (2 * RMAX + FMAX);
};

// CTAs per SM the FP32 tile's register allocation is sized for: enough for
// 1024 resident threads (32 warps, 64 registers each) where shared memory
// admits them (OT 1024^2 WENO5, TI 8: 0.220 -> 0.179 ms per launch against
// the compiler's own 80-register choice).  The FP64 tile keeps the compiler's
// choice (its shared memory admits two CTAs).
template <class M, typename R, int ORDER, int TI>
constexpr int fvs2d_min_blocks() {
  if (sizeof(R) == 8) return 1;
  const int by_smem = (int)(220 * 1024 / Fvs2dSmem<M, R, ORDER, TI>::bytes);
  const int by_threads = 1024 / (32 * TI);
  const int b = by_smem < by_threads ? by_smem : by_threads;
  return b < 1 ? 1 : b;
}

// Loads one cell's flux inputs (in R) and writes f+ and f- of direction `dir`.
template <class M, typename R>
__device__ __forceinline__ void split_cell(const Grid& g, const double* __restrict__ cons,
                                           const double* __restrict__ prims,
                                           const double* __restrict__ aux, long long cell, int dir,
                                           R* sp, R* sm, int stride) {
  R c[M::NC], p[M::NP], a[M::NA];
  M::template load_flux_inputs<R>(cons, prims, aux, g.Ntot, cell, c, p, a);
  R f[M::NC];
  M::template flux_g<R>(g, c, p, a, dir, f);
#pragma unroll
  for (int v = 0; v < M::NC; ++v) {
    if constexpr (sizeof(R) == 4) {
      // 0.5 f +- 0.5 c in one FP32x2 FMA: the same values, as halving is exact
      const float2 h = __ffma2_rn(make_float2(f[v], f[v]), f2(0.5f),
                                  __fmul2_rn(make_float2(c[v], c[v]), make_float2(0.5f, -0.5f)));
      sp[v * stride] = h.x;
      sm[v * stride] = h.y;
    } else {
      sp[v * stride] = R(0.5) * (f[v] + c[v]);
      sm[v * stride] = R(0.5) * (f[v] - c[v]);
    }
  }
}

// Flux difference of one cell along one direction, f_right / d - f_left / d
// (fluxVectorSplitting.cc:105-111): exactly so in FP64; in the FP32 form
// through one reciprocal of the cell size.
template <typename R>
__device__ __forceinline__ R face_diff(R right, R left, R d) {
  if constexpr (sizeof(R) == 8) {
    return right / d - left / d;
  } else {
    const R inv = R(1) / d;
    return right * inv - left * inv;
  }
}

// The stage's output for one interior cell from its flux difference `acc`
// (fnet of FVS::F): fnet itself, the Euler step U - dt fnet, the RK2
// corrector 1/2 (U^n + U^1 - dt fnet), or SSP2's final combination
// cons += -0.5 dt (flux1 + flux2 - source1 - source2) in the reference's
// order (SSP2.cc:155-166) with flux2 = fnet and source2 = S(stage state).
template <class M, typename R>
__device__ __forceinline__ void stage_update(const Grid& g, const double* __restrict__ cons,
                                             const double* __restrict__ aux, const double* u0,
                                             double* out, double dt, int mode,
                                             const StageTail& tail, long long cell,
                                             const R* acc) {
  constexpr int NC = M::NC;
  if (mode == STAGE_SSP2_FINAL) {
    double s2[NC];
    M::cell_source(cons, aux, g.Ntot, cell, tail.cp, s2);
#pragma unroll
    for (int v = 0; v < NC; ++v) {
      const long long o = (long long)v * g.Ntot + cell;
      out[o] = u0[o] + -0.5 * dt * (tail.flux1[o] + (double)acc[v] - tail.source1[o] - s2[v]);
    }
    return;
  }
#pragma unroll
  for (int v = 0; v < NC; ++v) {
    const long long o = (long long)v * g.Ntot + cell;
    const double fn = (double)acc[v];
    if (mode == STAGE_FNET) {
      out[o] = fn;
    } else if (mode == STAGE_EULER) {
      out[o] = cons[o] - dt * fn;
    } else {
      out[o] = 0.5 * (u0[o] + cons[o] - dt * fn);
    }
  }
}

// The epilogue's inputs that no earlier phase of the stage reads (U^n of
// the RK2 corrector; U^n, flux1 and source1 of SSP2's final combination),
// requested into L2 when the tile starts so that their latency overlaps the
// flux phases (OT 1024^2 corrector tile: 0.154 -> 0.151 ms average launch).
template <class M>
__device__ __forceinline__ void prefetch_tail(const Grid& g, const double* u0, int mode,
                                              const StageTail& tail, long long cell) {
  if (mode != STAGE_RK2_CORR && mode != STAGE_SSP2_FINAL) return;
#pragma unroll
  for (int v = 0; v < M::NC; ++v) {
    const long long o = (long long)v * g.Ntot + cell;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(u0 + o));
    if (mode == STAGE_SSP2_FINAL) {
      asm volatile("prefetch.global.L2 [%0];" ::"l"(tail.flux1 + o));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(tail.source1 + o));
    }
  }
}

// One TI x 32 tile (tile row ti, tile column tj) of the fused stage; the
// whole CTA participates and `smem_raw` holds Fvs2dSmem::bytes.
template <class M, typename R, int ORDER, int TI>
__device__ __forceinline__ void fvs2d_tile(const Grid& g, const double* __restrict__ cons,
                                           const double* __restrict__ prims,
                                           const double* __restrict__ aux, const double* u0,
                                           double* out, double dt, int mode, int ti, int tj,
                                           unsigned char* smem_raw, StageTail tail = {}) {
  using S = Fvs2dSmem<M, R, ORDER, TI>;
  constexpr int NC = M::NC, TJ = S::TJ, H = S::H, NT = 32 * TI;
  R* sp = reinterpret_cast<R*>(smem_raw);
  R* sm = sp + NC * S::RMAX;
  R* sr = sm + NC * S::RMAX;

  const int lane = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + lane;
  const int i0 = g.is + ti * TI, j0 = g.js + tj * TJ;
  const int ci = i0 + ty, cj = j0 + lane;
  R acc[NC];
  if (ci < g.ie && cj < g.je) prefetch_tail<M>(g, u0, mode, tail, cell_id(g, ci, cj, 0));

  // ---------------- x direction ----------------
  for (int e = tid; e < S::RX; e += NT) {
    int r = e / TJ, c = e - r * TJ;
    int gi = min(i0 - H + r, g.ie - 1 + H);
    int gj = min(j0 + c, g.je - 1);
    split_cell<M, R>(g, cons, prims, aux, mapped_cell(g, gi, gj, 0), 0, sp + e, sm + e, S::RX);
  }
  __syncthreads();
  // Item e = (v, fi, lane): a step of NT items is TI rows of faces, so the
  // lane stays fixed and (v, fi) advance without a division.
  for (int e = tid, v = 0, fi = ty; e < NC * S::FX; e += NT) {
    const R* P = sp + v * S::RX + lane;
    const R* Mm = sm + v * S::RX + lane;
    // face i0+fi: cell i-H sits at region row fi
    sr[e] = weno_face<ORDER, R>(P, Mm, TJ, fi);
    fi += TI;
    if (fi > TI) {
      fi -= TI + 1;
      ++v;
    }
  }
  __syncthreads();
  {
    const R dx = R(g.dx);
#pragma unroll
    for (int v = 0; v < NC; ++v)
      acc[v] = face_diff<R>(sr[v * S::FX + (ty + 1) * TJ + lane], sr[v * S::FX + ty * TJ + lane],
                            dx);
  }
  __syncthreads();

  // ---------------- y direction ----------------
  constexpr int WY = TJ + 2 * H;
  for (int e = tid; e < S::RY; e += NT) {
    int r = e / WY, c = e - r * WY;
    int gi = min(i0 + r, g.ie - 1);
    int gj = min(j0 - H + c, g.je - 1 + H);
    split_cell<M, R>(g, cons, prims, aux, mapped_cell(g, gi, gj, 0), 1, sp + e, sm + e, S::RY);
  }
  __syncthreads();
  // Item e = (v, r, fj), rows of TJ + 1 faces; (v, r, fj) advance by NT items
  // a step without a division (NT < FY, so v grows by one at most).
  {
    constexpr int RS = NT / (TJ + 1), FS = NT % (TJ + 1);
    int v = 0, r = tid / (TJ + 1), fj = tid % (TJ + 1);
    for (int e = tid; e < NC * S::FY; e += NT) {
      const R* P = sp + v * S::RY + r * WY;
      const R* Mm = sm + v * S::RY + r * WY;
      sr[e] = weno_face<ORDER, R>(P, Mm, 1, fj);
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
  if (ci < g.ie && cj < g.je) {
    const R dy = R(g.dy);
#pragma unroll
    for (int v = 0; v < NC; ++v)
      acc[v] = acc[v] + face_diff<R>(sr[v * S::FY + ty * (TJ + 1) + lane + 1],
                                     sr[v * S::FY + ty * (TJ + 1) + lane], dy);

    stage_update<M, R>(g, cons, aux, u0, out, dt, mode, tail, cell_id(g, ci, cj, 0), acc);
  }
}

template <class M, typename R, int ORDER, int TI>
__global__ void __launch_bounds__(32 * TI, (fvs2d_min_blocks<M, R, ORDER, TI>()))
    k_fvs2d(Grid g, const double* __restrict__ cons, const double* __restrict__ prims,
            const double* __restrict__ aux, const double* u0, double* out, double dt,
            int mode, StageTail tail, int ti0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fvs2d_tile<M, R, ORDER, TI>(g, cons, prims, aux, u0, out, dt, mode, ti0 + blockIdx.y,
                              blockIdx.x, smem_raw, tail);
}

}  // namespace mth
