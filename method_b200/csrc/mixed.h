// Mixed-precision ("chosen") form: FP32 flux / WENO, FP64 primitive recovery by
// a 1D Newton iteration whose initial guess comes from the previous state or
// from the learned guess network, FP64 conserved-state accumulation.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "launch.h"

namespace mth {

// Guess network 8 -> 64 -> 64 -> 64 -> 2 (BF16 weights, FP32 accumulate);
// packed parameter count of the layout in mlp.cuh (padding included).
constexpr int MLP_NPARAM = 9928;
constexpr int MLP_NSTAT = 20;

struct MixedWork {
  float* mlp_params = nullptr;  // FP32 master parameters (mlp.cuh layout), cast to BF16 on load
  float* feat_stats = nullptr;  // feature mean[8], inv_std[8]; target mean[2], std[2]
  double* zguess = nullptr;     // per-cell (Z, v^2) guesses written by the network (2 x Ntot)
  int has_mlp = 0;
};

namespace mlp {
size_t smem_bytes();
cudaError_t configure();
// model 0: SRMHD features of cons (9 vars); 1: SRRMHD (14 vars).
// Runs on the tcgen05 path (mlp_tc.cu); a bounded wait there that runs out
// sets ERR_DEVICE in *err when err is given.
cudaError_t launch_zguess(const Grid& g, long long n_cells, bool batch, const double* cons,
                          const float* P, const float* st, double* zguess, cudaStream_t s,
                          int model = 0, long long* err = nullptr);
}  // namespace mlp

// SSP2 implicit stage of the mixed form (closed-form psi/phi, Newton on E).
// SSP3(332) / SSP2(322) implicit stage `form` (as launch_imex_sweep) in the
// mixed form, with the exact solve for the cells it cannot converge.
cudaError_t launch_imex_fast_form(const Grid& g, int form, const double* cons,
                                  const double* zaux, const double* u1, const double* u2,
                                  const double* flux1, const double* flux2,
                                  const double* source1, const double* source2, double* out,
                                  double* zout, double dt, C2PWork w, cudaStream_t st);
// mw (may be null): with a guess network installed, the inner recoveries
// start from its Z for the stage's first iterate.
cudaError_t launch_imex_fast(const Grid& g, int stage, const double* cons,
                             const double* aux_guess, const double* u1, const double* flux1,
                             const double* source1, double* out, double dt, C2PWork w,
                             cudaStream_t st, const MixedWork* mw = nullptr);

// Batched primitive recovery of independent cells (variable-major, stride n).
// method: 0 Powell hybrid (reference), 1 Newton; guess: 0 previous state,
// 1 network (zguess planes), 2 cold start.  counters: cells, iterations,
// unconverged, fallbacks.
cudaError_t launch_c2p_batch(long long n, double gamma, int method, int guess,
                             const double* cons, double* prims, double* aux,
                             const double* zguess, long long* counters, cudaStream_t st);

cudaError_t mixed_init(MixedWork* w, const Grid& g, int model, cudaStream_t st);
void mixed_free(MixedWork* w);

// ti0, nti: the tile rows (of 8 interior rows) to update; all by default.
cudaError_t launch_fvs2d_fp32(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st,
                              StageTail tail = {}, int ti0 = 0, int nti = -1);

// guess: 0 = previous state, 1 = guess network (falls back to the previous
// state, then to the reference Powell-hybrid, when Newton does not converge).
// lean: write only what the flux tile, the source and the next implicit solve
// read back (SRMHD: prims 1-7, aux 1 and 4-8, no solution; SRRMHD: prims 1-4,
// aux 4-8 and 10), for an intermediate recovered state.
// t0, nt: the range of interior cells (k fastest, then j, then i) to
// recover; all by default.
cudaError_t launch_c2p_mixed(const Grid& g, int model, int guess, const double* cons,
                             const double* prims_guess, const double* aux_guess, double* prims,
                             double* aux, double* solution, C2PWork w, const MixedWork& mw,
                             bool lean, cudaStream_t st, long long t0 = 0, long long nt = -1);

}  // namespace mth
