// Mixed-precision ("chosen") form: FP32 flux / WENO, FP64 primitive recovery by
// a 1D Newton iteration whose initial guess comes from the previous state or
// from the learned guess network, FP64 conserved-state accumulation.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "launch.h"

namespace mth {

// Guess network 8 -> 64 -> 64 -> 64 -> 2 (BF16 weights, FP32 accumulate).
constexpr int MLP_IN = 8, MLP_H = 64, MLP_OUT = 2;
constexpr int MLP_NPARAM = MLP_IN * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H +
                           MLP_H * MLP_OUT + MLP_OUT;

struct MixedWork {
  void* mlp_params = nullptr;   // bf16 parameters, packed (W1,b1,W2,b2,W3,b3,W4,b4)
  float* feat_stats = nullptr;  // input normalisation: mean[8], inv_std[8]; output: mean[2], std[2]
  double* zguess = nullptr;     // per-cell Z guess written by the network (Ntot)
  int has_mlp = 0;
};

cudaError_t mixed_init(MixedWork* w, const Grid& g, int model, cudaStream_t st);
void mixed_free(MixedWork* w);

cudaError_t launch_fvs2d_fp32(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st);

// guess: 0 = previous state, 1 = guess network (falls back to the previous
// state, then to the reference Powell-hybrid, when Newton does not converge).
cudaError_t launch_c2p_mixed(const Grid& g, int model, int guess, const double* cons,
                             const double* prims_guess, const double* aux_guess, double* prims,
                             double* aux, double* solution, C2PWork w, const MixedWork& mw,
                             cudaStream_t st);

}  // namespace mth
