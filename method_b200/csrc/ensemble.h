// Ensembles of independent simulations advanced together.
//
// Every member keeps its own grid, state arrays, time, step counter and dt
// in a device-resident descriptor.  A phase of the time step (flux stage,
// primitive recovery, implicit stage, ...) is ONE persistent launch for all
// members: CTAs stride over a work list of (member, tile) or (member, cell
// chunk) items, so uneven member sizes share the SMs without one launch per
// member.  dt follows Simulation::updateTime per member on the device, so the
// captured step graph needs no host data and replays unchanged.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace mth {

enum EnsArray : int {
  EA_CONS = 0, EA_PRIMS, EA_AUX,
  EA_P1C, EA_P1P, EA_P1A,            // RK2 predictor state
  EA_U1, EA_U2, EA_F1, EA_S1,        // SSP2 stages (F(U2), S(U2) stay in registers)
  EA_SOL,                            // SRMHD C2P solution (2 planes)
  EA_ZG,                             // learned guess (Z, v^2 planes)
  EA_COUNT
};

struct Member {
  Grid g;
  double cfl, endTime, t, dt;
  int iters, model, integrator, pad;
  double* a[EA_COUNT];
  int* fail_list;     // Ntot ints
  int* fail_count;    // 1 int
  long long* counters;  // 16: as the single-simulation counters
};

// Work items: x = member, y = tile row (or first cell), z = tile column.
struct Item {
  int m, a, b, pad;
};

// ---- plain FP64 (kernels_fp64.cu) ----
cudaError_t ens_fvs_fp64(const Member* mem, const Item* items, int n_items, int model, int order,
                         int TI, int ic, int ip, int ia, int iu0, int iout, int mode, int grid,
                         cudaStream_t st);
cudaError_t ens_c2p_srmhd_hybrd(const Member* mem, const Item* items, int n_items, int ic,
                                int ipg, int iag, int ip, int ia, int grid, cudaStream_t st);
cudaError_t ens_c2p_retry(const Member* mem, int n_members, int ic, int ip, int ia,
                          cudaStream_t st);
// Reference (hybrd1) implicit solve of the cells queued by ens_imex_fast.
cudaError_t ens_imex_queued(const Member* mem, int n_members, int stage, cudaStream_t st);
cudaError_t ens_source(const Member* mem, const Item* items, int n_items, int ic, int ia,
                       int iout, int grid, cudaStream_t st);
cudaError_t ens_dt(Member* mem, int n_members, cudaStream_t st);
cudaError_t ens_advance(Member* mem, int n_members, cudaStream_t st);

// ---- mixed form (kernels_mixed.cu) ----
cudaError_t ens_fvs_fp32(const Member* mem, const Item* items, int n_items, int model, int order,
                         int TI, int ic, int ip, int ia, int iu0, int iout, int mode, int grid,
                         cudaStream_t st);
// guess_mode 1: members start Newton from the learned guess in EA_ZG.
// lean: write only what the stage's flux, source and next implicit solve read
// (SRMHD: prims 1-7, aux 1 and 4-8, no solution; SRRMHD: prims 1-4, aux 4-8
// and 10), for the intermediate recovered states of RK2 and SSP2.
cudaError_t ens_c2p_newton(const Member* mem, const Item* items, int n_items, int model,
                           int guess_mode, int ic, int ipg, int iag, int ip, int ia, bool lean,
                           int grid, cudaStream_t st);
// guess_mode 1: the inner recoveries start from the learned guess in EA_ZG.
cudaError_t ens_imex_fast(const Member* mem, const Item* items, int n_items, int stage, int grid,
                          cudaStream_t st, int guess_mode = 0);
// Stage 2's explicit part of every SRRMHD member into EA_U2 (the network's input).
cudaError_t ens_imex_explicit_part2(const Member* mem, const Item* items, int n_items, int grid,
                                    cudaStream_t st);
// ---- guess network (mlp.cu): EA_ZG of one model's members from state `ic`.
cudaError_t ens_mlp_zguess(const Member* mem, const Item* items, int n_items, int ic,
                           const float* params, const float* stats, int grid, cudaStream_t st,
                           int model = 0);

constexpr int ENS_CHUNK = 128;  // cells per cell-phase work item (= CTA size)

}  // namespace mth
