// Host-side launchers shared between the kernel translation units and the
// C-ABI.  Every launcher enqueues on `st` and returns the launch status.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "common.cuh"

namespace mth {

enum ModelId : int { MODEL_SRMHD = 0, MODEL_SRRMHD = 1, MODEL_HYBRID = 2 };

// Per-call C2P bookkeeping on the device.
struct C2PWork {
  int* fail_list;         // capacity Ntot cell ids
  int* fail_count;        // [0] = failures of the current call
  long long* counters;    // [0] cells, [1] nfev sum, [2] cells failed, [3] sticky error flags
};

enum ErrFlag : long long {
  ERR_C2P = 1,       // primitive recovery did not converge
  ERR_IMPLICIT = 2,  // implicit source solve did not converge
  ERR_DEVICE = 4,    // a bounded device-side wait ran out (tensor-core inference)
};

// Data::initData geometry (simData.cc:61-97) for a configuration; returns
// false for a configuration the reference rejects.  `c` is an mth_config.
bool grid_from_config(const void* c, Grid* g);

// Body of a SerialSaveData array file (textout.cu): every interior value of
// nvars variables as printf's "%.16f " with the reference's line breaks.
cudaError_t format_body(const Grid& g, const double* arr, int nvars, std::string& out,
                        cudaStream_t st);

// ---- plain FP64 (bit-compatible with the reference) --------------------------
cudaError_t launch_prims_to_all(const Grid& g, int model, const double* prims, double* cons,
                                double* aux, cudaStream_t st);
cudaError_t launch_apply_bcs(const Grid& g, double* arr, int nvars, cudaStream_t st);
// WenoBase::reconstructUpwind + reconstructDownwind of nc variables along dir
// on materialised ghosts: frecon = upwind(f+) + downwind(f-) on
// [shift, N - shift), zero elsewhere (fluxVectorSplitting.cc:36-49).
cudaError_t launch_weno_dir(const Grid& g, int nc, int order, int dir, const double* fplus,
                            const double* fminus, double* frecon, cudaStream_t st);

// REGIME, the resistive source extension of SRMHD (regime.cu).
struct RegimeWork {
  double *E, *q, *fp, *fm, *frx, *fry, *K, *DX, *DY;
};
// target (interior) += dt (S(cons) + S_REGIME).  `mixed`: the 2D tile
// reconstructs the stiff fluxes in FP32 (the diffusion vectors and the update
// stay FP64); otherwise every value is the reference's.
cudaError_t launch_regime_source_add(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     const RegimeWork& w, bool mixed, cudaStream_t st);
// REGIME::sourceExtension alone into ext (9 planes, interior cells): the
// Hybrid model's REGIME term (hybrid.cc:320-345); the fused tile where it
// applies (FP32 stiff-flux WENO when `mixed`), else the per-array chain.
cudaError_t launch_regime_ext(const Grid& g, int order, const double* cons, const double* prims,
                              const RegimeWork& w, double* ext, bool mixed, cudaStream_t st);
// The Hybrid model (hybrid.cu): flux + split along dir of every cell; the
// recovery of interior cells followed by Hybrid::finalise (which updates
// cons' E); the source of interior cells (+ REGIME when `regime`, into ext
// first); primsToAll's blend of resistive and ideal variables.
cudaError_t launch_hybrid_split(const Grid& g, const double* cons, const double* prims,
                                const double* aux, int dir, double* fplus, double* fminus,
                                cudaStream_t st);
cudaError_t launch_c2p_hybrid(const Grid& g, const double* cons, const double* prims_guess,
                              const double* aux_guess, double* prims, double* aux, C2PWork w,
                              cudaStream_t st);
// Hybrid::finalise on interior cells; the mixed-form recovery (FP64 Newton
// in both branches, kernels_mixed.cu) followed by it.
cudaError_t launch_hybrid_finalise(const Grid& g, double* cons, double* prims, cudaStream_t st);
cudaError_t launch_c2p_hybrid_mixed(const Grid& g, const double* cons, const double* prims_guess,
                                    const double* aux_guess, double* prims, double* aux,
                                    C2PWork w, cudaStream_t st);
cudaError_t launch_hybrid_source(const Grid& g, int order, const double* cons,
                                 const double* prims, const double* aux, double* src,
                                 const RegimeWork* regime, double* ext, bool mixed,
                                 cudaStream_t st);
cudaError_t launch_hybrid_blend(const Grid& g, double* cons, double* prims, double* aux,
                                const double* icons, const double* iaux, cudaStream_t st);
// cons += h src on interior cells.
cudaError_t launch_add_scaled(const Grid& g, int nc, double* cons, const double* src, double h,
                              cudaStream_t st);
// The fused 2D tile with FP32 stiff-flux reconstruction (regime_mixed.cu).
cudaError_t launch_regime_tile_mixed(const Grid& g, int order, const double* cons,
                                     const double* prims, double* target, double dt,
                                     cudaStream_t st, bool ext_only = false);
// Whether the fused tile serves the grid: two dimensions and a constant
// conductivity (with functionalSigma a halo cell's sigma would read cons[0]
// that a neighbouring CTA updates in place).
inline bool regime_tile_applies(const Grid& g) {
  return g.dims == 2 && g.Nz == 1 && !g.functional_sigma;
}
// Bcs::apply for the ghost cells of x-rows [r0, r1) (ghost-inclusive indices).
cudaError_t launch_apply_bcs_rows(const Grid& g, double* arr, int nvars, int r0, int r1,
                                  cudaStream_t st);
cudaError_t launch_fvs2d_fp64(const Grid& g, int model, int order, const double* cons,
                              const double* prims, const double* aux, const double* u0,
                              double* out, double dt, int mode, cudaStream_t st,
                              StageTail tail = {});
// Generic (1D/2D/3D) flux path: materialised ghosts, one pass per direction.
cudaError_t launch_fvs_generic(const Grid& g, int model, int order, double* cons, double* prims,
                               double* aux, double* fplus, double* fminus, double* frecon,
                               double* fnet, cudaStream_t st);
// FVS::F on the arrays as they are (ghost cells are read, not remapped).
cudaError_t launch_fvs_generic_raw(const Grid& g, int model, int order, const double* cons,
                                   const double* prims, const double* aux, double* fplus,
                                   double* fminus, double* frecon, double* fnet, cudaStream_t st);
cudaError_t launch_stage_update(const Grid& g, int nc, int mode, const double* u0,
                                const double* in, const double* fnet, double dt, double* out,
                                cudaStream_t st);
cudaError_t launch_c2p_srmhd(const Grid& g, const double* cons, const double* prims_guess,
                             const double* aux_guess, double* prims, double* aux,
                             double* solution, C2PWork w, cudaStream_t st);
cudaError_t launch_c2p_srrmhd(const Grid& g, const double* cons, const double* aux_guess,
                              double* prims, double* aux, C2PWork w, cudaStream_t st);
cudaError_t launch_source(const Grid& g, int model, const double* cons, const double* aux,
                          double* out, cudaStream_t st, bool all_cells = false);
cudaError_t launch_flux_vector(const Grid& g, int model, const double* cons, const double* prims,
                               const double* aux, int dir, double* f, cudaStream_t st);
cudaError_t launch_c2p_cells(int model, double gamma, double sigma, long long n,
                             const double* cons, double* prims, double* aux, double tol,
                             int* flag, cudaStream_t st);
cudaError_t launch_imex_stage(const Grid& g, int stage, const double* cons,
                              const double* aux_guess, const double* u1, const double* flux1,
                              const double* source1, double* out, double dt, C2PWork w,
                              cudaStream_t st);
// Reference SSP2 stage solve for the cells queued in w.fail_list (count in
// w.fail_count, reset to zero afterwards).
cudaError_t launch_imex_stage_queued(const Grid& g, int stage, const double* cons,
                                     const double* aux_guess, const double* u1,
                                     const double* flux1, const double* source1, double* out,
                                     double dt, C2PWork w, cudaStream_t st);
// SSP3(332) / SSP2(322) implicit stage `form` (1-3 SSP3, 4-6 SSP2322) over the
// interior: hybrd1 on 14 unknowns per cell, U_k into `out`, the last
// residual evaluation's Z into zout[10].
cudaError_t launch_imex_sweep(const Grid& g, int form, const double* cons, const double* zaux,
                              const double* u1, const double* u2, const double* flux1,
                              const double* flux2, const double* source1, const double* source2,
                              double* out, double* zout, double dt, C2PWork w, cudaStream_t st);
// The same solves for the cells queued in w.fail_list (mixed-form fallback);
// clears the queue count afterwards.
cudaError_t launch_imex_sweep_queued(const Grid& g, int form, const double* cons,
                                     const double* zaux, const double* u1, const double* u2,
                                     const double* flux1, const double* flux2,
                                     const double* source1, const double* source2, double* out,
                                     double* zout, double dt, C2PWork w, cudaStream_t st);
cudaError_t launch_ssp3_combine(const Grid& g, double* cons, const double* f1, const double* f2,
                                const double* f3, const double* s1, const double* s2,
                                const double* s3, double dt, cudaStream_t st);
cudaError_t launch_ssp2322_combine(const Grid& g, double* cons, const double* f2,
                                   const double* f3, const double* s2, const double* s3,
                                   double dt, cudaStream_t st);
cudaError_t launch_ssp2_combine(const Grid& g, int nc, double* cons, const double* flux1,
                                const double* flux2, const double* source1,
                                const double* source2, double dt, cudaStream_t st);
cudaError_t launch_source_add(const Grid& g, int model, const double* cons, const double* prims,
                              const double* aux, double* target, double dt, cudaStream_t st);

}  // namespace mth
