// C-ABI of METHOD-B200 (include/method_b200.h).
//
// One handle = one simulation: the state arrays of Data (cons, prims, aux),
// the work arrays of the chosen TimeIntegrator, and a CUDA stream.  A time
// step is captured once per distinct dt into a CUDA graph and replayed, so the
// host enters the device once per step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "launch.h"
#include "mixed.h"
#include "../../include/method_b200.h"

using namespace mth;

struct mth_handle {
  mth_config cfg{};
  Grid g{};
  int NC = 0, NP = 0, NA = 0;
  int device = 0;
  cudaStream_t st = nullptr;      // stream that carries this handle's work
  cudaStream_t own_st = nullptr;  // the handle's own stream (graph capture runs here)
  double *cons = nullptr, *prims = nullptr, *aux = nullptr;
  double *p1cons = nullptr, *p1prims = nullptr, *p1aux = nullptr;
  double* solution = nullptr;
  double *u1 = nullptr, *u2 = nullptr, *flux1 = nullptr, *flux2 = nullptr;
  double *src1 = nullptr, *src2 = nullptr;
  double *u3 = nullptr, *flux3 = nullptr, *src3 = nullptr;  // SSP3 / SSP2322
  double *tprims = nullptr, *taux = nullptr;                // their tempprims / tempaux
  double *fnet = nullptr, *fplus = nullptr, *fminus = nullptr, *frecon = nullptr;
  int* fail_list = nullptr;
  int* fail_count = nullptr;
  long long* counters = nullptr;  // [0..3] C2P, [4..7] implicit, [8..9] Newton fallbacks
  MixedWork mixed{};
  RegimeWork regime{};
  // RKSplit2's source array; the Hybrid model's REGIME term
  double *hsrc = nullptr, *hext = nullptr;
  double t = 0, dt = 0;
  int iters = 0;
  long long steps = 0;
  bool ghosts_dirty = false;
  bool fused = false;
  std::map<std::pair<uint64_t, int>, cudaGraphExec_t> graphs;  // (dt, part; -1 = whole step)
  std::string err;
  // eager per-kernel timing (mth_profile_step)
  struct ProfRec {
    std::string name;
    int launches;
    double ms;
    double bytes;
  };
  bool profiling = false;
  std::vector<ProfRec> prof;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // pipelined host-array step: copy streams and per-row-block events
  cudaStream_t up_st = nullptr, down_st = nullptr;
  std::vector<cudaEvent_t> ev_up, ev_fin;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr, ev_done = nullptr;
};

namespace {

mth_status fail(mth_handle* h, mth_status s, const std::string& msg) {
  if (h) h->err = msg;
  return s;
}

#define CU(h, expr)                                                                 \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess)                                                          \
      return fail(h, MTH_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

long long n_interior(const mth_handle* h) {
  const Grid& g = h->g;
  return (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
}

// Runs one launch helper; when profiling, brackets it with CUDA events and
// books its duration and algorithmic bytes (doubles per interior cell * 8).
cudaError_t timed(mth_handle* h, const char* name, double doubles_per_cell,
                  const std::function<cudaError_t()>& f) {
  if (!h->profiling) return f();
  cudaEventRecord(h->ev0, h->st);
  cudaError_t e = f();
  cudaEventRecord(h->ev1, h->st);
  cudaEventSynchronize(h->ev1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  const double bytes = 8.0 * doubles_per_cell * (double)n_interior(h);
  for (auto& r : h->prof)
    if (r.name == name) {
      r.launches++;
      r.ms += ms;
      r.bytes += bytes;
      return e;
    }
  h->prof.push_back({name, 1, (double)ms, bytes});
  return e;
}

C2PWork c2p_work(mth_handle* h) { return C2PWork{h->fail_list, h->fail_count, h->counters}; }
C2PWork imex_work(mth_handle* h) { return C2PWork{h->fail_list, h->fail_count, h->counters + 4}; }
// The guess network of an SRRMHD handle with MTH_GUESS_MLP, for its implicit stages.
const MixedWork* mlp_work(const mth_handle* h) {
  return (h->cfg.model == MTH_SRRMHD && h->cfg.guess == MTH_GUESS_MLP && h->mixed.has_mlp)
             ? &h->mixed
             : nullptr;
}

size_t bytes(const mth_handle* h, int nv) { return sizeof(double) * (size_t)nv * h->g.Ntot; }

cudaError_t alloc0(double** p, size_t n, cudaStream_t st) {
  cudaError_t e = cudaMalloc(p, n);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(*p, 0, n, st);
}

// Model::getPrimitiveVars of `cons` into prims/aux, seeded by the guess arrays.
// `lean`: an intermediate state (RK2 predictor, SSP2 stage) read only by the
// fused flux tile, the source and the next implicit solve, so the Newton
// recovery writes their inputs alone.
cudaError_t c2p_raw(mth_handle* h, const double* cons, const double* pg, const double* ag,
                double* prims, double* aux, bool lean) {
  if (h->cfg.model == MTH_HYBRID && h->cfg.precision == MTH_MIXED)
    return launch_c2p_hybrid_mixed(h->g, cons, pg, ag, prims, aux, c2p_work(h), h->st);
  if (h->cfg.precision == MTH_MIXED || h->cfg.guess == MTH_GUESS_MLP)
    return launch_c2p_mixed(h->g, h->cfg.model, h->cfg.guess, cons, pg, ag, prims, aux,
                            h->solution, c2p_work(h), h->mixed, lean && h->fused, h->st);
  if (h->cfg.model == MTH_SRMHD)
    return launch_c2p_srmhd(h->g, cons, pg, ag, prims, aux, h->solution, c2p_work(h), h->st);
  if (h->cfg.model == MTH_HYBRID)  // with Hybrid::finalise, which updates cons' E
    return launch_c2p_hybrid(h->g, cons, pg, ag, prims, aux, c2p_work(h), h->st);
  return launch_c2p_srrmhd(h->g, cons, ag, prims, aux, c2p_work(h), h->st);
}

// FVS::F of (c, p, a) combined with a stage update into `out`; the mixed
// form's fused tile may be restricted to tile rows [ti0, ti0 + nti).
cudaError_t flux_stage_raw(mth_handle* h, double* c, double* p, double* a, const double* u0,
                       double* out, double dt, int mode, int ti0 = 0, int nti = -1) {
  const Grid& g = h->g;
  const StageTail tail{h->flux1, h->src1, g.cp};
  if (h->fused) {
    if (h->cfg.precision == MTH_MIXED)
      return launch_fvs2d_fp32(g, h->cfg.model, h->cfg.weno_order, c, p, a, u0, out, dt, mode,
                               h->st, tail, ti0, nti);
    return launch_fvs2d_fp64(g, h->cfg.model, h->cfg.weno_order, c, p, a, u0, out, dt, mode,
                             h->st, tail);
  }
  cudaError_t e = launch_fvs_generic(g, h->cfg.model, h->cfg.weno_order, c, p, a, h->fplus,
                                     h->fminus, h->frecon, h->fnet, h->st);
  if (e != cudaSuccess) return e;
  if (mode == STAGE_FNET)
    return cudaMemcpyAsync(out, h->fnet, bytes(h, h->NC), cudaMemcpyDeviceToDevice, h->st);
  return launch_stage_update(g, h->NC, mode, u0, c, h->fnet, dt, out, h->st);
}

cudaError_t c2p(mth_handle* h, const double* cons, const double* pg, const double* ag,
                double* prims, double* aux, bool lean = false) {
  const bool srmhd = h->cfg.model == MTH_SRMHD;
  const bool mixed = h->cfg.precision == MTH_MIXED || h->cfg.guess == MTH_GUESS_MLP;
  const char* name = h->cfg.model == MTH_HYBRID
                         ? "c2p_hybrid"
                         : srmhd ? (mixed ? "c2p_newton_srmhd" : "c2p_hybrd_srmhd")
                                 : (mixed ? "c2p_newton_srrmhd" : "c2p_secant_srrmhd");
  // doubles per cell: SRMHD 14 read, 23 written (13 lean); SRRMHD 15 read, 28 written (10 lean)
  const bool lean_run = lean && mixed && h->fused;
  return timed(h, name, srmhd ? (lean_run ? 27 : 37) : (lean_run ? 25 : 43),
               [&] { return c2p_raw(h, cons, pg, ag, prims, aux, lean); });
}

cudaError_t flux_stage(mth_handle* h, double* c, double* p, double* a, const double* u0,
                       double* out, double dt, int mode) {
  const bool srmhd = h->cfg.model == MTH_SRMHD;
  const double in = srmhd ? 22 : 24, nc = h->NC;
  // flux inputs + the written state (+ u0 for the corrector; + u0, flux1,
  // source1 and the 6 source inputs for the fused SSP2 closing stage)
  const double dpc = in + nc + (mode == STAGE_RK2_CORR ? nc : 0) +
                     (mode == STAGE_SSP2_FINAL ? 3 * nc + 6 : 0);
  const char* name = h->fused ? (h->cfg.precision == MTH_MIXED ? "fvs2d_fp32" : "fvs2d_fp64")
                              : "fvs_generic";
  return timed(h, name, dpc, [&] { return flux_stage_raw(h, c, p, a, u0, out, dt, mode); });
}

// SSP3::step (SSP3.cc:43-216) and SSP2322::step (SSP2322.cc:68-249): three
// implicit stages, each followed by the recovery (seeded by the stage's last
// Z), the source and FVS::F of the stage value, then the combination and the
// final recovery.  SSP2322 never uses F(U1) (its residuals and combination
// read F2 and F3 only), so that flux is not computed.
cudaError_t enqueue_ssp3(mth_handle* h, double dt) {
  const bool s3 = h->cfg.integrator == MTH_SSP3;
  const int f0 = s3 ? 0 : 3;
  cudaError_t e;
  double* U[3] = {h->u1, h->u2, h->u3};
  double* F[3] = {h->flux1, h->flux2, h->flux3};
  double* S[3] = {h->src1, h->src2, h->src3};
  static const char* names[2][3] = {{"imex_ssp2322_stage1", "imex_ssp2322_stage2",
                                     "imex_ssp2322_stage3"},
                                    {"imex_ssp3_stage1", "imex_ssp3_stage2", "imex_ssp3_stage3"}};
  for (int k = 0; k < 3; ++k) {
    // Z seeds: SSP3 stage 2 starts from the recovered stage-1 state, every
    // other stage from the step's own aux (SSP3.cc:103-107, 146-159;
    // SSP2322.cc:86-89, 127-130, 166-186)
    const double* zaux = (s3 && k == 1) ? h->taux : h->aux;
    const bool fast = h->cfg.precision == MTH_MIXED;
    if ((e = timed(h, names[s3][k], 29 + 14 * k, [&] {
           return fast ? launch_imex_fast_form(h->g, f0 + k + 1, h->cons, zaux, h->u1, h->u2,
                                               h->flux1, h->flux2, h->src1, h->src2, U[k],
                                               h->taux, dt, imex_work(h), h->st)
                       : launch_imex_sweep(h->g, f0 + k + 1, h->cons, zaux, h->u1, h->u2,
                                           h->flux1, h->flux2, h->src1, h->src2, U[k], h->taux,
                                           dt, imex_work(h), h->st);
         })))
      return e;
    if ((e = c2p(h, U[k], h->tprims, h->taux, h->tprims, h->taux))) return e;
    if ((e = timed(h, "source", 31, [&] {
           return launch_source(h->g, h->cfg.model, U[k], h->taux, S[k], h->st);
         })))
      return e;
    if (!s3 && k == 0) continue;
    if ((e = flux_stage(h, U[k], h->tprims, h->taux, nullptr, F[k], dt, STAGE_FNET))) return e;
  }
  if ((e = timed(h, s3 ? "ssp3_combine" : "ssp2322_combine", s3 ? 98 : 70, [&] {
         return s3 ? launch_ssp3_combine(h->g, h->cons, h->flux1, h->flux2, h->flux3, h->src1,
                                         h->src2, h->src3, dt, h->st)
                   : launch_ssp2322_combine(h->g, h->cons, h->flux2, h->flux3, h->src2, h->src3,
                                            dt, h->st);
       })))
    return e;
  // SSP3 recovers from the step's own aux; SSP2322 first copies U3's
  // recovered prims / aux over them (SSP2322.cc:236-245), of which only
  // aux[10] seeds the recovery
  return c2p(h, h->cons, h->prims, s3 ? h->aux : h->taux, h->prims, h->aux);
}

// A time step is split into parts at the points where the reference applies
// the boundary conditions to an intermediate state (TimeIntegrator::finalise
// after each stage's recovery): RK2 / RKSplit 2 parts, SSP2 3, SSP3 and
// SSP2322 1.  An x-slab handle (mth_config.x_slab) runs the parts one at a
// time and its caller exchanges the slab halos of the part's state between
// them; every other handle runs all parts inside one step graph.
int n_parts(const mth_handle* h) {
  const int integ = h->cfg.integrator;
  if (integ == MTH_RK2 || integ == MTH_RKSPLIT) return 2;
  if (integ == MTH_SSP2) return 3;
  return 1;  // SSP3, SSP2322, RKSplit2
}

// The state a part leaves for the next part's flux (cons, prims, aux).
void part_state(mth_handle* h, int part, double** c, double** p, double** a) {
  *c = h->cons;
  *p = h->prims;
  *a = h->aux;
  const int integ = h->cfg.integrator;
  if ((integ == MTH_RK2 || integ == MTH_RKSPLIT) && part == 0) {
    *c = h->p1cons;
    *p = h->p1prims;
    *a = h->p1aux;
  } else if (integ == MTH_SSP2 && part == 0) {
    *c = h->u1;
  } else if (integ == MTH_SSP2 && part == 1) {
    *c = h->u2;
  }
}

cudaError_t enqueue_ssp2_part(mth_handle* h, double dt, int part);

// RKSplit2::setSource and the half step after it (rkSplit2ndOrder.cc:8-51):
// S(U) of the model (the Hybrid model's with its REGIME term) on the state
// whose ghosts the boundary conditions filled, U += dt/2 S, finalise.
cudaError_t rksplit2_half_source(mth_handle* h, double dt) {
  cudaError_t e;
  if ((e = launch_apply_bcs(h->g, h->cons, h->NC, h->st)) ||
      (e = launch_apply_bcs(h->g, h->prims, h->NP, h->st)) ||
      (e = launch_apply_bcs(h->g, h->aux, h->NA, h->st)))
    return e;
  if ((e = timed(h, "source", 2.0 * h->NC, [&] {
         if (h->cfg.model == MTH_HYBRID)
           return launch_hybrid_source(h->g, h->cfg.weno_order, h->cons, h->prims, h->aux,
                                       h->hsrc, h->cfg.regime ? &h->regime : nullptr, h->hext,
                                       h->cfg.precision == MTH_MIXED, h->st);
         return launch_source(h->g, h->cfg.model, h->cons, h->aux, h->hsrc, h->st);
       })))
    return e;
  if ((e = launch_add_scaled(h->g, h->NC, h->cons, h->hsrc, 0.5 * dt, h->st))) return e;
  return c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux);
}

// RKSplit2::step (rkSplit2ndOrder.cc:33-67): half source, RK2::step, half
// source, each followed by finalise.
cudaError_t enqueue_rksplit2(mth_handle* h, double dt) {
  cudaError_t e;
  if ((e = rksplit2_half_source(h, dt))) return e;
  if ((e = flux_stage(h, h->cons, h->prims, h->aux, nullptr, h->p1cons, dt, STAGE_EULER)))
    return e;
  if ((e = c2p(h, h->p1cons, h->prims, h->aux, h->p1prims, h->p1aux, true))) return e;
  if ((e = flux_stage(h, h->p1cons, h->p1prims, h->p1aux, h->cons, h->cons, dt,
                      STAGE_RK2_CORR)))
    return e;
  if ((e = c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux))) return e;
  return rksplit2_half_source(h, dt);
}

// Part `part` of one TimeIntegrator::step, enqueued on the handle's stream.
cudaError_t enqueue_part(mth_handle* h, double dt, int part) {
  cudaError_t e;
  const int integ = h->cfg.integrator;
  if (integ == MTH_RK2 || integ == MTH_RKSPLIT) {
    // RK2::step (RK2.cc:93-100): predictor, finalise(p1) | corrector, finalise.
    if (part == 0) {
      if ((e = flux_stage(h, h->cons, h->prims, h->aux, nullptr, h->p1cons, dt, STAGE_EULER)))
        return e;
      return c2p(h, h->p1cons, h->prims, h->aux, h->p1prims, h->p1aux, true);
    }
    if ((e = flux_stage(h, h->p1cons, h->p1prims, h->p1aux, h->cons, h->cons, dt,
                        STAGE_RK2_CORR)))
      return e;
    if ((e = c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux))) return e;
    if (integ == MTH_RKSPLIT) {
      // RKSplit::step (rkSplit.cc:31-53): U += dt S(U), finalise.
      if (h->cfg.regime) {
        // with the REGIME extension, whose stencils read the ghosts that
        // RK2's finalise leaves filled
        if ((e = launch_apply_bcs(h->g, h->cons, h->NC, h->st)) ||
            (e = launch_apply_bcs(h->g, h->prims, h->NP, h->st)))
          return e;
        // algorithmic traffic: prims (8) and cons (9) read, cons (9) written
        if ((e = timed(h, "regime_source_add", 26.0, [&] {
               return launch_regime_source_add(h->g, h->cfg.weno_order, h->cons, h->prims,
                                               h->cons, dt, h->regime,
                                               h->cfg.precision == MTH_MIXED, h->st);
             })))
          return e;
      } else if ((e = timed(h, "source_add", 2.0 * h->NC, [&] {
                    return launch_source_add(h->g, h->cfg.model, h->cons, h->prims, h->aux,
                                             h->cons, dt, h->st);
                  }))) {
        return e;
      }
      if ((e = c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux))) return e;
    }
    return cudaSuccess;
  }
  if (integ == MTH_SSP3 || integ == MTH_SSP2322) return enqueue_ssp3(h, dt);
  if (integ == MTH_RKSPLIT2) return enqueue_rksplit2(h, dt);
  return enqueue_ssp2_part(h, dt, part);
}

// SSP2::step (SSP2.cc:53-173): implicit stage 1, finalise(U1) | F(U1),
// implicit stage 2, finalise(U2) | F(U2), combination, finalise.
cudaError_t enqueue_ssp2_part(mth_handle* h, double dt, int part) {
  cudaError_t e;
  const bool fast = h->cfg.precision == MTH_MIXED;
  if (part == 0) {
    if ((e = timed(h, fast ? "imex_newton_stage1" : "imex_hybrd_stage1", 29, [&] {
           return fast ? launch_imex_fast(h->g, 1, h->cons, h->aux, nullptr, nullptr, nullptr,
                                          h->u1, dt, imex_work(h), h->st, mlp_work(h))
                       : launch_imex_stage(h->g, 1, h->cons, h->aux, nullptr, nullptr, nullptr,
                                           h->u1, dt, imex_work(h), h->st);
         })))
      return e;
    return c2p(h, h->u1, h->prims, h->aux, h->prims, h->aux, true);
  }
  if (part == 2) {
    // flux2 = F(U2), source2 = S(U2) and the combination (SSP2.cc:150-170) in
    // one pass: the stage-2 flux tile's epilogue updates cons in place
    if (h->fused) {
      if ((e = flux_stage(h, h->u2, h->prims, h->aux, h->cons, h->cons, dt, STAGE_SSP2_FINAL)))
        return e;
      return c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux);
    }
    if ((e = timed(h, "source", 31, [&] {
           return launch_source(h->g, h->cfg.model, h->u2, h->aux, h->src2, h->st);
         })))
      return e;
    if ((e = flux_stage(h, h->u2, h->prims, h->aux, nullptr, h->flux2, dt, STAGE_FNET))) return e;
    if ((e = timed(h, "ssp2_combine", 6.0 * h->NC, [&] {
           return launch_ssp2_combine(h->g, h->NC, h->cons, h->flux1, h->flux2, h->src1, h->src2,
                                      dt, h->st);
         })))
      return e;
    return c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux);
  }
  if ((e = timed(h, "source", 31, [&] {
         return launch_source(h->g, h->cfg.model, h->u1, h->aux, h->src1, h->st);
       })))
    return e;
  if ((e = flux_stage(h, h->u1, h->prims, h->aux, nullptr, h->flux1, dt, STAGE_FNET))) return e;
  if ((e = timed(h, fast ? "imex_newton_stage2" : "imex_hybrd_stage2", 71, [&] {
         return fast ? launch_imex_fast(h->g, 2, h->cons, h->aux, h->u1, h->flux1, h->src1,
                                        h->u2, dt, imex_work(h), h->st, mlp_work(h))
                     : launch_imex_stage(h->g, 2, h->cons, h->aux, h->u1, h->flux1, h->src1,
                                         h->u2, dt, imex_work(h), h->st);
       })))
    return e;
  return c2p(h, h->u2, h->prims, h->aux, h->prims, h->aux, true);
}

// One TimeIntegrator::step, enqueued on the handle's stream.
cudaError_t enqueue_step(mth_handle* h, double dt) {
  for (int part = 0; part < n_parts(h); ++part) {
    cudaError_t e = enqueue_part(h, dt, part);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

uint64_t dt_key(double dt) {
  uint64_t k;
  std::memcpy(&k, &dt, sizeof k);
  return k;
}

// The whole step (part -1) or one part of it as a CUDA graph, captured once
// per distinct dt.
mth_status launch_step(mth_handle* h, double dt, int part = -1) {
  const std::pair<uint64_t, int> key(dt_key(dt), part);
  auto it = h->graphs.find(key);
  cudaGraphExec_t exec = nullptr;
  if (it == h->graphs.end()) {
    if (h->graphs.size() >= 16) {
      for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
      h->graphs.clear();
    }
    cudaGraph_t graph;
    cudaStream_t work = h->st;
    h->st = h->own_st;  // capture always runs on the handle's own stream
    cudaError_t e0 = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal);
    if (e0 != cudaSuccess) {
      h->st = work;
      return fail(h, MTH_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e0));
    }
    cudaError_t e = part < 0 ? enqueue_step(h, dt) : enqueue_part(h, dt, part);
    cudaError_t e2 = cudaStreamEndCapture(h->st, &graph);
    h->st = work;
    if (e != cudaSuccess) return fail(h, MTH_ERR_CUDA, std::string("step: ") + cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(h, MTH_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e2));
    CU(h, cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    h->graphs[key] = exec;
  } else {
    exec = it->second;
  }
  CU(h, cudaGraphLaunch(exec, h->st));
  h->ghosts_dirty = true;
  if (part < 0 || part == n_parts(h) - 1) h->steps++;
  return MTH_OK;
}

// Simulation::updateTime's dt (simulation.cc:113-124).
double next_dt(const mth_handle* h) {
  const mth_config& c = h->cfg;
  const Grid& g = h->g;
  double dtX(c.cfl * g.dx / (1.0 * std::sqrt((double)g.dims)));
  double dtY(c.cfl * g.dy / (1.0 * std::sqrt((double)g.dims)));
  double dtZ(c.cfl * g.dz / (1.0 * std::sqrt((double)g.dims)));
  double dt = (dtX <= dtY && dtX <= dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
  if (h->iters < 15) dt *= 0.1;
  if (h->iters >= 15 && h->iters < 30) dt *= 0.25;
  if (h->t + dt > c.endTime) dt = c.endTime - h->t;
  return dt;
}

mth_status read_status(mth_handle* h) {
  CU(h, cudaStreamSynchronize(h->st));
  long long cnt[16];
  CU(h, cudaMemcpy(cnt, h->counters, sizeof cnt, cudaMemcpyDeviceToHost));
  long long flags = cnt[3] | cnt[7];
  if (flags) {  // the error words are sticky until read here; the counts stay
    CU(h, cudaMemsetAsync(h->counters + 3, 0, sizeof(long long), h->st));
    CU(h, cudaMemsetAsync(h->counters + 7, 0, sizeof(long long), h->st));
    CU(h, cudaStreamSynchronize(h->st));
  }
  if (flags & ERR_IMPLICIT)
    return fail(h, MTH_ERR_IMPLICIT,
                "IMEX time integrator could not converge to a solution (implicit stage)");
  if (flags & ERR_C2P) return fail(h, MTH_ERR_C2P, "C2P could not converge.");
  if (flags & ERR_DEVICE)
    return fail(h, MTH_ERR_CUDA, "a tensor-core wait of the guess network ran out");
  return MTH_OK;
}

}  // namespace

namespace mth {
bool grid_from_config(const void* cfg, Grid* out) {
  const mth_config& c = *static_cast<const mth_config*>(cfg);
  Grid& g = *out;
  g = Grid{};
  g.nx = c.nx;
  g.ny = c.ny;
  g.nz = c.nz;
  g.Ng = c.Ng;
  g.Nx = c.nx + 2 * c.Ng;
  g.Ny = c.ny + 2 * c.Ng;
  g.Nz = c.nz + 2 * c.Ng;
  g.dims = 3;
  double zmin = c.zmin, zmax = c.zmax, ymin = c.ymin, ymax = c.ymax;
  if (c.nz == 0) {
    g.Nz = 1;
    zmin = -1e20;
    zmax = 1e20;
    g.dims = 2;
  }
  if (c.ny == 0) {
    g.Nz = g.Ny = 1;
    zmin = ymin = -1e20;
    zmax = ymax = 1e20;
    g.dims = 1;
  }
  g.is = c.Ng; g.ie = g.Nx - c.Ng;
  g.js = c.Ng; g.je = g.Ny - c.Ng;
  g.ks = c.Ng; g.ke = g.Nz - c.Ng;
  if (g.dims < 3) { g.ks = 0; g.ke = 1; }
  if (g.dims < 2) { g.js = 0; g.je = 1; }
  // Periodic ghost copies must come from interior cells (in x, an x-slab's
  // halo rows come from its neighbours' interiors instead).
  if (c.x_slab) {
    if (c.nx < c.Ng || c.x_global_nx < c.nx || c.x_offset < 0 ||
        c.x_offset > c.x_global_nx - c.nx)
      return false;
  } else if ((c.bcs == MTH_PERIODIC || c.bcs == MTH_FLOW) && c.nx < c.Ng) {
    return false;
  }
  if (c.bcs == MTH_PERIODIC && ((g.dims > 1 && c.ny < c.Ng) || (g.dims > 2 && c.nz < c.Ng))) {
    return false;
  }
  // an x-slab reads its x halo rows as they are: its caller fills them
  g.bcx = c.x_slab ? DIM_NONE : (c.bcs == MTH_OUTFLOW ? DIM_OUTFLOW : DIM_PERIODIC);
  g.bcy = g.dims > 1 ? (c.bcs == MTH_PERIODIC ? DIM_PERIODIC : DIM_OUTFLOW) : DIM_NONE;
  g.bcz = g.dims > 2 ? (c.bcs == MTH_PERIODIC ? DIM_PERIODIC : DIM_OUTFLOW) : DIM_NONE;
  // an x-slab's cell size is the whole domain's (xmin, xmax are its bounds)
  g.dx = (c.xmax - c.xmin) / (c.x_slab ? c.x_global_nx : c.nx);
  g.dy = (ymax - ymin) / (c.ny);
  g.dz = (zmax - zmin) / (c.nz);
  g.gamma = c.gamma;
  g.sigma = c.sigma;
  g.functional_sigma = c.functional_sigma ? 1 : 0;
  g.sigma_exp = c.sigma_exp;
  g.sigma_cross = c.sigma_crossover;
  g.sigma_span = c.sigma_span;
  g.cp = c.cp;
  g.Ntot = (long long)g.Nx * g.Ny * g.Nz;
  return true;
}
}  // namespace mth

extern "C" {

mth_status mth_create(const mth_config* cfg, mth_handle** out) {
  if (!cfg || !out) return MTH_ERR_INVALID;
  *out = nullptr;
  mth_handle* h = new mth_handle();
  h->cfg = *cfg;
  const mth_config& c = *cfg;
  // Validation of Data::initData (simData.cc:98-107) and the WENO ghost rule
  // (weno.cc:13-20).
  if (c.model != MTH_SRMHD && c.model != MTH_SRRMHD && c.model != MTH_HYBRID) {
    delete h;
    return MTH_ERR_INVALID;
  }
  if (c.sigma < 0.0 ||
      (c.weno_order != 3 && c.weno_order != 5 && c.weno_order != 7 && c.weno_order != 9 &&
       c.weno_order != 11) ||
      c.Ng < (c.weno_order + 1) / 2 + 1 || c.nx <= 0 || c.ny < 0 || c.nz < 0 ||
      (c.ny == 0 && c.nz != 0) || c.bcs < 0 || c.bcs > 2 || c.integrator < 0 ||
      c.integrator > 5 ||
      (c.integrator >= MTH_SSP2 && c.integrator <= MTH_SSP2322 && c.model != MTH_SRRMHD) ||
      ((c.integrator == MTH_SSP3 || c.integrator == MTH_SSP2322) && c.guess != 0) ||
      c.precision < 0 || c.precision > 1 || c.guess < 0 || c.guess > 1 ||
      (c.x_slab && c.integrator != MTH_RK2 && c.integrator != MTH_RKSPLIT &&
       c.integrator != MTH_SSP2) ||
      (c.regime && c.model != MTH_HYBRID &&
       (c.model != MTH_SRMHD || c.integrator != MTH_RKSPLIT || c.nz != 0 || c.x_slab)) ||
      // the Hybrid model: RK2 or RKSplit2, previous-state guesses
      (c.model == MTH_HYBRID &&
       (c.guess != 0 || c.x_slab || !(c.sigma_span > 0) ||
        (c.integrator != MTH_RK2 && c.integrator != MTH_RKSPLIT2)))) {
    delete h;
    return MTH_ERR_INVALID;
  }
  if (!grid_from_config(&c, &h->g)) {
    delete h;
    return MTH_ERR_INVALID;
  }
  const Grid& g = h->g;
  h->NC = c.model == MTH_SRMHD ? 9 : 14;
  h->NP = c.model == MTH_SRMHD ? 8 : 11;
  h->NA = c.model == MTH_SRMHD ? 13 : 17;
  h->fused = (g.dims == 2) && (c.model != MTH_HYBRID || c.weno_order <= 5);
  h->device = c.device;

  auto bail = [&](const char* what, cudaError_t e) {
    std::fprintf(stderr, "mth_create: %s: %s\n", what, cudaGetErrorString(e));
    mth_destroy(h);
    return MTH_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(c.device)) != cudaSuccess) { delete h; return MTH_ERR_CUDA; }
  if ((e = cudaStreamCreateWithFlags(&h->own_st, cudaStreamNonBlocking))) return bail("stream", e);
  h->st = h->own_st;
  if ((e = cudaEventCreate(&h->ev0)) || (e = cudaEventCreate(&h->ev1))) return bail("events", e);
  if ((e = alloc0(&h->cons, bytes(h, h->NC), h->st))) return bail("cons", e);
  if ((e = alloc0(&h->prims, bytes(h, h->NP), h->st))) return bail("prims", e);
  if ((e = alloc0(&h->aux, bytes(h, h->NA), h->st))) return bail("aux", e);
  if (c.integrator == MTH_RK2 || c.integrator == MTH_RKSPLIT || c.integrator == MTH_RKSPLIT2) {
    if (c.integrator == MTH_RKSPLIT2 && (e = alloc0(&h->hsrc, bytes(h, h->NC), h->st)))
      return bail("source", e);
    if ((e = alloc0(&h->p1cons, bytes(h, h->NC), h->st))) return bail("p1cons", e);
    if ((e = alloc0(&h->p1prims, bytes(h, h->NP), h->st))) return bail("p1prims", e);
    if ((e = alloc0(&h->p1aux, bytes(h, h->NA), h->st))) return bail("p1aux", e);
  } else {
    for (double** p : {&h->u1, &h->u2, &h->flux1, &h->flux2, &h->src1, &h->src2})
      if ((e = alloc0(p, bytes(h, h->NC), h->st))) return bail("imex", e);
    if (c.integrator != MTH_SSP2) {
      for (double** p : {&h->u3, &h->flux3, &h->src3})
        if ((e = alloc0(p, bytes(h, h->NC), h->st))) return bail("imex3", e);
      if ((e = alloc0(&h->tprims, bytes(h, h->NP), h->st))) return bail("tempprims", e);
      if ((e = alloc0(&h->taux, bytes(h, h->NA), h->st))) return bail("tempaux", e);
    }
  }
  if (c.model == MTH_SRMHD && (e = alloc0(&h->solution, bytes(h, 2), h->st)))
    return bail("solution", e);
  if ((e = alloc0(&h->fnet, bytes(h, h->NC), h->st))) return bail("fnet", e);
  // the generic flux path's arrays; the Hybrid model's primsToAll also uses
  // fplus / fminus as scratch for the ideal cons and aux (prims_to_all)
  if (!h->fused || c.model == MTH_HYBRID) {
    for (double** p : {&h->fplus, &h->fminus, &h->frecon})
      if ((e = alloc0(p, bytes(h, h->NC), h->st))) return bail("generic", e);
  }
  if ((e = cudaMalloc(&h->fail_list, sizeof(int) * (size_t)g.Ntot))) return bail("fails", e);
  if ((e = cudaMalloc(&h->fail_count, sizeof(int)))) return bail("fails", e);
  if ((e = cudaMemsetAsync(h->fail_count, 0, sizeof(int), h->st))) return bail("fails", e);
  if ((e = cudaMalloc(&h->counters, sizeof(long long) * 16))) return bail("counters", e);
  if ((e = cudaMemsetAsync(h->counters, 0, sizeof(long long) * 16, h->st))) return bail("counters", e);
  if (c.precision == MTH_MIXED || c.guess == MTH_GUESS_MLP) {
    if ((e = mixed_init(&h->mixed, g, c.model, h->st))) return bail("mixed", e);
  }
  if (c.regime) {
    RegimeWork& w = h->regime;
    for (auto pn : {std::make_pair(&w.E, 3), std::make_pair(&w.q, 1), std::make_pair(&w.fp, 3),
                    std::make_pair(&w.fm, 3), std::make_pair(&w.frx, 3),
                    std::make_pair(&w.fry, 3), std::make_pair(&w.K, 3), std::make_pair(&w.DX, 8),
                    std::make_pair(&w.DY, 8)})
      if ((e = alloc0(pn.first, bytes(h, pn.second), h->st))) return bail("regime", e);
    if (c.model == MTH_HYBRID && (e = alloc0(&h->hext, bytes(h, 9), h->st)))
      return bail("regime", e);
  }
  if ((e = cudaStreamSynchronize(h->st))) return bail("sync", e);
  *out = h;
  return MTH_OK;
}

mth_status mth_destroy(mth_handle* h) {
  if (!h) return MTH_OK;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  for (double* p : {h->cons, h->prims, h->aux, h->p1cons, h->p1prims, h->p1aux, h->solution,
                    h->u1, h->u2, h->flux1, h->flux2, h->src1, h->src2, h->fnet, h->fplus,
                    h->fminus, h->frecon, h->u3, h->flux3, h->src3, h->tprims, h->taux,
                    h->regime.E, h->regime.q, h->regime.fp, h->regime.fm, h->regime.frx,
                    h->regime.fry, h->regime.K, h->regime.DX, h->regime.DY, h->hsrc,
                    h->hext})
    if (p) cudaFree(p);
  if (h->fail_list) cudaFree(h->fail_list);
  if (h->fail_count) cudaFree(h->fail_count);
  if (h->counters) cudaFree(h->counters);
  mixed_free(&h->mixed);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t ev : h->ev_up) cudaEventDestroy(ev);
  for (cudaEvent_t ev : h->ev_fin) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {h->ev_start, h->ev_end, h->ev_done})
    if (ev) cudaEventDestroy(ev);
  if (h->up_st) cudaStreamDestroy(h->up_st);
  if (h->down_st) cudaStreamDestroy(h->down_st);
  if (h->own_st) cudaStreamDestroy(h->own_st);
  delete h;
  return MTH_OK;
}

const char* mth_last_error(const mth_handle* h) { return h ? h->err.c_str() : "null handle"; }

mth_status mth_get_dims(const mth_handle* h, int* d) {
  if (!h || !d) return MTH_ERR_INVALID;
  d[0] = h->g.Nx; d[1] = h->g.Ny; d[2] = h->g.Nz;
  d[3] = h->NC; d[4] = h->NP; d[5] = h->NA; d[6] = h->g.dims;
  return MTH_OK;
}

// Model::primsToAll of the handle's prims.  The Hybrid model's
// (hybrid.cc:438-472): SRRMHD's, SRMHD's of the first eight prims into
// scratch planes, then the blend.
cudaError_t prims_to_all(mth_handle* h) {
  cudaError_t e;
  if (h->cfg.model != MTH_HYBRID)
    return launch_prims_to_all(h->g, h->cfg.model, h->prims, h->cons, h->aux, h->st);
  if (!h->fplus || !h->fminus) return cudaErrorInvalidValue;
  if ((e = launch_prims_to_all(h->g, MTH_SRRMHD, h->prims, h->cons, h->aux, h->st))) return e;
  if ((e = launch_prims_to_all(h->g, MTH_SRMHD, h->prims, h->fplus, h->fminus, h->st))) return e;
  return launch_hybrid_blend(h->g, h->cons, h->prims, h->aux, h->fplus, h->fminus, h->st);
}

mth_status mth_set_prims(mth_handle* h, const double* prims_host) {
  if (!h || !prims_host) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaMemcpyAsync(h->prims, prims_host, bytes(h, h->NP), cudaMemcpyHostToDevice, h->st));
  CU(h, prims_to_all(h));
  CU(h, launch_apply_bcs(h->g, h->cons, h->NC, h->st));
  CU(h, launch_apply_bcs(h->g, h->prims, h->NP, h->st));
  CU(h, launch_apply_bcs(h->g, h->aux, h->NA, h->st));
  h->t = 0;
  h->iters = 0;
  h->ghosts_dirty = false;
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_upload(mth_handle* h, const double* cons, const double* prims, const double* aux) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  if (cons) CU(h, cudaMemcpyAsync(h->cons, cons, bytes(h, h->NC), cudaMemcpyHostToDevice, h->st));
  if (prims) CU(h, cudaMemcpyAsync(h->prims, prims, bytes(h, h->NP), cudaMemcpyHostToDevice, h->st));
  if (aux) CU(h, cudaMemcpyAsync(h->aux, aux, bytes(h, h->NA), cudaMemcpyHostToDevice, h->st));
  h->ghosts_dirty = false;
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_apply_bcs(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, launch_apply_bcs(h->g, h->cons, h->NC, h->st));
  CU(h, launch_apply_bcs(h->g, h->prims, h->NP, h->st));
  CU(h, launch_apply_bcs(h->g, h->aux, h->NA, h->st));
  h->ghosts_dirty = false;
  return MTH_OK;
}

mth_status mth_download(mth_handle* h, double* cons, double* prims, double* aux) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  if (h->ghosts_dirty) {
    mth_status s = mth_apply_bcs(h);
    if (s != MTH_OK) return s;
  }
  if (cons) CU(h, cudaMemcpyAsync(cons, h->cons, bytes(h, h->NC), cudaMemcpyDeviceToHost, h->st));
  if (prims) CU(h, cudaMemcpyAsync(prims, h->prims, bytes(h, h->NP), cudaMemcpyDeviceToHost, h->st));
  if (aux) CU(h, cudaMemcpyAsync(aux, h->aux, bytes(h, h->NA), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_prims_to_all(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, prims_to_all(h));
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_c2p(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  // the reference recovers the interior only and leaves ghost cells as they are
  CU(h, c2p(h, h->cons, h->prims, h->aux, h->prims, h->aux));
  return read_status(h);
}

mth_status mth_flux_F(mth_handle* h, double* fnet_host) {
  if (!h || !fnet_host) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  if (!h->fplus) {
    for (double** p : {&h->fplus, &h->fminus, &h->frecon})
      CU(h, alloc0(p, bytes(h, h->NC), h->st));
  }
  // FVS::F on the arrays exactly as they are (ghosts included), like the
  // reference's F, which reads whatever the ghost cells hold.
  Grid g = h->g;
  g.bcx = g.bcy = g.bcz = DIM_NONE;  // no remapping: raw ghost values
  CU(h, cudaMemsetAsync(h->fnet, 0, bytes(h, h->NC), h->st));
  CU(h, launch_fvs_generic_raw(g, h->cfg.model, h->cfg.weno_order, h->cons, h->prims, h->aux,
                               h->fplus, h->fminus, h->frecon, h->fnet, h->st));
  CU(h, cudaMemcpyAsync(fnet_host, h->fnet, bytes(h, h->NC), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_source(mth_handle* h, double* source_host) {
  if (!h || !source_host) return MTH_ERR_INVALID;
  if (h->cfg.model == MTH_HYBRID) return MTH_ERR_INVALID;  // the step covers it
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaMemsetAsync(h->fnet, 0, bytes(h, h->NC), h->st));
  CU(h, launch_source(h->g, h->cfg.model, h->cons, h->aux, h->fnet, h->st, true));
  CU(h, cudaMemcpyAsync(source_host, h->fnet, bytes(h, h->NC), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_flux_vector(mth_handle* h, int dir, double* f_host) {
  if (!h || !f_host || dir < 0 || dir >= 3) return MTH_ERR_INVALID;
  if (h->cfg.model == MTH_HYBRID) return MTH_ERR_INVALID;  // the step covers it
  CU(h, cudaSetDevice(h->device));
  CU(h, launch_flux_vector(h->g, h->cfg.model, h->cons, h->prims, h->aux, dir, h->fnet, h->st));
  const size_t plane = bytes(h, 1);
  if (h->cfg.model == MTH_SRRMHD && dir == 2) {
    // SRRMHD's z flux writes Sy twice and never Sz (srrmhd.cc:159-171): the
    // caller's Sz plane keeps what it held.  (Inside FVS::F that is the
    // y-direction value, which the device flux supplies there.)
    CU(h, cudaMemcpyAsync(f_host, h->fnet, 3 * plane, cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaMemcpyAsync(f_host + 4 * (plane / sizeof(double)), h->fnet + 4 * (plane / sizeof(double)),
                          (h->NC - 4) * plane, cudaMemcpyDeviceToHost, h->st));
  } else {
    CU(h, cudaMemcpyAsync(f_host, h->fnet, h->NC * plane, cudaMemcpyDeviceToHost, h->st));
  }
  CU(h, cudaStreamSynchronize(h->st));
  return MTH_OK;
}

mth_status mth_c2p_cells(int model, double gamma, double sigma, long long n, const double* cons,
                         double* prims, double* aux, double tol, int device) {
  if ((model != MTH_SRMHD && model != MTH_SRRMHD) || n <= 0 || !cons || !prims || !aux)
    return MTH_ERR_INVALID;
  const int nc = model == MTH_SRMHD ? 9 : 14, np = model == MTH_SRMHD ? 8 : 11,
            na = model == MTH_SRMHD ? 13 : 17;
  if (cudaSetDevice(device) != cudaSuccess) return MTH_ERR_CUDA;
  double *dc = nullptr, *dp = nullptr, *da = nullptr;
  int* flag = nullptr;
  mth_status st = MTH_OK;
  int hflag = 0;
  const size_t b = sizeof(double) * (size_t)n;
  if (cudaMalloc(&dc, b * nc) || cudaMalloc(&dp, b * np) || cudaMalloc(&da, b * na) ||
      cudaMalloc(&flag, sizeof(int)) || cudaMemset(flag, 0, sizeof(int)) ||
      cudaMemcpy(dc, cons, b * nc, cudaMemcpyHostToDevice) ||
      cudaMemcpy(dp, prims, b * np, cudaMemcpyHostToDevice) ||
      cudaMemcpy(da, aux, b * na, cudaMemcpyHostToDevice) ||
      launch_c2p_cells(model, gamma, sigma, n, dc, dp, da, tol, flag, 0) ||
      cudaMemcpy(prims, dp, b * np, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(aux, da, b * na, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost)) {
    st = MTH_ERR_CUDA;
  } else if (hflag) {
    st = MTH_ERR_C2P;
  }
  cudaFree(dc);
  cudaFree(dp);
  cudaFree(da);
  cudaFree(flag);
  return st;
}

mth_status mth_step(mth_handle* h, double dt) {
  if (!h || !(dt > 0)) return fail(h, MTH_ERR_INVALID, "dt must be positive");
  if (h->cfg.x_slab) return fail(h, MTH_ERR_INVALID, "an x-slab steps by parts (mth_step_part)");
  CU(h, cudaSetDevice(h->device));
  h->dt = dt;
  return launch_step(h, dt);
}

// ---- x-slab decomposition ----------------------------------------------------
mth_status mth_step_parts(const mth_handle* h, int* n) {
  if (!h || !n) return MTH_ERR_INVALID;
  *n = n_parts(h);
  return MTH_OK;
}

mth_status mth_step_part(mth_handle* h, double dt, int part) {
  if (!h || !(dt > 0) || part < 0 || part >= n_parts(h))
    return fail(h, MTH_ERR_INVALID, "dt must be positive and part in [0, parts)");
  CU(h, cudaSetDevice(h->device));
  h->dt = dt;
  return launch_step(h, dt, part);
}

mth_status mth_next_dt(const mth_handle* h, double* dt) {
  if (!h || !dt) return MTH_ERR_INVALID;
  *dt = next_dt(h);
  return MTH_OK;
}

mth_status mth_advance_time(mth_handle* h, double dt) {
  if (!h) return MTH_ERR_INVALID;
  h->t += dt;
  h->iters++;
  return MTH_OK;
}

mth_status mth_halo_bytes(const mth_handle* h, unsigned long long* nbytes) {
  if (!h || !nbytes) return MTH_ERR_INVALID;
  const Grid& g = h->g;
  *nbytes = sizeof(double) * (unsigned long long)(h->NC + h->NP + h->NA) * g.Ng * g.Ny * g.Nz;
  return MTH_OK;
}

namespace {
// Copies Ng x-rows of (cons, prims, aux) of a part's state between the grid
// (rows starting at `row`) and a packed buffer [var][Ng rows][Ny*Nz].
mth_status halo_copy(mth_handle* h, int part, int row, void* buf, bool to_buf) {
  double *c, *p, *a;
  if (part < 0) {
    c = h->cons;
    p = h->prims;
    a = h->aux;
  } else {
    part_state(h, part, &c, &p, &a);
  }
  const Grid& g = h->g;
  const size_t plane = sizeof(double) * (size_t)g.Ny * g.Nz;  // one x-row of one variable
  const size_t block = plane * g.Ng;
  char* b = static_cast<char*>(buf);
  const double* arrs[3] = {c, p, a};
  const int nv[3] = {h->NC, h->NP, h->NA};
  for (int q = 0; q < 3; ++q) {
    char* grid_rows = reinterpret_cast<char*>(const_cast<double*>(arrs[q])) + plane * row;
    const size_t pitch = sizeof(double) * (size_t)g.Ntot;
    if (to_buf)
      CU(h, cudaMemcpy2DAsync(b, block, grid_rows, pitch, block, nv[q], cudaMemcpyDeviceToDevice,
                              h->st));
    else
      CU(h, cudaMemcpy2DAsync(grid_rows, pitch, b, block, block, nv[q], cudaMemcpyDeviceToDevice,
                              h->st));
    b += block * nv[q];
  }
  return MTH_OK;
}
}  // namespace

mth_status mth_halo_pack(mth_handle* h, int part, int side, void* dst) {
  if (!h || !dst || side < 0 || side > 1 || part < -1 || part >= n_parts(h))
    return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  return halo_copy(h, part, side == 0 ? h->g.is : h->g.ie - h->g.Ng, dst, true);
}

mth_status mth_halo_unpack(mth_handle* h, int part, int side, const void* src) {
  if (!h || !src || side < 0 || side > 1 || part < -1 || part >= n_parts(h))
    return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  return halo_copy(h, part, side == 0 ? 0 : h->g.ie, const_cast<void*>(src), false);
}

mth_status mth_halo_outflow(mth_handle* h, int part, int side) {
  if (!h || side < 0 || side > 1 || part < -1 || part >= n_parts(h)) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  double *c = h->cons, *p = h->prims, *a = h->aux;
  if (part >= 0) part_state(h, part, &c, &p, &a);
  const Grid& g = h->g;
  const size_t plane = sizeof(double) * (size_t)g.Ny * g.Nz;
  const size_t pitch = sizeof(double) * (size_t)g.Ntot;
  const int src_row = side == 0 ? g.is : g.ie - 1, first = side == 0 ? 0 : g.ie;
  double* arrs[3] = {c, p, a};
  const int nv[3] = {h->NC, h->NP, h->NA};
  // Outflow::apply (boundaryConds.cc:5-145) in x: every ghost row copies the
  // boundary's interior row
  for (int q = 0; q < 3; ++q) {
    char* base = reinterpret_cast<char*>(arrs[q]);
    for (int r = 0; r < g.Ng; ++r)
      CU(h, cudaMemcpy2DAsync(base + plane * (first + r), pitch, base + plane * src_row, pitch,
                              plane, nv[q], cudaMemcpyDeviceToDevice, h->st));
  }
  return MTH_OK;
}

mth_status mth_update_time(mth_handle* h, int n) {
  if (!h) return MTH_ERR_INVALID;
  if (h->cfg.x_slab) return fail(h, MTH_ERR_INVALID, "an x-slab steps by parts (mth_step_part)");
  CU(h, cudaSetDevice(h->device));
  for (int s = 0; s < n; ++s) {
    double dt = next_dt(h);
    h->dt = dt;
    mth_status st = launch_step(h, dt);
    if (st != MTH_OK) return st;
    h->t += dt;
    h->iters++;
  }
  return MTH_OK;
}

mth_status mth_evolve(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  while (h->t < h->cfg.endTime) {
    mth_status s = mth_update_time(h, 1);
    if (s != MTH_OK) return s;
  }
  return mth_sync(h);
}

mth_status mth_sync(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  return read_status(h);
}

mth_status mth_get_stats(mth_handle* h, mth_stats* s) {
  if (!h || !s) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  mth_status st = read_status(h);
  long long cnt[16];
  CU(h, cudaMemcpy(cnt, h->counters, sizeof cnt, cudaMemcpyDeviceToHost));
  s->c2p_cells = cnt[0];
  s->c2p_evals = cnt[1];
  s->c2p_unconverged = cnt[2];
  s->implicit_cells = cnt[4];
  s->implicit_evals = cnt[5];
  s->implicit_failed = cnt[6];
  s->steps = h->steps;
  s->t = h->t;
  s->dt = h->dt;
  s->iters = h->iters;
  s->c2p_fallbacks = cnt[8] + cnt[9];
  s->implicit_fallbacks = cnt[12];
  return st;
}

mth_status mth_reset_stats(mth_handle* h) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaMemsetAsync(h->counters, 0, sizeof(long long) * 16, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  h->steps = 0;
  return MTH_OK;
}

mth_status mth_set_stream(mth_handle* h, void* stream) {
  if (!h) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaStreamSynchronize(h->st));
  h->st = stream ? static_cast<cudaStream_t>(stream) : h->own_st;
  return MTH_OK;
}

mth_status mth_pin_host(void* ptr, unsigned long long bytes) {
  if (!ptr) return MTH_ERR_INVALID;
  return cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault) == cudaSuccess
             ? MTH_OK
             : MTH_ERR_CUDA;
}

mth_status mth_unpin_host(void* ptr) {
  if (!ptr) return MTH_ERR_INVALID;
  return cudaHostUnregister(ptr) == cudaSuccess ? MTH_OK : MTH_ERR_CUDA;
}

// Variables of the input prims / aux that one step reads (bit v = variable
// v).  Mixed form on the fused 2D path: the flux tile reads prims 1-7 and aux
// 1, 4-8 (SRMHD) or prims 1-4 and aux 4-8, 10 (SRRMHD); the Newton recoveries
// seed from prims 0-3 and aux 0 (SRMHD) or aux 10 (SRRMHD); SSP2 reads only
// aux 10, its stage recoveries supplying the rest.  Everything else (the
// plain form's retry reads aux 10-12 of failed cells, the generic path reads
// whole arrays) is uploaded whole.
static void step_inputs(const mth_handle* h, unsigned& pmask, unsigned& amask) {
  pmask = (1u << h->NP) - 1;
  amask = (1u << h->NA) - 1;
  if (!h->fused || h->cfg.precision != MTH_MIXED) return;
  const int integ = h->cfg.integrator;
  const bool rk = integ == MTH_RK2 || integ == MTH_RKSPLIT;
  if (h->cfg.model == MTH_SRMHD && rk) {
    amask = 0x1F3u;  // aux 0, 1, 4-8
  } else if (h->cfg.model == MTH_SRRMHD && rk) {
    pmask = 0x1Eu;   // prims 1-4
    amask = 0x5F0u;  // aux 4-8, 10
  } else if (h->cfg.model == MTH_SRRMHD && integ == MTH_SSP2) {
    pmask = 0u;
    amask = 1u << 10;
  }
}

// Uploads the variables of `mask`, one copy per run of consecutive variables.
static cudaError_t upload_vars(mth_handle* h, double* dst, const double* src, unsigned mask,
                               int nv) {
  const size_t per = bytes(h, 1) / sizeof(double);
  for (int v = 0; v < nv;) {
    if (!(mask >> v & 1u)) {
      ++v;
      continue;
    }
    int e = v;
    while (e < nv && (mask >> e & 1u)) ++e;
    cudaError_t r = cudaMemcpyAsync(dst + v * per, src + v * per, bytes(h, e - v),
                                    cudaMemcpyHostToDevice, h->st);
    if (r != cudaSuccess) return r;
    v = e;
  }
  return cudaSuccess;
}

mth_status mth_step_host_bytes(mth_handle* h, unsigned long long* h2d, unsigned long long* d2h) {
  if (!h || !h2d || !d2h) return MTH_ERR_INVALID;
  unsigned pm, am;
  step_inputs(h, pm, am);
  *h2d = bytes(h, h->NC + __builtin_popcount(pm) + __builtin_popcount(am));
  *d2h = bytes(h, h->NC + h->NP + h->NA);
  return MTH_OK;
}

namespace {
// Copies x-rows [a, b) of the variables in `mask` between a host array and
// the device array of the same layout, one strided copy per run of
// consecutive variables.
cudaError_t copy_rows(const mth_handle* h, double* dst, const double* src, unsigned mask, int nv,
                      int a, int b, cudaMemcpyKind kind, cudaStream_t st) {
  const size_t plane = (size_t)h->g.Ny * h->g.Nz, pitch = sizeof(double) * (size_t)h->g.Ntot;
  for (int v = 0; v < nv;) {
    if (!(mask >> v & 1u)) {
      ++v;
      continue;
    }
    int e = v;
    while (e < nv && (mask >> e & 1u)) ++e;
    const size_t off = (size_t)v * h->g.Ntot + (size_t)a * plane;
    cudaError_t r = cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch,
                                      sizeof(double) * plane * (b - a), e - v, kind, st);
    if (r != cudaSuccess) return r;
    v = e;
  }
  return cudaSuccess;
}

constexpr int kPipeRows = 64;  // interior x-rows per block of the pipelined host step

bool pipelined(const mth_handle* h) {
  return h->fused && h->cfg.precision == MTH_MIXED && h->cfg.guess == MTH_GUESS_PREVIOUS &&
         h->cfg.integrator == MTH_RK2 && (h->g.ie - h->g.is) >= 4 * kPipeRows;
}

// TimeIntegrator::step on host arrays for the mixed RK2 form, pipelined over
// blocks of x-rows so that host->device copies, the two stages and
// device->host copies overlap: block k's predictor runs once blocks k-1..k+1
// are on the device, its corrector once their predictor states are
// recovered, and its final rows leave for the host while later blocks are
// still arriving.  Every kernel is the whole-grid step's, on a row range;
// the results are those of mth_step.
mth_status step_host_pipelined(mth_handle* h, double* cons, double* prims, double* aux,
                               double dt, unsigned pm, unsigned am) {
  const Grid& g = h->g;
  const int nrow = g.ie - g.is, B = (nrow + kPipeRows - 1) / kPipeRows;
  const long long nj = (long long)(g.je - g.js) * (g.ke - g.ks);
  if (!h->up_st) {
    CU(h, cudaStreamCreateWithFlags(&h->up_st, cudaStreamNonBlocking));
    CU(h, cudaStreamCreateWithFlags(&h->down_st, cudaStreamNonBlocking));
    for (cudaEvent_t* ev : {&h->ev_start, &h->ev_end, &h->ev_done})
      CU(h, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  }
  while ((int)h->ev_up.size() < B) {
    cudaEvent_t a, b;
    CU(h, cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    CU(h, cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    h->ev_up.push_back(a);
    h->ev_fin.push_back(b);
  }
  const unsigned all_c = (1u << h->NC) - 1, all_p = (1u << h->NP) - 1, all_a = (1u << h->NA) - 1;
  auto r0 = [&](int k) { return g.is + k * kPipeRows; };
  auto r1 = [&](int k) { return std::min(g.is + (k + 1) * kPipeRows, g.ie); };
  // uploads, block by block, after the handle's earlier work
  CU(h, cudaEventRecord(h->ev_start, h->st));
  CU(h, cudaStreamWaitEvent(h->up_st, h->ev_start, 0));
  CU(h, cudaStreamWaitEvent(h->down_st, h->ev_start, 0));
  for (int k = 0; k < B; ++k) {
    CU(h, copy_rows(h, h->cons, cons, all_c, h->NC, r0(k), r1(k), cudaMemcpyHostToDevice,
                    h->up_st));
    CU(h, copy_rows(h, h->prims, prims, pm, h->NP, r0(k), r1(k), cudaMemcpyHostToDevice,
                    h->up_st));
    CU(h, copy_rows(h, h->aux, aux, am, h->NA, r0(k), r1(k), cudaMemcpyHostToDevice, h->up_st));
    CU(h, cudaEventRecord(h->ev_up[k], h->up_st));
  }
  auto tiles = [&](int k, int* ti0, int* nti) {
    *ti0 = (r0(k) - g.is) / 8;
    *nti = (r1(k) - r0(k) + 7) / 8;
  };
  auto pred = [&](int k) -> cudaError_t {
    cudaError_t e;
    for (int q : {(k + B - 1) % B, k, (k + 1) % B})
      if ((e = cudaStreamWaitEvent(h->st, h->ev_up[q], 0))) return e;
    int ti0, nti;
    tiles(k, &ti0, &nti);
    if ((e = flux_stage_raw(h, h->cons, h->prims, h->aux, nullptr, h->p1cons, dt, STAGE_EULER,
                            ti0, nti)))
      return e;
    return launch_c2p_mixed(g, h->cfg.model, h->cfg.guess, h->p1cons, h->prims, h->aux,
                            h->p1prims, h->p1aux, h->solution, c2p_work(h), h->mixed, true, h->st,
                            (r0(k) - g.is) * nj, (r1(k) - r0(k)) * nj);
  };
  auto corr = [&](int k) -> cudaError_t {
    cudaError_t e;
    int ti0, nti;
    tiles(k, &ti0, &nti);
    if ((e = flux_stage_raw(h, h->p1cons, h->p1prims, h->p1aux, h->cons, h->cons, dt,
                            STAGE_RK2_CORR, ti0, nti)))
      return e;
    if ((e = launch_c2p_mixed(g, h->cfg.model, h->cfg.guess, h->cons, h->prims, h->aux, h->prims,
                              h->aux, h->solution, c2p_work(h), h->mixed, false, h->st,
                              (r0(k) - g.is) * nj, (r1(k) - r0(k)) * nj)))
      return e;
    // finalise: the rows' own ghost cells (y and z), then the rows go home
    for (auto arr : {std::make_pair(h->cons, h->NC), std::make_pair(h->prims, h->NP),
                     std::make_pair(h->aux, h->NA)})
      if ((e = launch_apply_bcs_rows(g, arr.first, arr.second, r0(k), r1(k), h->st))) return e;
    if ((e = cudaEventRecord(h->ev_fin[k], h->st))) return e;
    if ((e = cudaStreamWaitEvent(h->down_st, h->ev_fin[k], 0))) return e;
    if ((e = copy_rows(h, cons, h->cons, all_c, h->NC, r0(k), r1(k), cudaMemcpyDeviceToHost,
                       h->down_st)) ||
        (e = copy_rows(h, prims, h->prims, all_p, h->NP, r0(k), r1(k), cudaMemcpyDeviceToHost,
                       h->down_st)))
      return e;
    return copy_rows(h, aux, h->aux, all_a, h->NA, r0(k), r1(k), cudaMemcpyDeviceToHost,
                     h->down_st);
  };
  // block order: predictors from block 1 on, each corrector as soon as its
  // neighbours' predictors are done, block 0 (whose halo wraps to the last
  // block) once the last block has arrived
  CU(h, pred(1));
  CU(h, pred(2));
  for (int k = 3; k < B; ++k) {
    CU(h, pred(k));
    CU(h, corr(k - 1));
  }
  CU(h, pred(0));
  CU(h, corr(B - 1));
  CU(h, corr(0));
  CU(h, corr(1));
  // the x ghost rows (the boundary conditions across x, corners included)
  for (auto arr : {std::make_pair(h->cons, h->NC), std::make_pair(h->prims, h->NP),
                   std::make_pair(h->aux, h->NA)}) {
    CU(h, launch_apply_bcs_rows(g, arr.first, arr.second, 0, g.is, h->st));
    CU(h, launch_apply_bcs_rows(g, arr.first, arr.second, g.ie, g.Nx, h->st));
  }
  CU(h, cudaEventRecord(h->ev_end, h->st));
  CU(h, cudaStreamWaitEvent(h->down_st, h->ev_end, 0));
  for (int side = 0; side < 2; ++side) {
    const int a = side == 0 ? 0 : g.ie, b = side == 0 ? g.is : g.Nx;
    CU(h, copy_rows(h, cons, h->cons, all_c, h->NC, a, b, cudaMemcpyDeviceToHost, h->down_st));
    CU(h, copy_rows(h, prims, h->prims, all_p, h->NP, a, b, cudaMemcpyDeviceToHost, h->down_st));
    CU(h, copy_rows(h, aux, h->aux, all_a, h->NA, a, b, cudaMemcpyDeviceToHost, h->down_st));
  }
  CU(h, cudaEventRecord(h->ev_done, h->down_st));
  CU(h, cudaStreamWaitEvent(h->st, h->ev_done, 0));
  h->ghosts_dirty = false;
  h->steps++;
  return read_status(h);
}
}  // namespace

mth_status mth_step_host(mth_handle* h, double* cons, double* prims, double* aux, double dt) {
  if (!h || !cons || !prims || !aux || !(dt > 0) || h->cfg.x_slab) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  unsigned pm, am;
  step_inputs(h, pm, am);
  h->dt = dt;
  if (pipelined(h)) return step_host_pipelined(h, cons, prims, aux, dt, pm, am);
  CU(h, cudaMemcpyAsync(h->cons, cons, bytes(h, h->NC), cudaMemcpyHostToDevice, h->st));
  CU(h, upload_vars(h, h->prims, prims, pm, h->NP));
  CU(h, upload_vars(h, h->aux, aux, am, h->NA));
  mth_status s = launch_step(h, dt);
  if (s != MTH_OK) return s;
  // the reference leaves its arrays with boundary conditions applied (finalise)
  CU(h, launch_apply_bcs(h->g, h->cons, h->NC, h->st));
  CU(h, launch_apply_bcs(h->g, h->prims, h->NP, h->st));
  CU(h, launch_apply_bcs(h->g, h->aux, h->NA, h->st));
  h->ghosts_dirty = false;
  CU(h, cudaMemcpyAsync(cons, h->cons, bytes(h, h->NC), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaMemcpyAsync(prims, h->prims, bytes(h, h->NP), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaMemcpyAsync(aux, h->aux, bytes(h, h->NA), cudaMemcpyDeviceToHost, h->st));
  return read_status(h);
}

mth_status mth_profile_step(mth_handle* h, double dt, int reps, mth_kernel_time* out,
                            int max_out, int* n_out) {
  if (!h || !out || !n_out || reps <= 0 || !(dt > 0)) return MTH_ERR_INVALID;
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaStreamSynchronize(h->st));
  h->prof.clear();
  h->profiling = true;
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < reps && e == cudaSuccess; ++r) e = enqueue_step(h, dt);
  h->profiling = false;
  if (e != cudaSuccess) return fail(h, MTH_ERR_CUDA, cudaGetErrorString(e));
  h->ghosts_dirty = true;
  int n = 0;
  for (auto& r : h->prof) {
    if (n < max_out) {
      std::snprintf(out[n].name, sizeof out[n].name, "%s", r.name.c_str());
      out[n].launches = r.launches;
      out[n].total_ms = r.ms;
      out[n].bytes_per_launch = r.bytes / r.launches;
    }
    ++n;
  }
  *n_out = n;
  return read_status(h);
}

mth_status mth_set_mlp(mth_handle* h, const float* params, const float* stats) {
  if (!h || !params || !stats) return MTH_ERR_INVALID;
  if (!h->mixed.mlp_params) return fail(h, MTH_ERR_INVALID, "handle has no mixed-form work");
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaMemcpyAsync(h->mixed.mlp_params, params, sizeof(float) * MLP_NPARAM,
                        cudaMemcpyHostToDevice, h->st));
  CU(h, cudaMemcpyAsync(h->mixed.feat_stats, stats, sizeof(float) * MLP_NSTAT,
                        cudaMemcpyHostToDevice, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  h->mixed.has_mlp = 1;
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);  // re-capture with the network
  h->graphs.clear();
  return MTH_OK;
}

}  // extern "C"

struct mth_c2p_ctx {
  int device = 0;
  long long max_n = 0;
  float* P = nullptr;       // network parameters (device)
  float* S = nullptr;       // network statistics (device)
  double* zg = nullptr;     // guess planes, 2 x max_n
  long long* cnt = nullptr; // cells, iterations, unconverged, fallbacks
  bool has_mlp = false;
};

extern "C" {

mth_status mth_c2p_ctx_create(long long max_n, int device, mth_c2p_ctx** out) {
  if (max_n <= 0 || !out) return MTH_ERR_INVALID;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return MTH_ERR_CUDA;
  mth_c2p_ctx* c = new mth_c2p_ctx();
  c->device = device;
  c->max_n = max_n;
  if (mlp::configure() != cudaSuccess || cudaMalloc(&c->P, sizeof(float) * MLP_NPARAM) ||
      cudaMalloc(&c->S, sizeof(float) * MLP_NSTAT) ||
      cudaMalloc(&c->zg, sizeof(double) * 2 * max_n) ||
      cudaMalloc(&c->cnt, sizeof(long long) * 4) ||
      cudaMemset(c->cnt, 0, sizeof(long long) * 4)) {
    mth_c2p_ctx_destroy(c);
    return MTH_ERR_CUDA;
  }
  *out = c;
  return MTH_OK;
}

mth_status mth_c2p_ctx_destroy(mth_c2p_ctx* c) {
  if (!c) return MTH_OK;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  cudaFree(c->P);
  cudaFree(c->S);
  cudaFree(c->zg);
  cudaFree(c->cnt);
  delete c;
  return MTH_OK;
}

mth_status mth_c2p_ctx_set_mlp(mth_c2p_ctx* c, const float* params, const float* stats) {
  if (!c || !params || !stats) return MTH_ERR_INVALID;
  if (cudaSetDevice(c->device) ||
      cudaMemcpy(c->P, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice) ||
      cudaMemcpy(c->S, stats, sizeof(float) * MLP_NSTAT, cudaMemcpyHostToDevice))
    return MTH_ERR_CUDA;
  c->has_mlp = true;
  return MTH_OK;
}

mth_status mth_c2p_ctx_run(mth_c2p_ctx* c, double gamma, long long n, const double* cons,
                           double* prims, double* aux, int method, int guess, void* stream) {
  if (!c || n <= 0 || n > c->max_n || !cons || !prims || !aux || method < 0 || method > 1 ||
      guess < 0 || guess > 2 || (guess == MTH_GUESS_MLP && !c->has_mlp))
    return MTH_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return MTH_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(c->cnt, 0, sizeof(long long) * 4, st) != cudaSuccess) return MTH_ERR_CUDA;
  if (guess == MTH_GUESS_MLP) {
    Grid g{};
    g.Ntot = n;
    if (mlp::launch_zguess(g, n, true, cons, c->P, c->S, c->zg, st) != cudaSuccess)
      return MTH_ERR_CUDA;
  }
  if (launch_c2p_batch(n, gamma, method, guess, cons, prims, aux,
                       guess == MTH_GUESS_MLP ? c->zg : nullptr, c->cnt, st) != cudaSuccess)
    return MTH_ERR_CUDA;
  return MTH_OK;
}

mth_status mth_c2p_ctx_stats(mth_c2p_ctx* c, void* stream, mth_c2p_batch_stats* stats) {
  if (!c || !stats) return MTH_ERR_INVALID;
  if (cudaSetDevice(c->device) != cudaSuccess) return MTH_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  long long h[4] = {0, 0, 0, 0};
  if (cudaMemcpyAsync(h, c->cnt, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MTH_ERR_CUDA;
  stats->cells = h[0];
  stats->iterations = h[1];
  stats->unconverged = h[2];
  stats->fallbacks = h[3];
  return h[2] > 0 ? MTH_ERR_C2P : MTH_OK;
}

mth_status mth_c2p_batch(double gamma, long long n, const double* cons, double* prims,
                         double* aux, int method, int guess, const float* mlp_params,
                         const float* mlp_stats, void* stream, mth_c2p_batch_stats* stats) {
  if (n <= 0 || !cons || !prims || !aux || method < 0 || method > 1 || guess < 0 || guess > 2 ||
      (guess == MTH_GUESS_MLP && (!mlp_params || !mlp_stats)))
    return MTH_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MTH_ERR_CUDA;
  mth_c2p_ctx* c = nullptr;
  mth_status rc = mth_c2p_ctx_create(n, dev, &c);
  if (rc == MTH_OK && guess == MTH_GUESS_MLP) rc = mth_c2p_ctx_set_mlp(c, mlp_params, mlp_stats);
  if (rc == MTH_OK) rc = mth_c2p_ctx_run(c, gamma, n, cons, prims, aux, method, guess, stream);
  mth_c2p_batch_stats local{};
  if (rc == MTH_OK) rc = mth_c2p_ctx_stats(c, stream, stats ? stats : &local);
  mth_c2p_ctx_destroy(c);
  return rc;
}

mth_status mth_save_text(mth_handle* h, const char* dir, const char* app, int which) {
  if (!h || !dir) return MTH_ERR_INVALID;
  if (!app) app = "";
  CU(h, cudaSetDevice(h->device));
  CU(h, cudaStreamSynchronize(h->st));
  const mth_config& c = h->cfg;
  const Grid& g = h->g;
  // Data labels of the two models (srmhd.cc / srrmhd.cc constructors)
  static const char* srmhd_labels[3][13] = {
      {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz", "phi"},
      {"rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz"},
      {"h", "W", "e", "c", "b0", "bx", "by", "bz", "bsq", "vsq", "BS", "Bsq", "Ssq"}};
  static const char* srrmhd_labels[3][17] = {
      {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "psi", "phi", "qch"},
      {"rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "Ex", "Ey", "Ez"},
      {"h", "W", "e", "c", "Jx", "Jy", "Jz", "Bsq", "Esq", "vsq", "rhohWsq", "vE", "Sbarx",
       "Sbary", "Sbarz", "Sbarsq", "tauBar"}};
  const char* key[3] = {"cons", "prims", "aux"};
  const char* sub[3] = {"/Conserved/cons", "/Primitive/prims", "/Auxiliary/aux"};
  const int nv[3] = {h->NC, h->NP, h->NA};
  const double* arr[3] = {h->cons, h->prims, h->aux};
  for (int q = 0; q < 3; ++q) {
    if (!(which & (1 << q))) continue;
    std::string body;
    CU(h, format_body(g, arr[q], nv[q], body, h->st));
    const std::string fname = std::string(dir) + sub[q] + app + ".dat";
    FILE* f = std::fopen(fname.c_str(), "w");
    if (!f) return fail(h, MTH_ERR_INVALID, "could not open " + fname + " for writing");
    std::fprintf(f, "%s = ", key[q]);
    for (int v = 0; v < nv[q]; ++v) {
      const char* lab = c.model == MTH_SRMHD ? srmhd_labels[q][v] : srrmhd_labels[q][v];
      std::fprintf(f, v + 1 < nv[q] ? "%s, " : "%s\n", lab);
    }
    const bool ok = std::fwrite(body.data(), 1, body.size(), f) == body.size();
    std::fclose(f);
    if (!ok) return fail(h, MTH_ERR_INVALID, "short write to " + fname);
  }
  // Domain and constants: Data::initData moves the bounds of collapsed
  // dimensions to +-1e20 (simData.cc:72-85); the Simulation constructor sets
  // dx..dz, the cell centres and the initial dt (simulation.cc:34-61).
  double ymin = c.ymin, ymax = c.ymax, zmin = c.zmin, zmax = c.zmax;
  if (g.dims < 3) {
    zmin = -1e20;
    zmax = 1e20;
  }
  if (g.dims < 2) {
    ymin = -1e20;
    ymax = 1e20;
  }
  const double dx = g.dx, dy = (ymax - ymin) / (c.ny), dz = (zmax - zmin) / (c.nz);
  const int x0 = c.x_slab ? c.x_offset : 0;  // an x-slab writes its own columns
  if (which & MTH_SAVE_DOMAIN) {
    const std::string fname = std::string(dir) + "/Domain/domain" + app + ".dat";
    FILE* f = std::fopen(fname.c_str(), "w");
    if (!f) return fail(h, MTH_ERR_INVALID, "could not open " + fname + " for writing");
    for (int i = 0; i < g.Nx; ++i) std::fprintf(f, "%.16f ", c.xmin + (i + x0 + 0.5 - c.Ng) * dx);
    std::fprintf(f, "\n");
    for (int j = 0; j < g.Ny; ++j) std::fprintf(f, "%.16f ", ymin + (j + 0 + 0.5 - c.Ng) * dy);
    std::fprintf(f, "\n");
    for (int k = 0; k < g.Nz; ++k) std::fprintf(f, "%.16f ", zmin + (k + 0 + 0.5 - c.Ng) * dz);
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  if (which & MTH_SAVE_CONSTS) {
    const std::string fname = std::string(dir) + "/Constants/constants" + app + ".dat";
    FILE* f = std::fopen(fname.c_str(), "w");
    if (!f) return fail(h, MTH_ERR_INVALID, "could not open " + fname + " for writing");
    const double sq = std::sqrt((double)g.dims);
    const double dtX = c.cfl * dx / (1.0 * sq), dtY = c.cfl * dy / (1.0 * sq),
                 dtZ = c.cfl * dz / (1.0 * sq);
    const double dt0 = (dtX < dtY && dtX < dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
    std::fprintf(f, "constants = nx, ny, nz, Nx, Ny, Nz, xmin, xmax, ymin, ymax, zmin, zmax, "
                    "endTime, cfl, Ng, gamma, sigma, ");
    std::fprintf(f, "Ncons, Nprims, Naux, cp, dt, t, dx, dy, dz\n");
    std::fprintf(f,
                 "%d %d %d %d %d %d %.16f %.16f %.16f %.16f %.16f %.16f %.16f %.16f %d %.16f "
                 "%.16f %d %d %d %.16f %.16f %.16f %.16f %.16f %.16f\n",
                 c.nx, c.ny, c.nz, g.Nx, g.Ny, g.Nz, c.xmin, c.xmax, ymin, ymax, zmin, zmax,
                 c.endTime, c.cfl, c.Ng, c.gamma, c.sigma, h->NC, h->NP, h->NA, c.cp,
                 h->iters > 0 ? h->dt : dt0, h->t, dx, dy, dz);
    std::fclose(f);
  }
  return MTH_OK;
}

mth_status mth_device_state(mth_handle* h, double** cons, double** prims, double** aux) {
  if (!h) return MTH_ERR_INVALID;
  if (cons) *cons = h->cons;
  if (prims) *prims = h->prims;
  if (aux) *aux = h->aux;
  return MTH_OK;
}

}  // extern "C"
