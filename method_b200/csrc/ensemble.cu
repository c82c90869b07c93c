// Ensembles: host side (C ABI in method_b200.h).
//
// Members are 2D simulations: SRMHD with RK2 (plain FP64 or mixed form) and
// SRRMHD with SSP2 (mixed form).  One time step of the whole ensemble is a
// single CUDA graph: per-member dt on the device, then one persistent launch
// per phase covering every member of a model, then the time advance.  The
// flux phases are split by member size class; each class's tile height (4, 8
// or 16 rows of 32 cells) is picked by the autotuner below, which times the
// candidates on the ensemble itself.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ensemble.h"
#include "launch.h"
#include "mixed.h"
#include "../../include/method_b200.h"

using namespace mth;

namespace {

constexpr int kClasses = 3;           // nx <= 96, nx <= 192, larger
constexpr int kTiles[3] = {4, 8, 16};

int size_class(int nx) { return nx <= 96 ? 0 : (nx <= 192 ? 1 : 2); }

}  // namespace

// Per-phase event timing for mth_ensemble_profile (null when not profiling).
struct PhaseTimer {
  struct Rec {
    std::string name;
    int launches = 0;
    double ms = 0;
  };
  std::vector<Rec> recs;
  cudaEvent_t a = nullptr, b = nullptr;
};

struct mth_ensemble {
  int n = 0;
  int precision = MTH_MIXED;
  int order = 3;
  int device = 0;
  std::vector<mth_config> cfg;
  std::vector<Member> mem;  // host mirror of the descriptors
  Member* d_mem = nullptr;
  std::vector<void*> allocs;
  // work lists: flux tiles per (model, class), cells per model
  Item* d_flux[2][kClasses] = {};
  int n_flux[2][kClasses] = {};
  Item* d_cells[2] = {};
  int n_cells[2] = {};
  int ti[kClasses] = {8, 8, 8};
  int fgrid[kClasses] = {0, 0, 0};  // flux-phase CTAs per class (0: one per item, capped)
  int sms = 148;
  int grid_cells = 148 * 8;
  float tune_default_ms = 0.f, tune_best_ms = 0.f;  // autotuner's measured phase sums
  int grid_mlp = 148 * 2;
  bool has_model[2] = {false, false};
  int guess = MTH_GUESS_PREVIOUS;  // MTH_GUESS_MLP: members use their model's network
  float* mlp_params = nullptr;     // device, MLP_NPARAM: SRMHD network
  float* mlp_stats = nullptr;      // device, MLP_NSTAT
  bool has_mlp = false;
  float* mlp_params_r = nullptr;   // SRRMHD network
  float* mlp_stats_r = nullptr;
  bool has_mlp_r = false;
  cudaStream_t own = nullptr, st = nullptr;
  cudaStream_t side = nullptr;  // second branch of the captured step
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  PhaseTimer* timer = nullptr;
  cudaGraphExec_t graph = nullptr;
  std::string err;
};

namespace {

mth_status efail(mth_ensemble* e, mth_status s, const std::string& m) {
  if (e) e->err = m;
  return s;
}

#define ECU(e, x)                                                                     \
  do {                                                                                \
    cudaError_t _r = (x);                                                             \
    if (_r != cudaSuccess)                                                            \
      return efail(e, MTH_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_r)); \
  } while (0)

cudaError_t dalloc(mth_ensemble* e, void** p, size_t bytes) {
  cudaError_t r = cudaMalloc(p, bytes);
  if (r == cudaSuccess) {
    e->allocs.push_back(*p);
    r = cudaMemsetAsync(*p, 0, bytes, e->st);
  }
  return r;
}

// Rebuilds the flux work lists for the current tile heights (largest members
// first, so the strided assignment starts the long tiles early).
cudaError_t build_flux_items(mth_ensemble* e) {
  for (int md = 0; md < 2; ++md)
    for (int c = 0; c < kClasses; ++c) {
      if (e->d_flux[md][c]) cudaFree(e->d_flux[md][c]);
      e->d_flux[md][c] = nullptr;
      e->n_flux[md][c] = 0;
      std::vector<Item> items;
      std::vector<int> order;
      for (int m = 0; m < e->n; ++m)
        if (e->cfg[m].model == md && size_class(e->cfg[m].nx) == c) order.push_back(m);
      std::sort(order.begin(), order.end(),
                [&](int a, int b) { return e->cfg[a].nx * e->cfg[a].ny > e->cfg[b].nx * e->cfg[b].ny; });
      const int T = e->ti[c];
      for (int m : order) {
        const Grid& g = e->mem[m].g;
        const int nti = (g.ie - g.is + T - 1) / T, ntj = (g.je - g.js + 31) / 32;
        for (int a = 0; a < nti; ++a)
          for (int b = 0; b < ntj; ++b) items.push_back(Item{m, a, b, 0});
      }
      if (items.empty()) continue;
      cudaError_t r = cudaMalloc(&e->d_flux[md][c], sizeof(Item) * items.size());
      if (r != cudaSuccess) return r;
      r = cudaMemcpy(e->d_flux[md][c], items.data(), sizeof(Item) * items.size(),
                     cudaMemcpyHostToDevice);
      if (r != cudaSuccess) return r;
      e->n_flux[md][c] = (int)items.size();
    }
  return cudaSuccess;
}

// CTAs of a flux phase of size class c: one per work item unless the
// autotuner chose fewer persistent CTAs; the launcher caps it at the
// resident capacity.
int flux_grid(const mth_ensemble* e, int n_items, int c) {
  const int g = e->fgrid[c] > 0 ? std::min(e->fgrid[c], n_items) : n_items;
  return std::max(1, g);
}

template <class F>
cudaError_t phase(mth_ensemble* e, cudaStream_t s, const char* name, F&& f) {
  PhaseTimer* pt = e->timer;
  if (!pt) return f();
  cudaError_t r = cudaEventRecord(pt->a, s);
  if (r == cudaSuccess) r = f();
  if (r == cudaSuccess) r = cudaEventRecord(pt->b, s);
  if (r == cudaSuccess) r = cudaEventSynchronize(pt->b);
  float ms = 0.f;
  if (r == cudaSuccess) r = cudaEventElapsedTime(&ms, pt->a, pt->b);
  if (r != cudaSuccess) return r;
  for (auto& x : pt->recs)
    if (x.name == name) {
      x.launches++;
      x.ms += ms;
      return cudaSuccess;
    }
  pt->recs.push_back({name, 1, ms});
  return cudaSuccess;
}

// One flux phase of every member of a model (all size classes).
cudaError_t flux_phase(mth_ensemble* e, cudaStream_t s, int md, int ic, int ip, int ia, int iu0,
                       int iout, int mode) {
  for (int c = 0; c < kClasses; ++c) {
    const int n = e->n_flux[md][c];
    if (!n) continue;
    static const char* names[2][2][kClasses] = {
        {{"fvs_fp64_srmhd_c0", "fvs_fp64_srmhd_c1", "fvs_fp64_srmhd_c2"},
         {"fvs_fp64_srrmhd_c0", "fvs_fp64_srrmhd_c1", "fvs_fp64_srrmhd_c2"}},
        {{"fvs_fp32_srmhd_c0", "fvs_fp32_srmhd_c1", "fvs_fp32_srmhd_c2"},
         {"fvs_fp32_srrmhd_c0", "fvs_fp32_srrmhd_c1", "fvs_fp32_srrmhd_c2"}}};
    const bool mixed = e->precision == MTH_MIXED;
    cudaError_t r = phase(e, s, names[mixed][md][c], [&] {
      return mixed ? ens_fvs_fp32(e->d_mem, e->d_flux[md][c], n, md, e->order, e->ti[c], ic, ip,
                                  ia, iu0, iout, mode, flux_grid(e, n, c), s)
                   : ens_fvs_fp64(e->d_mem, e->d_flux[md][c], n, md, e->order, e->ti[c], ic, ip,
                                  ia, iu0, iout, mode, flux_grid(e, n, c), s);
    });
    if (r != cudaSuccess) return r;
  }
  return cudaSuccess;
}

// 1 when members of model `md` start their solves from the learned guess.
int net_mode(const mth_ensemble* e, int md) {
  if (e->guess != MTH_GUESS_MLP) return 0;
  return (md == MODEL_SRMHD ? e->has_mlp : e->has_mlp_r) ? 1 : 0;
}

// lean: an intermediate recovered state (RK2 predictor, SSP2 stage) that only
// the next flux, source and implicit solve read (mixed form: only their
// inputs are written).
cudaError_t c2p_phase(mth_ensemble* e, cudaStream_t s, int md, int ic, int ipg, int iag, int ip,
                      int ia, bool lean = false) {
  const int n = e->n_cells[md];
  if (!n) return cudaSuccess;
  const int grid = std::max(1, std::min(n, e->grid_cells));
  if (e->precision == MTH_MIXED) {
    const int gm = net_mode(e, md);
    if (gm) {
      cudaError_t r = phase(e, s, "mlp_zguess", [&] {
        return ens_mlp_zguess(e->d_mem, e->d_cells[md], n, ic,
                              md == MODEL_SRMHD ? e->mlp_params : e->mlp_params_r,
                              md == MODEL_SRMHD ? e->mlp_stats : e->mlp_stats_r, e->grid_mlp, s,
                              md);
      });
      if (r != cudaSuccess) return r;
    }
    return phase(e, s, md == MODEL_SRMHD ? "c2p_newton_srmhd" : "c2p_newton_srrmhd", [&] {
      return ens_c2p_newton(e->d_mem, e->d_cells[md], n, md, gm, ic, ipg, iag, ip, ia, lean, grid,
                            s);
    });
  }
  cudaError_t r = phase(e, s, "c2p_hybrd_srmhd", [&] {
    return ens_c2p_srmhd_hybrd(e->d_mem, e->d_cells[md], n, ic, ipg, iag, ip, ia, grid, s);
  });
  if (r != cudaSuccess) return r;
  return phase(e, s, "c2p_retry", [&] { return ens_c2p_retry(e->d_mem, e->n, ic, ip, ia, s); });
}

// RK2 (RK2.cc:93-100) of every SRMHD member.
cudaError_t srmhd_rk2(mth_ensemble* e, cudaStream_t s) {
  const int md = MODEL_SRMHD;
  cudaError_t r;
  if ((r = flux_phase(e, s, md, EA_CONS, EA_PRIMS, EA_AUX, -1, EA_P1C, STAGE_EULER))) return r;
  if ((r = c2p_phase(e, s, md, EA_P1C, EA_PRIMS, EA_AUX, EA_P1P, EA_P1A, true))) return r;
  if ((r = flux_phase(e, s, md, EA_P1C, EA_P1P, EA_P1A, EA_CONS, EA_CONS, STAGE_RK2_CORR)))
    return r;
  return c2p_phase(e, s, md, EA_CONS, EA_PRIMS, EA_AUX, EA_PRIMS, EA_AUX);
}

// SSP2 (SSP2.cc:53-173), mixed form, of every SRRMHD member.
cudaError_t srrmhd_ssp2(mth_ensemble* e, cudaStream_t s) {
  const int md = MODEL_SRRMHD;
  const int n = e->n_cells[md];
  const int grid = std::max(1, std::min(n, e->grid_cells));
  Item* it = e->d_cells[md];
  cudaError_t r;
  const int gm = net_mode(e, md);
  for (int stage = 1; stage <= 2; ++stage) {
    const int u = stage == 1 ? EA_U1 : EA_U2;
    if (gm) {  // the network's Z for the stage's first iterate (its explicit part)
      if (stage == 2 && (r = phase(e, s, "imex_explicit_part", [&] {
                           return ens_imex_explicit_part2(e->d_mem, it, n, grid, s);
                         })))
        return r;
      if ((r = phase(e, s, "mlp_zguess", [&] {
             return ens_mlp_zguess(e->d_mem, it, n, stage == 1 ? EA_CONS : EA_U2, e->mlp_params_r,
                                   e->mlp_stats_r, e->grid_mlp, s, MODEL_SRRMHD);
           })))
        return r;
    }
    if ((r = phase(e, s, "imex_newton", [&] {
           return ens_imex_fast(e->d_mem, it, n, stage, grid, s, gm);
         })))
      return r;
    if ((r = phase(e, s, "imex_queued", [&] { return ens_imex_queued(e->d_mem, e->n, stage, s); })))
      return r;
    if ((r = c2p_phase(e, s, md, u, EA_PRIMS, EA_AUX, EA_PRIMS, EA_AUX, true))) return r;
    if (stage == 2) break;
    if ((r = phase(e, s, "source", [&] {
           return ens_source(e->d_mem, it, n, u, EA_AUX, EA_S1, grid, s);
         })))
      return r;
    if ((r = flux_phase(e, s, md, u, EA_PRIMS, EA_AUX, -1, EA_F1, STAGE_FNET))) return r;
  }
  // F(U2), S(U2) and the combination (SSP2.cc:150-170) fused into the stage-2
  // flux phase, cons updated in place
  if ((r = flux_phase(e, s, md, EA_U2, EA_PRIMS, EA_AUX, EA_CONS, EA_CONS, STAGE_SSP2_FINAL)))
    return r;
  return c2p_phase(e, s, md, EA_CONS, EA_PRIMS, EA_AUX, EA_PRIMS, EA_AUX);
}

// One time step of every member (updateTime semantics per member).  The two
// models' members are independent, so while capturing (fork = true) the
// SRRMHD branch runs on a second stream beside the SRMHD one and each
// branch's persistent launches fill the other's tails.
cudaError_t enqueue_ens_step(mth_ensemble* e, bool fork) {
  cudaStream_t s = e->st;
  cudaError_t r = phase(e, s, "dt", [&] { return ens_dt(e->d_mem, e->n, s); });
  if (r != cudaSuccess) return r;
  const bool both = e->has_model[MODEL_SRMHD] && e->has_model[MODEL_SRRMHD];
  if (fork && both) {
    if ((r = cudaEventRecord(e->ev_fork, s))) return r;
    if ((r = cudaStreamWaitEvent(e->side, e->ev_fork, 0))) return r;
    if ((r = srrmhd_ssp2(e, e->side))) return r;
    if ((r = cudaEventRecord(e->ev_join, e->side))) return r;
    if ((r = srmhd_rk2(e, s))) return r;
    if ((r = cudaStreamWaitEvent(s, e->ev_join, 0))) return r;
  } else {
    if (e->has_model[MODEL_SRMHD] && (r = srmhd_rk2(e, s))) return r;
    if (e->has_model[MODEL_SRRMHD] && (r = srrmhd_ssp2(e, s))) return r;
  }
  return phase(e, s, "advance", [&] { return ens_advance(e->d_mem, e->n, s); });
}

mth_status capture(mth_ensemble* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  cudaStream_t work = e->st;
  e->st = e->own;
  cudaGraph_t g;
  ECU(e, cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
  cudaError_t r = enqueue_ens_step(e, true);
  cudaError_t r2 = cudaStreamEndCapture(e->st, &g);
  e->st = work;
  if (r != cudaSuccess || r2 != cudaSuccess)
    return efail(e, MTH_ERR_CUDA, cudaGetErrorString(r != cudaSuccess ? r : r2));
  ECU(e, cudaGraphInstantiate(&e->graph, g, 0));
  cudaGraphDestroy(g);
  return MTH_OK;
}

size_t nbytes(const Grid& g, int nv) { return sizeof(double) * (size_t)nv * g.Ntot; }

}  // namespace

extern "C" {

mth_status mth_ensemble_create(const mth_config* cfgs, int n, mth_ensemble** out) {
  if (!cfgs || n <= 0 || !out) return MTH_ERR_INVALID;
  *out = nullptr;
  mth_ensemble* e = new mth_ensemble();
  e->n = n;
  e->cfg.assign(cfgs, cfgs + n);
  e->precision = cfgs[0].precision;
  e->order = cfgs[0].weno_order;
  e->device = cfgs[0].device;
  e->guess = cfgs[0].guess;
  e->mem.resize(n);
  for (int m = 0; m < n; ++m) {
    const mth_config& c = cfgs[m];
    const bool ok_model = (c.model == MTH_SRMHD && c.integrator == MTH_RK2) ||
                          (c.model == MTH_SRRMHD && c.integrator == MTH_SSP2 &&
                           c.precision == MTH_MIXED);
    Member& d = e->mem[m];
    d = Member{};
    if (!ok_model || c.ny <= 0 || c.nz != 0 || c.precision != e->precision ||
        c.weno_order != e->order || (c.weno_order != 3 && c.weno_order != 5) ||
        c.device != e->device || c.sigma < 0 || c.x_slab || c.regime ||
        c.guess != cfgs[0].guess ||
        (c.guess == MTH_GUESS_MLP && c.precision != MTH_MIXED) ||
        c.Ng < (c.weno_order + 1) / 2 + 1 || !grid_from_config(&c, &d.g)) {
      delete e;
      return MTH_ERR_INVALID;
    }
    d.cfl = c.cfl;
    d.endTime = c.endTime;
    d.model = c.model;
    d.integrator = c.integrator;
    e->has_model[c.model] = true;
  }
  auto bail = [&](cudaError_t r) {
    std::fprintf(stderr, "mth_ensemble_create: %s\n", cudaGetErrorString(r));
    mth_ensemble_destroy(e);
    return MTH_ERR_CUDA;
  };
  cudaError_t r;
  if ((r = cudaSetDevice(e->device))) { delete e; return MTH_ERR_CUDA; }
  if ((r = cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking))) return bail(r);
  if ((r = cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking))) return bail(r);
  if ((r = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming))) return bail(r);
  if ((r = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming))) return bail(r);
  e->st = e->own;
  for (int m = 0; m < n; ++m) {
    Member& d = e->mem[m];
    const int nc = d.model == MTH_SRMHD ? 9 : 14, np = d.model == MTH_SRMHD ? 8 : 11,
              na = d.model == MTH_SRMHD ? 13 : 17;
    const int sizes[EA_COUNT] = {nc, np, na, nc, np, na, nc, nc, nc, nc, 2, 2};
    const bool need[EA_COUNT] = {true, true, true,
                                 d.model == MTH_SRMHD, d.model == MTH_SRMHD, d.model == MTH_SRMHD,
                                 d.model == MTH_SRRMHD, d.model == MTH_SRRMHD,
                                 d.model == MTH_SRRMHD, d.model == MTH_SRRMHD,
                                 d.model == MTH_SRMHD,
                                 e->guess == MTH_GUESS_MLP};
    for (int a = 0; a < EA_COUNT; ++a) {
      d.a[a] = nullptr;
      if (need[a] && (r = dalloc(e, (void**)&d.a[a], nbytes(d.g, sizes[a])))) return bail(r);
    }
    if ((r = dalloc(e, (void**)&d.fail_list, sizeof(int) * (size_t)d.g.Ntot))) return bail(r);
    if ((r = dalloc(e, (void**)&d.fail_count, sizeof(int)))) return bail(r);
    if ((r = dalloc(e, (void**)&d.counters, sizeof(long long) * 16))) return bail(r);
  }
  if ((r = dalloc(e, (void**)&e->d_mem, sizeof(Member) * n))) return bail(r);
  if ((r = dalloc(e, (void**)&e->mlp_params, sizeof(float) * MLP_NPARAM))) return bail(r);
  if ((r = dalloc(e, (void**)&e->mlp_stats, sizeof(float) * 32))) return bail(r);
  if ((r = dalloc(e, (void**)&e->mlp_params_r, sizeof(float) * MLP_NPARAM))) return bail(r);
  if ((r = dalloc(e, (void**)&e->mlp_stats_r, sizeof(float) * 32))) return bail(r);
  if ((r = cudaMemcpyAsync(e->d_mem, e->mem.data(), sizeof(Member) * n, cudaMemcpyHostToDevice,
                           e->st)))
    return bail(r);
  // cell work lists
  for (int md = 0; md < 2; ++md) {
    std::vector<Item> items;
    for (int m = 0; m < n; ++m) {
      if (e->cfg[m].model != md) continue;
      const Grid& g = e->mem[m].g;
      const long long nI = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
      for (long long o = 0; o < nI; o += ENS_CHUNK) items.push_back(Item{m, (int)o, 0, 0});
    }
    if (items.empty()) continue;
    if ((r = cudaMalloc(&e->d_cells[md], sizeof(Item) * items.size()))) return bail(r);
    if ((r = cudaMemcpy(e->d_cells[md], items.data(), sizeof(Item) * items.size(),
                        cudaMemcpyHostToDevice)))
      return bail(r);
    e->n_cells[md] = (int)items.size();
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  e->sms = sms;
  e->grid_cells = sms * 8;
  e->grid_mlp = sms * 2;
  if ((r = build_flux_items(e))) return bail(r);
  if ((r = mlp::configure())) return bail(r);
  if ((r = cudaStreamSynchronize(e->st))) return bail(r);
  *out = e;
  return MTH_OK;
}

mth_status mth_ensemble_destroy(mth_ensemble* e) {
  if (!e) return MTH_OK;
  cudaSetDevice(e->device);
  if (e->own) cudaStreamSynchronize(e->own);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  for (void* p : e->allocs) cudaFree(p);
  for (int md = 0; md < 2; ++md) {
    for (int c = 0; c < kClasses; ++c)
      if (e->d_flux[md][c]) cudaFree(e->d_flux[md][c]);
    if (e->d_cells[md]) cudaFree(e->d_cells[md]);
  }
  if (e->own) cudaStreamDestroy(e->own);
  if (e->side) cudaStreamDestroy(e->side);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  delete e;
  return MTH_OK;
}

const char* mth_ensemble_last_error(const mth_ensemble* e) { return e ? e->err.c_str() : ""; }

mth_status mth_ensemble_set_prims(mth_ensemble* e, int m, const double* prims) {
  if (!e || m < 0 || m >= e->n || !prims) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  Member& d = e->mem[m];
  const int np = d.model == MTH_SRMHD ? 8 : 11;
  const int nc = d.model == MTH_SRMHD ? 9 : 14, na = d.model == MTH_SRMHD ? 13 : 17;
  ECU(e, cudaMemcpyAsync(d.a[EA_PRIMS], prims, nbytes(d.g, np), cudaMemcpyHostToDevice, e->st));
  ECU(e, launch_prims_to_all(d.g, d.model, d.a[EA_PRIMS], d.a[EA_CONS], d.a[EA_AUX], e->st));
  ECU(e, launch_apply_bcs(d.g, d.a[EA_CONS], nc, e->st));
  ECU(e, launch_apply_bcs(d.g, d.a[EA_PRIMS], np, e->st));
  ECU(e, launch_apply_bcs(d.g, d.a[EA_AUX], na, e->st));
  // t = 0, iters = 0 for this member
  Member host;
  ECU(e, cudaMemcpyAsync(&host, e->d_mem + m, sizeof(Member), cudaMemcpyDeviceToHost, e->st));
  ECU(e, cudaStreamSynchronize(e->st));
  host.t = 0;
  host.iters = 0;
  host.dt = 0;
  ECU(e, cudaMemcpyAsync(e->d_mem + m, &host, sizeof(Member), cudaMemcpyHostToDevice, e->st));
  ECU(e, cudaStreamSynchronize(e->st));
  return MTH_OK;
}

mth_status mth_ensemble_download(mth_ensemble* e, int m, double* cons, double* prims,
                                 double* aux) {
  if (!e || m < 0 || m >= e->n) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  Member& d = e->mem[m];
  const int nc = d.model == MTH_SRMHD ? 9 : 14, np = d.model == MTH_SRMHD ? 8 : 11,
            na = d.model == MTH_SRMHD ? 13 : 17;
  ECU(e, launch_apply_bcs(d.g, d.a[EA_CONS], nc, e->st));
  ECU(e, launch_apply_bcs(d.g, d.a[EA_PRIMS], np, e->st));
  ECU(e, launch_apply_bcs(d.g, d.a[EA_AUX], na, e->st));
  if (cons) ECU(e, cudaMemcpyAsync(cons, d.a[EA_CONS], nbytes(d.g, nc), cudaMemcpyDeviceToHost, e->st));
  if (prims) ECU(e, cudaMemcpyAsync(prims, d.a[EA_PRIMS], nbytes(d.g, np), cudaMemcpyDeviceToHost, e->st));
  if (aux) ECU(e, cudaMemcpyAsync(aux, d.a[EA_AUX], nbytes(d.g, na), cudaMemcpyDeviceToHost, e->st));
  ECU(e, cudaStreamSynchronize(e->st));
  return MTH_OK;
}

namespace {
mth_status set_network(mth_ensemble* e, int md, const float* params, const float* stats) {
  if (!e || !params || !stats || e->guess != MTH_GUESS_MLP) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  float* P = md == MODEL_SRMHD ? e->mlp_params : e->mlp_params_r;
  float* S = md == MODEL_SRMHD ? e->mlp_stats : e->mlp_stats_r;
  ECU(e, cudaMemcpyAsync(P, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, e->st));
  ECU(e, cudaMemcpyAsync(S, stats, sizeof(float) * MLP_NSTAT, cudaMemcpyHostToDevice, e->st));
  ECU(e, cudaStreamSynchronize(e->st));
  (md == MODEL_SRMHD ? e->has_mlp : e->has_mlp_r) = true;
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  return MTH_OK;
}
}  // namespace

mth_status mth_ensemble_set_mlp(mth_ensemble* e, const float* params, const float* stats) {
  return set_network(e, MODEL_SRMHD, params, stats);
}

mth_status mth_ensemble_set_mlp_srrmhd(mth_ensemble* e, const float* params, const float* stats) {
  return set_network(e, MODEL_SRRMHD, params, stats);
}

mth_status mth_ensemble_set_stream(mth_ensemble* e, void* stream) {
  if (!e) return MTH_ERR_INVALID;
  ECU(e, cudaStreamSynchronize(e->st));
  e->st = stream ? static_cast<cudaStream_t>(stream) : e->own;
  return MTH_OK;
}

// Times each candidate tile height per size class on the ensemble's own
// first flux phase and keeps the fastest; returns the choice in ti_out[3].
namespace {
// Event time of `reps` launches of one flux phase (after one warm-up launch).
cudaError_t time_flux(mth_ensemble* e, int c, int T, int grid, int reps, cudaEvent_t a,
                      cudaEvent_t b, float* ms_out) {
  float total = 0.f;
  for (int md = 0; md < 2; ++md) {
    if (!e->n_flux[md][c]) continue;
    const int iout = md == MODEL_SRMHD ? EA_P1C : EA_F1;
    const int mode = md == MODEL_SRMHD ? STAGE_EULER : STAGE_FNET;
    const int n = e->n_flux[md][c];
    const int g = grid > 0 ? std::min(grid, n) : n;
    for (int rep = 0; rep <= reps; ++rep) {
      cudaError_t r = cudaEventRecord(a, e->st);
      if (r != cudaSuccess) return r;
      r = (e->precision == MTH_MIXED)
              ? ens_fvs_fp32(e->d_mem, e->d_flux[md][c], n, md, e->order, T, EA_CONS, EA_PRIMS,
                             EA_AUX, -1, iout, mode, g, e->st)
              : ens_fvs_fp64(e->d_mem, e->d_flux[md][c], n, md, e->order, T, EA_CONS, EA_PRIMS,
                             EA_AUX, -1, iout, mode, g, e->st);
      if (r != cudaSuccess) return r;
      if ((r = cudaEventRecord(b, e->st)) || (r = cudaEventSynchronize(b))) return r;
      float ms = 0.f;
      if ((r = cudaEventElapsedTime(&ms, a, b))) return r;
      if (rep > 0) total += ms;
    }
  }
  *ms_out = total;
  return cudaSuccess;
}

// Event time of `reps` primitive-recovery phases of every model at the
// current cell-phase grid (mixed form): each member's state is recovered into
// its stage scratch arrays (SRMHD: the RK2 predictor's prims / aux; SRRMHD:
// U2 / U1, which hold what the lean recovery writes), so no state changes.
cudaError_t time_cells(mth_ensemble* e, int reps, cudaEvent_t a, cudaEvent_t b, float* ms_out) {
  float total = 0.f;
  for (int rep = 0; rep <= reps; ++rep) {
    cudaError_t r = cudaEventRecord(a, e->st);
    if (r != cudaSuccess) return r;
    if ((r = c2p_phase(e, e->st, MODEL_SRMHD, EA_CONS, EA_PRIMS, EA_AUX, EA_P1P, EA_P1A, true)))
      return r;
    if ((r = c2p_phase(e, e->st, MODEL_SRRMHD, EA_CONS, EA_PRIMS, EA_AUX, EA_U2, EA_U1, true)))
      return r;
    if ((r = cudaEventRecord(b, e->st)) || (r = cudaEventSynchronize(b))) return r;
    float ms = 0.f;
    if ((r = cudaEventElapsedTime(&ms, a, b))) return r;
    if (rep > 0) total += ms;
  }
  *ms_out = total;
  return cudaSuccess;
}
}  // namespace

mth_status mth_ensemble_autotune(mth_ensemble* e, int reps, int* ti_out) {
  if (!e || reps <= 0) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  ECU(e, ens_dt(e->d_mem, e->n, e->st));
  cudaEvent_t a, b;
  ECU(e, cudaEventCreate(&a));
  ECU(e, cudaEventCreate(&b));
  float def_total = 0.f, best_total = 0.f;
  // flux phases: tile height x persistent grid, per member size class
  const int grids[3] = {0, e->sms * 4, e->sms * 2};
  for (int c = 0; c < kClasses; ++c) {
    bool any = false;
    for (int m = 0; m < e->n; ++m) any |= size_class(e->cfg[m].nx) == c;
    if (!any) continue;
    float best = 1e30f, def = 0.f;
    int best_ti = 8, best_grid = 0;
    for (int T : kTiles) {
      e->ti[c] = T;
      ECU(e, build_flux_items(e));
      for (int G : grids) {
        float ms = 0.f;
        ECU(e, time_flux(e, c, T, G, reps, a, b, &ms));
        if (T == 8 && G == 0) def = ms;
        if (ms < best) {
          best = ms;
          best_ti = T;
          best_grid = G;
        }
      }
    }
    e->ti[c] = best_ti;
    e->fgrid[c] = best_grid;
    def_total += def;
    best_total += best;
  }
  ECU(e, build_flux_items(e));
  // cell phases (recoveries, implicit stages): CTAs per SM of the persistent
  // grid, timed on the mixed form's recoveries; the members' statistics are
  // restored afterwards
  if (e->precision == MTH_MIXED) {
    std::vector<long long> saved(16 * (size_t)e->n);
    for (int m = 0; m < e->n; ++m)
      ECU(e, cudaMemcpyAsync(&saved[16 * (size_t)m], e->mem[m].counters, 16 * sizeof(long long),
                             cudaMemcpyDeviceToHost, e->st));
    ECU(e, cudaStreamSynchronize(e->st));
    float best = 1e30f, def = 0.f;
    int best_g = e->sms * 8;
    for (int per_sm : {8, 4, 16}) {
      e->grid_cells = e->sms * per_sm;
      float ms = 0.f;
      ECU(e, time_cells(e, reps, a, b, &ms));
      if (per_sm == 8) def = ms;
      if (ms < best) {
        best = ms;
        best_g = e->grid_cells;
      }
    }
    e->grid_cells = best_g;
    def_total += def;
    best_total += best;
    for (int m = 0; m < e->n; ++m)
      ECU(e, cudaMemcpyAsync(e->mem[m].counters, &saved[16 * (size_t)m], 16 * sizeof(long long),
                             cudaMemcpyHostToDevice, e->st));
    ECU(e, cudaStreamSynchronize(e->st));
  }
  e->tune_default_ms = def_total / reps;
  e->tune_best_ms = best_total / reps;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  if (ti_out)
    for (int c = 0; c < kClasses; ++c) ti_out[c] = e->ti[c];
  return MTH_OK;
}

mth_status mth_ensemble_tuning(const mth_ensemble* e, mth_tuning_report* t) {
  if (!e || !t) return MTH_ERR_INVALID;
  for (int c = 0; c < kClasses; ++c) {
    t->tile_height[c] = e->ti[c];
    t->flux_ctas[c] = e->fgrid[c];
  }
  t->cell_ctas = e->grid_cells;
  t->default_ms = e->tune_default_ms;
  t->tuned_ms = e->tune_best_ms;
  return MTH_OK;
}

mth_status mth_ensemble_step(mth_ensemble* e, int n_steps) {
  if (!e || n_steps < 0) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  if (!e->graph) {
    mth_status s = capture(e);
    if (s != MTH_OK) return s;
  }
  for (int s = 0; s < n_steps; ++s) ECU(e, cudaGraphLaunch(e->graph, e->st));
  return MTH_OK;
}

mth_status mth_ensemble_profile(mth_ensemble* e, int reps, mth_kernel_time* out, int max_out,
                                int* n_out) {
  if (!e || reps <= 0 || (!out && max_out > 0)) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  PhaseTimer pt;
  ECU(e, cudaEventCreate(&pt.a));
  ECU(e, cudaEventCreate(&pt.b));
  e->timer = &pt;
  cudaError_t r = cudaSuccess;
  for (int i = 0; i < reps && r == cudaSuccess; ++i) r = enqueue_ens_step(e, false);
  e->timer = nullptr;
  cudaEventDestroy(pt.a);
  cudaEventDestroy(pt.b);
  ECU(e, r);
  int n = 0;
  for (const auto& x : pt.recs) {
    if (n < max_out) {
      std::snprintf(out[n].name, sizeof out[n].name, "%s", x.name.c_str());
      out[n].launches = x.launches;
      out[n].total_ms = x.ms;
      out[n].bytes_per_launch = 0;
    }
    ++n;
  }
  if (n_out) *n_out = n;
  return mth_ensemble_sync(e);
}

mth_status mth_ensemble_sync(mth_ensemble* e) {
  if (!e) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  ECU(e, cudaStreamSynchronize(e->st));
  long long flags = 0;
  for (int m = 0; m < e->n; ++m) {
    long long c[16];
    ECU(e, cudaMemcpy(c, e->mem[m].counters, sizeof c, cudaMemcpyDeviceToHost));
    flags |= c[3] | c[7];
    if (c[3] | c[7]) {  // sticky until read here; the counts stay
      ECU(e, cudaMemsetAsync(e->mem[m].counters + 3, 0, sizeof(long long), e->st));
      ECU(e, cudaMemsetAsync(e->mem[m].counters + 7, 0, sizeof(long long), e->st));
    }
  }
  ECU(e, cudaStreamSynchronize(e->st));
  if (flags & ERR_IMPLICIT) return efail(e, MTH_ERR_IMPLICIT, "implicit stage did not converge");
  if (flags & ERR_C2P) return efail(e, MTH_ERR_C2P, "C2P could not converge.");
  return MTH_OK;
}

mth_status mth_ensemble_stats(mth_ensemble* e, int m, mth_stats* s) {
  if (!e || m < 0 || m >= e->n || !s) return MTH_ERR_INVALID;
  ECU(e, cudaSetDevice(e->device));
  ECU(e, cudaStreamSynchronize(e->st));
  long long c[16];
  Member d;
  ECU(e, cudaMemcpy(c, e->mem[m].counters, sizeof c, cudaMemcpyDeviceToHost));
  ECU(e, cudaMemcpy(&d, e->d_mem + m, sizeof(Member), cudaMemcpyDeviceToHost));
  std::memset(s, 0, sizeof *s);
  s->c2p_cells = c[0];
  s->c2p_evals = c[1];
  s->c2p_unconverged = c[2];
  s->implicit_cells = c[4];
  s->implicit_evals = c[5];
  s->implicit_failed = c[6];
  s->c2p_fallbacks = c[8] + c[9];
  s->implicit_fallbacks = c[12];
  s->t = d.t;
  s->dt = d.dt;
  s->iters = d.iters;
  s->steps = d.iters;
  return MTH_OK;
}

mth_status mth_ensemble_info(const mth_ensemble* e, long long* interior_cells, int* ti3) {
  if (!e) return MTH_ERR_INVALID;
  long long total = 0;
  for (int m = 0; m < e->n; ++m) {
    const Grid& g = e->mem[m].g;
    total += (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  }
  if (interior_cells) *interior_cells = total;
  if (ti3)
    for (int c = 0; c < kClasses; ++c) ti3[c] = e->ti[c];
  return MTH_OK;
}

}  // extern "C"
