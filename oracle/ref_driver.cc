// Test infrastructure only: a C-ABI driver around the UNMODIFIED METHOD CPU
// classes (Project/CPU/Src/*.cc), compiled out of tree by oracle/Makefile into
// oracle/_ref/.  It is the checker for the CUDA path and the CPU baseline of
// bench.py; nothing in the product links or loads it.
//
// The driver wires the reference objects together exactly as the reference's
// own tests do (Tests/CPU/Src/test_rk2.cc:25-41, test_imex.cc), then exposes:
//   * whole time steps through Simulation::updateTime (simulation.cc:104-133),
//   * the single pieces of the hot path: FVS::F (fluxVectorSplitting.cc:58-131),
//     Model::getPrimitiveVars, primsToAll, sourceTerm, Bcs::apply,
//   * the point kernels weno3_upwind / weno5_upwind (wenoUpwinds.cc:5-83),
//   * hybrd1 on the known-answer systems of Tests/CPU/Src/test_cminpack.cc.
// All arrays are in the reference layout ID(var,i,j,k) (simData.h:10).

#include <cstdio>
#include <cstring>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "simData.h"
#include "simulation.h"
#include "initFunc.h"
#include "srmhd.h"
#include "srrmhd.h"
#include "weno.h"
#include "REGIME.h"
#include "wenoUpwinds.h"
#include "fluxVectorSplitting.h"
#include "boundaryConds.h"
#include "RK2.h"
#include "rkSplit.h"
#include "rkSplit2ndOrder.h"
#include "hybrid.h"
#include "SSP2.h"
#include "SSP3.h"
#include "serialEnv.h"
#include "serialSaveData.h"

// ref_driver_ssp2322.cc
TimeIntegrator* mref_new_ssp2322(Data* data, Model* model, Bcs* bcs, FluxMethod* flux);
#include "cminpack.h"

extern "C" {

typedef struct {
  int model;       // 0 = SRMHD, 1 = SRRMHD, 2 = Hybrid
  int nx, ny, nz;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double endTime, cfl;
  int Ng;
  double gamma, sigma, cp;
  int weno;        // 3 or 5
  int bcs;         // 0 = Outflow, 1 = Periodic, 2 = Flow
  int integrator;  // 0 = RK2, 1 = RKSplit, 2 = SSP2, 3 = SSP3, 4 = SSP2322, 5 = RKSplit2
  int init;        // 0 = caller prims, 1 = OTVortexSingleFluid, 2 = KHInstabilitySingleFluid,
                   // 3 = KHRandomInstabilitySingleFluid, 4 = BrioWuSingleFluid,
                   // 5 = CurrentSheetSingleFluid
  int init_arg0, init_arg1;
  int functional_sigma;  // Data::functionalSigma
  double sigma_exp;      // Data::gam
  int extension;         // 0 = none, 1 = REGIME (RKSplit's model extension)
  double sigma_crossover;  // Hybrid(data, sigmaCrossOver, sigmaSpan, useREGIME)
  double sigma_span;
  int use_regime;
} mref_config;

}  // extern "C"

namespace {

// Sets d->prims from a caller array after the base class zeroed the state
// (initFunc.cc:10-40), which is how a project InitialFunc supplies data.
class ArrayInit : public InitialFunc {
 public:
  ArrayInit(Data* d, const double* prims) : InitialFunc(d) {
    std::memcpy(d->prims, prims, sizeof(double) * d->Nprims * d->Nx * d->Ny * d->Nz);
  }
};

struct RefSim {
  SerialEnv* env = nullptr;
  Data* data = nullptr;
  Model* model = nullptr;
  WenoBase* weno = nullptr;
  FVS* flux = nullptr;
  Bcs* bcs = nullptr;
  Outflow* outflow = nullptr;   // Bcs has a protected destructor, so the
  Periodic* periodic = nullptr; // concrete object is kept for deletion
  Flow* flow = nullptr;
  Simulation* sim = nullptr;
  InitialFunc* init = nullptr;
  TimeIntegrator* timeInt = nullptr;
  ModelExtension* ext = nullptr;
  ~RefSim() {
    delete timeInt;
    delete ext;
    delete init;
    delete sim;
    delete outflow;
    delete periodic;
    delete flow;
    delete flux;
    delete weno;
    delete model;
    delete data;
    delete env;
  }
};

}  // namespace

extern "C" {

void* mref_create(const mref_config* c, const double* prims) {
  RefSim* r = new RefSim();
  try {
    r->env = new SerialEnv(0, NULL, 1, 1, 1, 1);
    // reportItersPeriod is set large so updateTime prints nothing.
    r->data = new Data(c->nx, c->ny, c->nz, c->xmin, c->xmax, c->ymin, c->ymax,
                       c->zmin, c->zmax, c->endTime, r->env, c->cfl, c->Ng,
                       c->gamma, c->sigma, c->cp, -1.0e4, 1.0e4, 10, 1 << 30,
                       c->functional_sigma != 0, c->sigma_exp);
    Hybrid* hybrid = nullptr;
    if (c->model == 0) r->model = new SRMHD(r->data);
    else if (c->model == 1) r->model = new SRRMHD(r->data);
    else
      r->model = hybrid = new Hybrid(r->data, c->sigma_crossover, c->sigma_span,
                                     c->use_regime != 0);
    if (c->weno == 3) r->weno = new Weno3(r->data);
    else if (c->weno == 5) r->weno = new Weno5(r->data);
    else if (c->weno == 7) r->weno = new Weno7(r->data);
    else if (c->weno == 9) r->weno = new Weno9(r->data);
    else r->weno = new Weno11(r->data);
    r->flux = new FVS(r->data, r->weno, r->model);
    if (hybrid) {
      hybrid->setupREGIME(r->flux);  // as Examples/Hybrid/*/main.cc
      // Hybrid::sourceTerm adds all nine planes of regimeSource (hybrid.cc:
      // 330-343), but REGIME::sourceExtension never writes its last plane
      // (REGIME.cc:97-133), so the reference reads memory it did not
      // initialise.  A fresh process gets that buffer zeroed from the OS; in a
      // process that has freed earlier simulations the heap may recycle a
      // used chunk.  Zero it here, which is the fresh-process behaviour.
      if (c->use_regime)
        std::memset(hybrid->regimeSource, 0,
                    sizeof(double) * 9 * r->data->Nx * r->data->Ny * r->data->Nz);
    }
    if (c->bcs == 0) r->bcs = r->outflow = new Outflow(r->data);
    else if (c->bcs == 1) r->bcs = r->periodic = new Periodic(r->data);
    else r->bcs = r->flow = new Flow(r->data);
    r->sim = new Simulation(r->data, r->env);
    switch (c->init) {
      case 0: r->init = new ArrayInit(r->data, prims); break;
      case 1: r->init = new OTVortexSingleFluid(r->data); break;
      case 2: r->init = new KHInstabilitySingleFluid(r->data, c->init_arg0); break;
      case 3: r->init = new KHRandomInstabilitySingleFluid(r->data, c->init_arg0, c->init_arg1); break;
      case 4: r->init = new BrioWuSingleFluid(r->data, c->init_arg0); break;
      default: r->init = new CurrentSheetSingleFluid(r->data, c->init_arg0); break;
    }
    if (c->integrator == 0) r->timeInt = new RK2(r->data, r->model, r->bcs, r->flux);
    else if (c->integrator == 1) {
      if (c->extension == 1) r->ext = new REGIME(r->data, r->flux);
      r->timeInt = new RKSplit(r->data, r->model, r->bcs, r->flux, r->ext);
    }
    else if (c->integrator == 5) r->timeInt = new RKSplit2(r->data, r->model, r->bcs, r->flux);
    else if (c->integrator == 3) r->timeInt = new SSP3(r->data, r->model, r->bcs, r->flux);
    else if (c->integrator == 4) r->timeInt = mref_new_ssp2322(r->data, r->model, r->bcs, r->flux);
    else r->timeInt = new SSP2(r->data, r->model, r->bcs, r->flux);
    r->sim->set(r->init, r->model, r->timeInt, r->bcs, r->flux, NULL);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "mref_create: %s\n", e.what());
    delete r;
    return nullptr;
  }
  return r;
}

void mref_destroy(void* h) { delete static_cast<RefSim*>(h); }

// Runs n calls of Simulation::updateTime.  Returns 0, or 1 if the reference threw.
int mref_update_time(void* h, int n) {
  RefSim* r = static_cast<RefSim*>(h);
  try {
    for (int s = 0; s < n; s++) r->sim->updateTime();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "mref_update_time: %s\n", e.what());
    return 1;
  }
  return 0;
}

// Runs the integrator's step with an explicit dt (no slow start, no clock update).
int mref_step_dt(void* h, double dt) {
  RefSim* r = static_cast<RefSim*>(h);
  try {
    r->timeInt->step(r->data->cons, r->data->prims, r->data->aux, dt);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "mref_step_dt: %s\n", e.what());
    return 1;
  }
  return 0;
}

void mref_info(void* h, int* ints, double* dbls) {
  RefSim* r = static_cast<RefSim*>(h);
  Data* d = r->data;
  ints[0] = d->Nx; ints[1] = d->Ny; ints[2] = d->Nz;
  ints[3] = d->Ncons; ints[4] = d->Nprims; ints[5] = d->Naux;
  ints[6] = d->iters; ints[7] = d->dims;
  dbls[0] = d->t; dbls[1] = d->dt; dbls[2] = d->dx; dbls[3] = d->dy; dbls[4] = d->dz;
}

// SerialSaveData::saveCons / savePrims / saveAux / saveDomain / saveConsts
// (serialSaveData.cc:31-246) into dir (< 50 characters, as the reference's
// char dir[50]; subdirectories must exist).  Returns 0, or 1 for a too-long
// argument.
int mref_save_text(void* h, const char* dir, const char* app) {
  RefSim* r = static_cast<RefSim*>(h);
  if (std::strlen(dir) >= 50 || std::strlen(app) >= 50) return 1;
  SerialSaveData save(r->data, r->env);
  std::strcpy(save.dir, dir);
  std::strcpy(save.app, app);
  save.saveCons();
  save.savePrims();
  save.saveAux();
  save.saveDomain();
  save.saveConsts();
  return 0;
}

void mref_get_state(void* h, double* cons, double* prims, double* aux) {
  RefSim* r = static_cast<RefSim*>(h);
  Data* d = r->data;
  size_t n = (size_t)d->Nx * d->Ny * d->Nz;
  if (cons) std::memcpy(cons, d->cons, sizeof(double) * n * d->Ncons);
  if (prims) std::memcpy(prims, d->prims, sizeof(double) * n * d->Nprims);
  if (aux) std::memcpy(aux, d->aux, sizeof(double) * n * d->Naux);
}

void mref_set_state(void* h, const double* cons, const double* prims, const double* aux) {
  RefSim* r = static_cast<RefSim*>(h);
  Data* d = r->data;
  size_t n = (size_t)d->Nx * d->Ny * d->Nz;
  if (cons) std::memcpy(d->cons, cons, sizeof(double) * n * d->Ncons);
  if (prims) std::memcpy(d->prims, prims, sizeof(double) * n * d->Nprims);
  if (aux) std::memcpy(d->aux, aux, sizeof(double) * n * d->Naux);
}

// FVS::F on caller arrays; fnet receives Ncons*Ntot doubles (interior written).
int mref_flux_F(void* h, double* cons, double* prims, double* aux, double* fnet) {
  RefSim* r = static_cast<RefSim*>(h);
  try {
    r->flux->F(cons, prims, aux, r->data->f, fnet);
  } catch (const std::exception& e) {
    return 1;
  }
  return 0;
}

// Model::fluxVector for one direction over all cells.
void mref_flux_vector(void* h, double* cons, double* prims, double* aux, double* f, int dir) {
  RefSim* r = static_cast<RefSim*>(h);
  r->model->fluxVector(cons, prims, aux, f, dir);
}

int mref_c2p(void* h, double* cons, double* prims, double* aux) {
  RefSim* r = static_cast<RefSim*>(h);
  try {
    r->model->getPrimitiveVars(cons, prims, aux);
  } catch (const std::exception& e) {
    return 1;
  }
  return 0;
}

int mref_c2p_single(void* h, double* cons, double* prims, double* aux) {
  RefSim* r = static_cast<RefSim*>(h);
  try {
    r->model->getPrimitiveVarsSingleCell(cons, prims, aux, -1, -1, -1);
  } catch (const std::exception& e) {
    return 1;
  }
  return 0;
}

void mref_prims_to_all(void* h, double* cons, double* prims, double* aux) {
  static_cast<RefSim*>(h)->model->primsToAll(cons, prims, aux);
}

void mref_source(void* h, double* cons, double* prims, double* aux, double* source) {
  static_cast<RefSim*>(h)->model->sourceTerm(cons, prims, aux, source);
}

void mref_apply_bcs(void* h, double* cons, double* prims, double* aux) {
  static_cast<RefSim*>(h)->bcs->apply(cons, prims, aux);
}

double mref_weno3_upwind(double a, double b, double c) { return weno3_upwind(a, b, c); }
double mref_weno5_upwind(double a, double b, double c, double d, double e) {
  return weno5_upwind(a, b, c, d, e);
}

}  // extern "C"

namespace {
// Known-answer systems of Tests/CPU/Src/test_cminpack.cc:5-29, restated.
int which_kat = 0;
int kat_fcn(void* p, int n, const double* x, double* fvec, int iflag) {
  (void)p; (void)n; (void)iflag;
  if (which_kat == 0) {          // roots (-4, 2.5)
    fvec[0] = (x[0] + 4) * (x[0] + 4) * (x[0] + 4);
    fvec[1] = (x[1] - 2.5) * (x[1] - 2.5);
  } else if (which_kat == 1) {   // no real root
    fvec[0] = x[0] * x[0] + 5.0;
    fvec[1] = -x[1] * x[1] - 5.0;
  } else {                       // exp/sin system
    fvec[0] = std::exp(x[0]) + x[0] * x[1] - 1;
    fvec[1] = std::sin(x[0] * x[1]) + x[0] + x[1] - 1;
  }
  return 1;
}
}  // namespace

// hybrd1 (CminpackLibrary/Src/hybrd1.cc) on a known-answer system; lwa is the
// caller's, so lwa < n(3n+13)/2 reproduces the info=0 check.
extern "C" int mref_hybrd1_kat(int which, int n, double* x, double* fvec, double tol, int lwa) {
  which_kat = which;
  std::vector<double> wa(lwa > 0 ? lwa : 1);
  return __cminpack_func__(hybrd1)(&kat_fcn, NULL, n, x, fvec, tol, wa.data(), lwa);
}
