// C++ drop-in classes of include/method_b200/method.hpp over the C ABI.
// Host logic only: every numerical operation runs on the device through
// method_b200.h.  Comments cite the reference behaviour each method keeps.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "../../include/method_b200/method.hpp"

namespace {

void throw_status(mth_status s, mth_handle* h, const char* what) {
  if (s == MTH_OK) return;
  std::string msg = std::string(what) + ": " + (h ? mth_last_error(h) : "");
  if (s == MTH_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

}  // namespace

// ---------------------------------------------------------------- platform
SerialEnv::SerialEnv(int*, char**[], int nxRanks, int nyRanks, int nzRanks, int testing)
    : PlatformEnv(testing) {
  this->nxRanks = nxRanks;
  this->nyRanks = nyRanks;
  this->nzRanks = nzRanks;
}

// -------------------------------------------------------------------- Data
// Data::Data + Data::initData (simData.cc:11-112).
Data::Data(int nx, int ny, int nz, double xmin, double xmax, double ymin, double ymax,
           double zmin, double zmax, double endTime, PlatformEnv* env, double cfl, int Ng,
           double gamma, double sigma, double cp, double mu1, double mu2, int frameskip,
           int reportItersPeriod, bool funtionalSigma, double gam)
    : nx(nx), ny(ny), nz(nz), xmin(xmin), xmax(xmax), ymin(ymin), ymax(ymax), zmin(zmin),
      zmax(zmax), endTime(endTime), cfl(cfl), Ng(Ng), gamma(gamma), sigma(sigma), memSet(0),
      bcsSet(0), Ncons(0), Nprims(0), Naux(0), cp(cp), mu1(mu1), mu2(mu2), frameSkip(frameskip),
      reportItersPeriod(reportItersPeriod), functionalSigma(funtionalSigma), gam(gam), t(0),
      dt(0), dx(0), dy(0), dz(0), alphaX(1), alphaY(1), alphaZ(1), iters(0), cons(nullptr),
      prims(nullptr), aux(nullptr), f(nullptr), fnet(nullptr), source(nullptr),
      sourceExtension(nullptr), x(nullptr), y(nullptr), z(nullptr) {
  if (env->nxRanks * env->nyRanks * env->nzRanks != 1)
    throw std::invalid_argument("METHOD-B200 runs one domain per GPU (1x1x1 ranks)");
  Nx = nx + 2 * Ng;
  Ny = ny + 2 * Ng;
  Nz = nz + 2 * Ng;
  dims = 3;
  if (nz == 0) {
    Nz = 1;
    this->zmin = -1e20;
    this->zmax = 1e20;
    dims = 2;
  }
  if (ny == 0) {
    Nz = Ny = 1;
    this->zmin = this->ymin = -1e20;
    this->zmax = this->ymax = 1e20;
    dims = 1;
  }
  Ntot = Nx * Ny * Nz;
  is = Ng; ie = Nx - Ng;
  js = Ng; je = Ny - Ng;
  ks = Ng; ke = Nz - Ng;
  if (dims < 3) { ks = 0; ke = 1; }
  if (dims < 2) { js = 0; je = 1; }
  if (this->sigma < 0.0)
    throw std::invalid_argument("Conductivity must be non-negative, sigma >= 0.\n");
  if (this->mu1 > 0.0 or this->mu2 < 0.0)
    throw std::invalid_argument(
        "Species 1 must have negative charge, mu1 < 0, and species 2 must have positive charge, "
        "mu2 > 0.\n");
}

Data::~Data() { invalidateGpu(); }

// Data::sigmaFunc (simData.cc:114-127).
double Data::sigmaFunc(double* cons, double*, double*, int i, int j, int k) {
  if (!functionalSigma) return sigma;
  if (i < 0 || j < 0 || k < 0) return sigma * pow(cons[0], gam);
  return sigma * pow(cons[id(0, i, j, k)], gam);
}

void Data::invalidateGpu() {
  if (gpu_) mth_destroy(gpu_);
  gpu_ = nullptr;
  deviceCurrent = false;
}

void Data::check(mth_status s, const char* what) { throw_status(s, gpu_, what); }

mth_handle* Data::gpu() {
  if (gpu_) return gpu_;
  if (!model_) throw std::runtime_error("Must set model before using the device");
  mth_config c{};
  c.model = model_->modelId();
  c.nx = nx; c.ny = ny; c.nz = nz;
  c.xmin = xmin; c.xmax = xmax; c.ymin = ymin; c.ymax = ymax; c.zmin = zmin; c.zmax = zmax;
  if (dims < 3) { c.zmin = 0; c.zmax = 1; }
  if (dims < 2) { c.ymin = 0; c.ymax = 1; }
  c.endTime = endTime;
  c.cfl = cfl;
  c.Ng = Ng;
  c.gamma = gamma;
  c.sigma = sigma;
  c.cp = cp;
  c.weno_order = weno_ ? weno_->order : 3;
  c.bcs = bcs_ ? bcs_->bcId() : MTH_OUTFLOW;
  c.integrator = timeInt_ ? timeInt_->integratorId() : MTH_RK2;
  if (c.integrator >= MTH_SSP2 && c.integrator <= MTH_SSP2322 && c.model != MTH_SRRMHD)
    throw std::invalid_argument("the IMEX integrators are provided for the SRRMHD model");
  if (const Hybrid* hy = dynamic_cast<const Hybrid*>(model_)) {
    c.sigma_crossover = hy->sigmaCrossOver;
    c.sigma_span = hy->sigmaSpan;
    c.regime = hy->useREGIME ? 1 : 0;
    if (timeInt_ && timeInt_->integratorId() != MTH_RK2 &&
        timeInt_->integratorId() != MTH_RKSPLIT2)
      throw std::invalid_argument("the Hybrid model runs with RK2 or RKSplit2");
  }
  if (timeInt_ && timeInt_->integratorId() == MTH_RKSPLIT2 && timeInt_->modelExtension &&
      timeInt_->modelExtension->sourceExists)
    throw std::invalid_argument("RKSplit2 takes no model extension here");
  if (timeInt_ && timeInt_->integratorId() == MTH_RKSPLIT && timeInt_->modelExtension &&
      timeInt_->modelExtension->sourceExists && timeInt_->modelExtension->extensionId() == 1) {
    if (c.model != MTH_SRMHD || dims == 3)
      throw std::invalid_argument("REGIME extends the SRMHD model in one or two dimensions");
    c.regime = 1;
  }
  c.precision = precision;
  c.guess = guess;
  c.device = device;
  c.functional_sigma = functionalSigma ? 1 : 0;
  c.sigma_exp = gam;
  mth_status s = mth_create(&c, &gpu_);
  if (s != MTH_OK) {
    gpu_ = nullptr;
    throw_status(s, nullptr, "creating the device simulation");
  }
  deviceCurrent = false;
  return gpu_;
}

// ------------------------------------------------------------------- Model
SRMHD::SRMHD() : Model() { Ncons = 9; Nprims = 8; Naux = 13; }
SRMHD::SRMHD(Data* d) : Model(d) {
  Ncons = d->Ncons = 9;
  Nprims = d->Nprims = 8;
  Naux = d->Naux = 13;
  d->consLabels = {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz", "phi"};
  d->primsLabels = {"rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz"};
  d->auxLabels = {"h", "W", "e", "c", "b0", "bx", "by", "bz", "bsq", "vsq", "BS", "Bsq", "Ssq"};
  d->model_ = this;
  d->invalidateGpu();
}
SRRMHD::SRRMHD() : Model() { Ncons = 14; Nprims = 11; Naux = 17; }
SRRMHD::SRRMHD(Data* d) : Model(d) {
  Ncons = d->Ncons = 14;
  Nprims = d->Nprims = 11;
  Naux = d->Naux = 17;
  d->consLabels = {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "psi",
                   "phi", "qch"};
  d->primsLabels = {"rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "Ex", "Ey", "Ez"};
  d->auxLabels = {"h", "W", "e", "c", "Jx", "Jy", "Jz", "Bsq", "Esq", "vsq", "rhohWsq", "vE",
                  "Sbarx", "Sbary", "Sbarz", "Sbarsq", "tauBar"};
  d->model_ = this;
  d->invalidateGpu();
}

Hybrid::Hybrid() : Model() { Ncons = 14; Nprims = 11; Naux = 17; }
Hybrid::Hybrid(Data* d, double crossOver, double span, bool regime)
    : Model(d), sigmaCrossOver(crossOver), sigmaSpan(span), useREGIME(regime) {
  // the same variables and labels as SRRMHD (hybrid.cc:26-77)
  Ncons = d->Ncons = 14;
  Nprims = d->Nprims = 11;
  Naux = d->Naux = 17;
  d->consLabels = {"D", "Sx", "Sy", "Sz", "tau", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "psi",
                   "phi", "qch"};
  d->primsLabels = {"rho", "vx", "vy", "vz", "p", "Bx", "By", "Bz", "Ex", "Ey", "Ez"};
  d->auxLabels = {"h", "W", "e", "c", "Jx", "Jy", "Jz", "Bsq", "Esq", "vsq", "rhohWsq", "vE",
                  "Sbarx", "Sbary", "Sbarz", "Sbarsq", "tauBar"};
  d->model_ = this;
  d->invalidateGpu();
}
void Hybrid::sourceTermSingleCell(double*, double*, double*, double*, int, int, int) {
  throw std::invalid_argument("Hybrid::sourceTermSingleCell is not provided on the host");
}
void Hybrid::getPrimitiveVarsSingleCell(double*, double*, double*, int, int, int) {
  throw std::invalid_argument("Hybrid::getPrimitiveVarsSingleCell is not provided on the host");
}

namespace {
// Runs one device operation on caller arrays: upload, op, download.
template <class Op>
void on_device(Data* d, double* cons, double* prims, double* aux, Op op, bool down_cons,
               bool down_prims, bool down_aux, const char* what) {
  mth_handle* h = d->gpu();
  d->check(mth_upload(h, cons, prims, aux), what);
  d->check(op(h), what);
  d->check(mth_download(h, down_cons ? cons : nullptr, down_prims ? prims : nullptr,
                        down_aux ? aux : nullptr),
           what);
  d->deviceCurrent = (cons == d->cons && prims == d->prims && aux == d->aux);
}
}  // namespace

void Model::getPrimitiveVars(double* cons, double* prims, double* aux) {
  on_device(data, cons, prims, aux, [](mth_handle* h) { return mth_c2p(h); }, false, true, true,
            "getPrimitiveVars");
}

void Model::primsToAll(double* cons, double* prims, double* aux) {
  on_device(data, cons, prims, aux, [](mth_handle* h) { return mth_prims_to_all(h); }, true,
            false, true, "primsToAll");
}

void Model::sourceTerm(double* cons, double* prims, double* aux, double* source) {
  mth_handle* h = data->gpu();
  data->check(mth_upload(h, cons, prims, aux), "sourceTerm");
  data->check(mth_source(h, source), "sourceTerm");
  data->deviceCurrent = (cons == data->cons && prims == data->prims && aux == data->aux);
}

void Model::fluxVector(double* cons, double* prims, double* aux, double* f, int dir) {
  mth_handle* h = data->gpu();
  data->check(mth_upload(h, cons, prims, aux), "fluxVector");
  data->check(mth_flux_vector(h, dir, f), "fluxVector");
  data->deviceCurrent = (cons == data->cons && prims == data->prims && aux == data->aux);
}

// Single-cell methods run as one-cell batches on the device.
void SRMHD::sourceTermSingleCell(double* cons, double*, double*, double* source, int, int, int) {
  for (int v = 0; v < 9; ++v) source[v] = 0;
  source[8] = -cons[8] / (data->cp * data->cp);
}
void SRRMHD::sourceTermSingleCell(double* cons, double*, double* aux, double* source, int, int,
                                  int) {
  source[0] = source[1] = source[2] = source[3] = source[4] = source[5] = source[6] = source[7] =
      source[13] = 0.0;
  source[8] = -aux[4];
  source[9] = -aux[5];
  source[10] = -aux[6];
  source[11] = cons[13] - cons[11] / (data->cp * data->cp);
  source[12] = -cons[12] / (data->cp * data->cp);
}
void SRMHD::getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int, int, int) {
  mth_status s = mth_c2p_cells(MTH_SRMHD, data->gamma, data->sigma, 1, cons, prims, aux,
                               1.4e-8, data->device);
  if (s == MTH_ERR_C2P) throw std::runtime_error("C2P could not converge.\n");
  throw_status(s, nullptr, "getPrimitiveVarsSingleCell");
}
void SRRMHD::getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int, int, int) {
  mth_status s = mth_c2p_cells(MTH_SRRMHD, data->gamma, data->sigmaFunc(cons, prims, aux), 1,
                               cons, prims, aux, 0.0, data->device);
  if (s == MTH_ERR_C2P) throw std::runtime_error("C2P could not converge.\n");
  throw_status(s, nullptr, "getPrimitiveVarsSingleCell");
}

// -------------------------------------------------------------------- WENO
WenoBase::WenoBase(Data* data, int order) : data(data), order(order) {
  shift = (order + 1) / 2;
  checkSufficientGhostZones();
  data->weno_ = this;
  data->invalidateGpu();
}

void WenoBase::checkSufficientGhostZones() {
  if (data->Ng < shift + 1) {
    std::printf("This order Weno reconstruction requires at least %d ghost zones, you have %d...",
                shift + 1, data->Ng);
    throw std::invalid_argument("You must increase number of boundary cells.");
  }
}

// ---------------------------------------------------------------- FVS
FVS::FVS(Data* data, WenoBase* weno, Model* model) : FluxMethod(data, model), weno(weno) {}

void FVS::F(double* cons, double* prims, double* aux, double* f, double* fnet) {
  (void)f;
  mth_handle* h = data->gpu();
  data->check(mth_upload(h, cons, prims, aux), "F");
  data->check(mth_flux_F(h, fnet), "F");
  data->deviceCurrent = (cons == data->cons && prims == data->prims && aux == data->aux);
}

// ---------------------------------------------------------------- Bcs
Bcs::Bcs(Data* data) : data(data) {
  data->bcsSet = 1;
  data->bcs_ = this;
  data->invalidateGpu();
}

void Bcs::apply(double* cons, double* prims, double* aux) {
  on_device(data, cons, prims, aux, [](mth_handle* h) { return mth_apply_bcs(h); }, true,
            prims != nullptr, aux != nullptr, "Bcs::apply");
}

// ------------------------------------------------------- time integrators
TimeIntegrator::TimeIntegrator(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod)
    : data(data), model(model), bcs(bcs), fluxMethod(fluxMethod) {
  data->timeInt_ = this;
  data->invalidateGpu();
}

void TimeIntegrator::step(double* cons, double* prims, double* aux, double dt) {
  if (dt <= 0) dt = data->dt;
  mth_handle* h = data->gpu();
  data->check(mth_step_host(h, cons, prims, aux, dt), "step");
  data->deviceCurrent = (cons == data->cons && prims == data->prims && aux == data->aux);
}

void TimeIntegrator::finalise(double* cons, double* prims, double* aux) {
  on_device(data, cons, prims, aux,
            [](mth_handle* h) {
              mth_status s = mth_c2p(h);
              return s != MTH_OK ? s : mth_apply_bcs(h);
            },
            true, true, true, "finalise");
}

// ------------------------------------------------------------ initial data
InitialFunc::InitialFunc(Data* data) : data(data) {
  Data* d = data;
  if (d->memSet != 1)
    throw std::runtime_error(
        "Must construct simulation class before implementing initial state. Need to allocate "
        "arrays.");
  std::memset(d->cons, 0, sizeof(double) * d->Ncons * d->Ntot);
  std::memset(d->f, 0, sizeof(double) * d->Ncons * d->Ntot);
  std::memset(d->fnet, 0, sizeof(double) * d->Ncons * d->Ntot);
  std::memset(d->source, 0, sizeof(double) * d->Ncons * d->Ntot);
  std::memset(d->prims, 0, sizeof(double) * d->Nprims * d->Ntot);
  std::memset(d->aux, 0, sizeof(double) * d->Naux * d->Ntot);
  d->deviceCurrent = false;
}

OTVortexSingleFluid::OTVortexSingleFluid(Data* data) : InitialFunc(data) {
  Data* d = data;
  const double PI = 3.14159265358979323;
  if (d->xmin != 0.0 || d->xmax != 1.0 || d->ymin != 0.0 || d->ymax != 1.0)
    throw std::invalid_argument(
        "Boundaries are not as expected for OTVortex, uasually (x,y) E [0, 1]");
  if (d->ny == 0)
    throw std::invalid_argument("System must be at least two dimensional for this initial set up.");
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++)
      for (int k = 0; k < d->Nz; k++) {
        d->prims[ID(0, i, j, k)] = 25.0 / 36.0 / PI;
        d->prims[ID(4, i, j, k)] = 5.0 / 12.0 / PI;
        d->prims[ID(5, i, j, k)] = -sin(2.0 * PI * d->y[j]) / sqrt(4.0 * PI);
        d->prims[ID(6, i, j, k)] = sin(4.0 * PI * d->x[i]) / sqrt(4.0 * PI);
        if (d->dims == 2) {
          d->prims[ID(1, i, j, k)] = -0.5 * sin(2.0 * PI * d->y[j]);
          d->prims[ID(2, i, j, k)] = 0.5 * sin(2.0 * PI * d->x[i]);
        } else {
          d->prims[ID(1, i, j, k)] = -0.5 * sin(2.0 * PI * d->y[j]) * (1 + 0.2 * sin(2.0 * PI * d->z[j]));
          d->prims[ID(2, i, j, k)] = 0.5 * sin(2.0 * PI * d->x[i]) * (1 + 0.2 * sin(2.0 * PI * d->z[j]));
          d->prims[ID(3, i, j, k)] = 0.2 * sin(2.0 * PI * d->z[j]);
        }
      }
}

namespace {
void ideal_E(Data* d) {
  if (d->Nprims < 11) return;
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++)
      for (int k = 0; k < d->Nz; k++) {
        double* p = d->prims;
        auto P = [&](int v) -> double& { return p[ID(v, i, j, k)]; };
        P(8) = -(P(2) * P(7) - P(3) * P(6));
        P(9) = -(P(3) * P(5) - P(1) * P(7));
        P(10) = -(P(1) * P(6) - P(2) * P(5));
      }
}
}  // namespace

KHShearLayerSingleFluid::KHShearLayerSingleFluid(Data* data, int seed, double shear)
    : InitialFunc(data) {
  Data* d = data;
  std::mt19937 gen(seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++)
      for (int k = 0; k < d->Nz; k++) {
        d->prims[ID(0, i, j, k)] = 1.0;
        d->prims[ID(4, i, j, k)] = 1.0;
        d->prims[ID(1, i, j, k)] = d->y[j] > 0 ? shear * tanh((d->y[j] - 0.5) / 0.01)
                                               : -shear * tanh((d->y[j] + 0.5) / 0.01);
        d->prims[ID(2, i, j, k)] = 0.01 * U(gen);
      }
  ideal_E(d);
}

OrszagTangUnit::OrszagTangUnit(Data* data) : InitialFunc(data) {
  Data* d = data;
  const double PI = 3.14159265358979323;
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++)
      for (int k = 0; k < d->Nz; k++) {
        d->prims[ID(0, i, j, k)] = 1.0;
        d->prims[ID(4, i, j, k)] = 1.0;
        d->prims[ID(1, i, j, k)] = -0.5 * sin(2.0 * PI * d->y[j]);
        d->prims[ID(2, i, j, k)] = 0.5 * sin(2.0 * PI * d->x[i]);
        d->prims[ID(5, i, j, k)] = -sin(2.0 * PI * d->y[j]);
        d->prims[ID(6, i, j, k)] = sin(4.0 * PI * d->x[i]);
      }
  ideal_E(d);
}

HarrisCurrentSheet::HarrisCurrentSheet(Data* data, int seed) : InitialFunc(data) {
  Data* d = data;
  if (d->Nprims < 11) throw std::invalid_argument("HarrisCurrentSheet needs the SRRMHD model");
  std::mt19937 gen(seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++)
      for (int k = 0; k < d->Nz; k++) {
        d->prims[ID(0, i, j, k)] = 1.0;
        d->prims[ID(4, i, j, k)] = 50.0;
        d->prims[ID(6, i, j, k)] = tanh(d->x[i] / 0.01);
        for (int v = 1; v <= 3; ++v) d->prims[ID(v, i, j, k)] = 1e-3 * U(gen);
      }
  ideal_E(d);
}

// -------------------------------------------------------------- simulation
// Simulation::Simulation (simulation.cc:8-61).
Simulation::Simulation(Data* data, PlatformEnv* env) : data(data), env(env) {
  Data* d = data;
  if (d->Ncons == 0) throw std::runtime_error("Must set model before constructing simulation");
  if (d->bcsSet != 1)
    throw std::runtime_error(
        "Must construct boundary condition class before implementing simulation. Need to set "
        "domain decomposition parameters including periodicity.");
  const size_t N = (size_t)d->Ntot;
  d->cons = (double*)std::malloc(sizeof(double) * N * d->Ncons);
  d->f = (double*)std::malloc(sizeof(double) * N * d->Ncons);
  d->fnet = (double*)std::malloc(sizeof(double) * N * d->Ncons);
  d->source = (double*)std::malloc(sizeof(double) * N * d->Ncons);
  d->prims = (double*)std::malloc(sizeof(double) * N * d->Nprims);
  d->aux = (double*)std::malloc(sizeof(double) * N * d->Naux);
  d->x = (double*)std::malloc(sizeof(double) * d->Nx);
  d->y = (double*)std::malloc(sizeof(double) * d->Ny);
  d->z = (double*)std::malloc(sizeof(double) * d->Nz);
  d->dx = (d->xmax - d->xmin) / (d->nx);
  d->dy = (d->ymax - d->ymin) / (d->ny);
  d->dz = (d->zmax - d->zmin) / (d->nz);
  d->iters = 0;
  d->alphaX = d->alphaY = d->alphaZ = 1.0;
  double dtX(d->cfl * d->dx / (d->alphaX * sqrt(d->dims)));
  double dtY(d->cfl * d->dy / (d->alphaY * sqrt(d->dims)));
  double dtZ(d->cfl * d->dz / (d->alphaZ * sqrt(d->dims)));
  d->dt = (dtX < dtY && dtX < dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
  d->memSet = 1;
  for (int i = 0; i < d->Nx; i++) d->x[i] = d->xmin + (i + 0.5 - d->Ng) * d->dx;
  for (int j = 0; j < d->Ny; j++) d->y[j] = d->ymin + (j + 0.5 - d->Ng) * d->dy;
  for (int k = 0; k < d->Nz; k++) d->z[k] = d->zmin + (k + 0.5 - d->Ng) * d->dz;
}

Simulation::~Simulation() {
  data->invalidateGpu();
  for (double* p : {data->cons, data->f, data->fnet, data->source, data->prims, data->aux,
                    data->x, data->y, data->z})
    std::free(p);
  data->cons = data->prims = data->aux = nullptr;
}

// Simulation::set (simulation.cc:80-101): primsToAll and boundary conditions.
void Simulation::set(InitialFunc* init, Model* model, TimeIntegrator* timeInt, Bcs* bcs,
                     FluxMethod* fluxMethod, SaveData* save) {
  this->init = init;
  this->model = model;
  this->timeInt = timeInt;
  this->bcs = bcs;
  this->fluxMethod = fluxMethod;
  this->save = save;
  Data* d = data;
  mth_handle* h = d->gpu();
  d->check(mth_set_prims(h, d->prims), "set");
  d->check(mth_download(h, d->cons, d->prims, d->aux), "set");
  d->deviceCurrent = true;
}

void Simulation::syncHost() {
  Data* d = data;
  if (!d->gpu_ || !d->deviceCurrent) return;
  d->check(mth_download(d->gpu_, d->cons, d->prims, d->aux), "download");
}

// Simulation::updateTime (simulation.cc:104-133) with the step on the device.
void Simulation::updateTime() {
  Data* d = data;
  if (env->rank == 0 && (d->iters % d->reportItersPeriod == 0)) std::printf("t = %f\n", d->t);
  double dtX(d->cfl * d->dx / (d->alphaX * sqrt(d->dims)));
  double dtY(d->cfl * d->dy / (d->alphaY * sqrt(d->dims)));
  double dtZ(d->cfl * d->dz / (d->alphaZ * sqrt(d->dims)));
  d->dt = (dtX <= dtY && dtX <= dtZ) ? dtX : ((dtY < dtZ) ? dtY : dtZ);
  if (d->iters < 15) d->dt *= 0.1;
  if (d->iters >= 15 && d->iters < 30) d->dt *= 0.25;
  if (d->t + d->dt > d->endTime) d->dt = d->endTime - d->t;
  mth_handle* h = d->gpu();
  if (!d->deviceCurrent) {
    d->check(mth_upload(h, d->cons, d->prims, d->aux), "updateTime");
    d->deviceCurrent = true;
  }
  d->check(mth_step(h, d->dt), "updateTime");
  d->check(mth_sync(h), "updateTime");
  d->t += d->dt;
  d->iters++;
  if (d->hostSync) syncHost();
}

// Simulation::evolve (simulation.cc:135-171): the state stays on the device
// between output frames.
void Simulation::evolve(bool output, int safety) {
  Data* d = data;
  const bool keep = d->hostSync;
  d->hostSync = false;
  if (output && save) {
    syncHost();
    save->saveVar("rho", 1);
  }
  try {
    while (d->t < d->endTime) {
      updateTime();
      if (output && save && d->iters % d->frameSkip == 0) {
        syncHost();
        save->saveVar("rho", 1);
      }
      if (safety > 0 && d->iters % safety == 0 && save) {
        syncHost();
        save->saveAll(true);
      }
    }
  } catch (...) {
    d->hostSync = keep;
    throw;
  }
  d->hostSync = keep;
  syncHost();
  if (output && save) save->saveVar("rho", 1);
}

// ---------------------------------------------------------------- SaveData
SaveData::SaveData(Data* data, int test) : d(data), Nouts(0), Ncount(0), test(test) {
  dir[0] = '\0';
  app[0] = '\0';
  if (test) std::strcpy(dir, "../../");
}

namespace {

// The device state is authoritative unless the host arrays were changed
// since the last download; bring the device up to date before formatting.
mth_handle* current_device_state(Data* d) {
  mth_handle* h = d->gpu();
  if (!d->deviceCurrent) {
    d->check(mth_upload(h, d->cons, d->prims, d->aux), "save");
    d->deviceCurrent = true;
  }
  return h;
}

FILE* open_or_exit(const std::string& fname, const char* what) {
  FILE* f = std::fopen(fname.c_str(), "w");
  if (!f) {  // the reference prints and exits (serialSaveData.cc:45-48)
    std::printf("Error: could not open '%s' for writing.\n", what);
    std::exit(1);
  }
  return f;
}

void save_device_array(Data* d, const char* dir, const char* app, int which, const char* what) {
  mth_status s = mth_save_text(current_device_state(d), dir, app, which);
  if (s == MTH_ERR_INVALID) {
    std::printf("Error: could not open '%s' for writing.\n", what);
    std::exit(1);
  }
  d->check(s, "save");
}

}  // namespace

void SerialSaveData::saveCons() { save_device_array(d, dir, app, MTH_SAVE_CONS, "cons.dat"); }
void SerialSaveData::savePrims() { save_device_array(d, dir, app, MTH_SAVE_PRIMS, "prims.dat"); }
void SerialSaveData::saveAux() { save_device_array(d, dir, app, MTH_SAVE_AUX, "aux.dat"); }

void SerialSaveData::saveDomain() {
  FILE* f = open_or_exit(std::string(dir) + "/Domain/domain" + app + ".dat", "domain.dat");
  for (int i = 0; i < d->Nx; i++) std::fprintf(f, "%.16f ", d->x[i]);
  std::fprintf(f, "\n");
  for (int j = 0; j < d->Ny; j++) std::fprintf(f, "%.16f ", d->y[j]);
  std::fprintf(f, "\n");
  for (int k = 0; k < d->Nz; k++) std::fprintf(f, "%.16f ", d->z[k]);
  std::fprintf(f, "\n");
  std::fclose(f);
}

void SerialSaveData::saveConsts() {
  FILE* f = open_or_exit(std::string(dir) + "/Constants/constants" + app + ".dat",
                         "constants.dat");
  std::fprintf(f, "constants = nx, ny, nz, Nx, Ny, Nz, xmin, xmax, ymin, ymax, zmin, zmax, "
                  "endTime, cfl, Ng, gamma, sigma, ");
  std::fprintf(f, "Ncons, Nprims, Naux, cp, dt, t, dx, dy, dz\n");
  std::fprintf(f,
               "%d %d %d %d %d %d %.16f %.16f %.16f %.16f %.16f %.16f %.16f %.16f %d %.16f %.16f "
               "%d %d %d %.16f %.16f %.16f %.16f %.16f %.16f\n",
               d->nx, d->ny, d->nz, d->Nx, d->Ny, d->Nz, d->xmin, d->xmax, d->ymin, d->ymax,
               d->zmin, d->zmax, d->endTime, d->cfl, d->Ng, d->gamma, d->sigma, d->Ncons,
               d->Nprims, d->Naux, d->cp, d->dt, d->t, d->dx, d->dy, d->dz);
  std::fclose(f);
}

void SerialSaveData::saveAll(bool timeSeries) {
  dir[0] = '\0';
  if (test) std::strcpy(dir, "../../");
  if (!timeSeries && std::strcmp(dir, "Data/Final") != 0) {
    std::strcat(dir, "Data/Final");
    app[0] = 0;
  } else {
    std::strcat(dir, "Data/TimeSeries");
    std::snprintf(app, sizeof app, "%d", Nouts++);
  }
  saveCons();
  savePrims();
  saveAux();
  saveDomain();
  saveConsts();
}

void SerialSaveData::saveVar(std::string variable, int num) {
  int cpa = 0, nvar = 0;  // cons = 1, prims = 2, aux = 3
  for (int v = 0; v < d->Ncons && !cpa; v++)
    if (d->consLabels[v] == variable) { cpa = 1; nvar = v; }
  for (int v = 0; v < d->Nprims && !cpa; v++)
    if (d->primsLabels[v] == variable) { cpa = 2; nvar = v; }
  for (int v = 0; v < d->Naux && !cpa; v++)
    if (d->auxLabels[v] == variable) { cpa = 3; nvar = v; }
  if (!cpa) {
    std::printf("Error: Could not find user specified variable '%s'\n", variable.c_str());
    std::exit(1);
  }
  if (d->gpu_ && d->deviceCurrent)
    d->check(mth_download(d->gpu_, d->cons, d->prims, d->aux), "save");
  const std::string base = test ? "../../Data/TimeSeries/UserDef/" : "Data/TimeSeries/UserDef/";
  std::snprintf(app, sizeof app, "%d", Nouts);
  FILE* f = std::fopen((base + variable + app + ".dat").c_str(), "w");
  if (!f) {
    std::printf("Error: could not open user-defined file for writing.\n");
    std::exit(1);
  }
  const double* arr = cpa == 1 ? d->cons : (cpa == 2 ? d->prims : d->aux);
  std::fprintf(f, "var = %s, t = %18.16f\n", variable.c_str(), d->t);
  for (int i = 0; i < d->Nx; i++)
    for (int j = 0; j < d->Ny; j++) {
      for (int k = 0; k < d->Nz; k++) std::fprintf(f, "%.16f ", arr[d->id(nvar, i, j, k)]);
      std::fprintf(f, "\n");
    }
  std::fclose(f);
  if (Nouts == 0) {  // the first output lists the saved variables
    const std::string info = base + "info";
    FILE* g = std::fopen(info.c_str(), Ncount == 0 ? "w" : "a");
    if (g) {
      std::fprintf(g, "%s\n", variable.c_str());
      std::fclose(g);
    }
  }
  Ncount++;
  if (Ncount == num) {
    Ncount = 0;
    Nouts++;
  }
}
