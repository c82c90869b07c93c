// C++ drop-in for the hot path of METHOD's class API, running on the B200
// through the C ABI of method_b200.h.
//
// Class names, constructor arguments and method signatures follow the
// reference (Project/CPU/Include/{simData,platformEnv,serialEnv,model,srmhd,
// srrmhd,flux,fluxVectorSplitting,weno,boundaryConds,timeInt,RK2,rkSplit,
// SSP2,SSP3,SSP2322,initFunc,simulation}.h), so a reference driver such as
// Examples/KelvinHelmholtz/SingleFluidIdealSerial/main.cc compiles against
// these headers and links against libmethod_b200.so.  The per-name headers
// in this directory (simData.h, simulation.h, ...) all include this file.
//
// State: Simulation allocates the host arrays d->cons/prims/aux exactly as
// the reference does (simulation.cc:22-30).  The device copy is the working
// state: Simulation::updateTime steps on the device and, when
// Data::hostSync is true (the default), copies the new state back into the
// host arrays so that code reading them after each step sees the reference's
// values.  Simulation::evolve keeps the state on the device and copies it
// back when it returns.  Model / FluxMethod / Bcs / TimeIntegrator methods
// that take host arrays run the device kernels on those arrays.
//
// Errors: non-convergence throws std::runtime_error, invalid configurations
// std::invalid_argument, as in the reference.
#ifndef METHOD_B200_METHOD_HPP
#define METHOD_B200_METHOD_HPP

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "../method_b200.h"

#define ID(variable, idx, jdx, kdx) \
  ((variable) * (d->Nx) * (d->Ny) * (d->Nz) + (idx) * (d->Ny) * (d->Nz) + (jdx) * (d->Nz) + (kdx))

class Model;
class WenoBase;
class FluxMethod;
class Bcs;
class TimeIntegrator;

// ---------------------------------------------------------------- platform
class PlatformEnv {
 public:
  int nProc = 1, rank = 0, nxRanks = 1, nyRanks = 1, nzRanks = 1;
  int xRankId = 0, yRankId = 0, zRankId = 0;
  int leftXNeighbourRank = 0, rightXNeighbourRank = 0, leftYNeighbourRank = 0,
      rightYNeighbourRank = 0, leftZNeighbourRank = 0, rightZNeighbourRank = 0;
  int isLeftBoundary = 1, isRightBoundary = 1, isTopBoundary = 1, isBottomBoundary = 1,
      isFrontBoundary = 1, isBackBoundary = 1;
  int testing = 0;
  explicit PlatformEnv(int testing = 0) : testing(testing) {}
  virtual ~PlatformEnv() {}
};

// Single process, single GPU (serialEnv.h:18-30).
class SerialEnv : public PlatformEnv {
 public:
  SerialEnv(int* argcP, char** argvP[], int nxRanks, int nyRanks, int nzRanks, int testing = 0);
  virtual ~SerialEnv() {}
};

// -------------------------------------------------------------------- Data
class Data {
 public:
  int nx, ny, nz;
  double xmin, xmax, ymin, ymax, zmin, zmax, endTime, cfl;
  int Ng;
  double gamma, sigma;
  int memSet, bcsSet;
  int Ncons, Nprims, Naux;
  double cp, mu1, mu2;
  int frameSkip, reportItersPeriod;
  bool functionalSigma;
  double gam;
  double t, dt, dx, dy, dz;
  double alphaX, alphaY, alphaZ;
  int iters, Nx, Ny, Nz, Ntot, dims, is, ie, js, je, ks, ke;
  double *cons, *prims, *aux, *f, *fnet, *source, *sourceExtension, *x, *y, *z;
  std::vector<std::string> consLabels, primsLabels, auxLabels;
  int nOptionalSimArgs = 0;
  std::vector<double> optionalSimArgs;
  std::vector<std::string> optionalSimArgNames;

  // ---- B200 additions
  bool hostSync = true;  // copy the state to the host arrays after every updateTime
  int device = 0;        // CUDA device of this simulation
  int precision = MTH_PLAIN_FP64;
  int guess = MTH_GUESS_PREVIOUS;
  Model* model_ = nullptr;
  WenoBase* weno_ = nullptr;
  Bcs* bcs_ = nullptr;
  TimeIntegrator* timeInt_ = nullptr;
  mth_handle* gpu_ = nullptr;
  bool deviceCurrent = false;  // device state newer than / equal to the host arrays

  Data(int nx, int ny, int nz, double xmin, double xmax, double ymin, double ymax, double zmin,
       double zmax, double endTime, PlatformEnv* env, double cfl = 0.5, int Ng = 4,
       double gamma = 5.0 / 3.0, double sigma = 1e3, double cp = 0.1, double mu1 = -1.0e4,
       double mu2 = 1.0e4, int frameskip = 10, int reportItersPeriod = 1,
       bool funtionalSigma = false, double gam = 12);
  ~Data();

  int id(int var, int i, int j, int k) {
    return var * Nx * Ny * Nz + i * Ny * Nz + j * Nz + k;
  }
  double sigmaFunc(double* cons, double* prims, double* aux, int i = -1, int j = -1, int k = -1);

  // The device handle for the current component choice (created on demand).
  mth_handle* gpu();
  void invalidateGpu();
  void check(mth_status s, const char* what);
};

// ------------------------------------------------------------------- Model
class Model {
 public:
  Data* data = nullptr;
  int Ncons = 0, Nprims = 0, Naux = 0;
  Model() {}
  explicit Model(Data* data) : data(data) {}
  virtual ~Model() {}
  virtual int modelId() const = 0;
  virtual void sourceTermSingleCell(double* cons, double* prims, double* aux, double* source,
                                    int i = -1, int j = -1, int k = -1) = 0;
  virtual void sourceTerm(double* cons, double* prims, double* aux, double* source);
  virtual void getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int i = -1,
                                          int j = -1, int k = -1) = 0;
  virtual void getPrimitiveVars(double* cons, double* prims, double* aux);
  virtual void primsToAll(double* cons, double* prims, double* aux);
  virtual void fluxVector(double* cons, double* prims, double* aux, double* f, int dir);
  virtual void finalise(double* cons, double* prims, double* aux) {}
};

// Ideal SRMHD (srmhd.h:93-301).
class SRMHD : public Model {
 public:
  SRMHD();
  explicit SRMHD(Data* data);
  int modelId() const override { return MTH_SRMHD; }
  void sourceTermSingleCell(double* cons, double* prims, double* aux, double* source, int i = -1,
                            int j = -1, int k = -1) override;
  void getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int i = -1,
                                  int j = -1, int k = -1) override;
};

// Resistive SRMHD (srrmhd.h:77-204).
class SRRMHD : public Model {
 public:
  SRRMHD();
  explicit SRRMHD(Data* data);
  int modelId() const override { return MTH_SRRMHD; }
  void sourceTermSingleCell(double* cons, double* prims, double* aux, double* source, int i = -1,
                            int j = -1, int k = -1) override;
  void getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int i = -1,
                                  int j = -1, int k = -1) override;
};

// The Hybrid model (hybrid.h:33-296): SRRMHD's variables, the ideal and
// resistive models blended by the conductivity (weight 0 below
// sigmaCrossOver - sigmaSpan, 1 above sigmaCrossOver + sigmaSpan), with the
// REGIME term on the ideal part when useREGIME.  Runs inside the device step
// (RK2 or RKSplit2); its single-cell methods are not provided on the host.
class Hybrid : public Model {
 public:
  double sigmaCrossOver = 150, sigmaSpan = 50;
  bool useREGIME = true;
  Hybrid();
  Hybrid(Data* data, double sigmaCrossOver = 150, double sigmaSpan = 50, bool useREGIME = true);
  int modelId() const override { return MTH_HYBRID; }
  // The device step builds the REGIME term from the flux method's WENO order.
  void setupREGIME(FluxMethod* fluxMethod) { (void)fluxMethod; }
  void sourceTermSingleCell(double* cons, double* prims, double* aux, double* source, int i = -1,
                            int j = -1, int k = -1) override;
  void getPrimitiveVarsSingleCell(double* cons, double* prims, double* aux, int i = -1,
                                  int j = -1, int k = -1) override;
};

// -------------------------------------------------------------------- WENO
class WenoBase {
 public:
  Data* data;
  int order, shift;
  WenoBase(Data* data, int order);
  virtual ~WenoBase() {}
  void checkSufficientGhostZones();
};
class Weno3 : public WenoBase {
 public:
  explicit Weno3(Data* data) : WenoBase(data, 3) {}
};
class Weno5 : public WenoBase {
 public:
  explicit Weno5(Data* data) : WenoBase(data, 5) {}
};
// Higher orders (weno.h:346-624): the same Jiang-Shu scheme on 7, 9, 11 points.
class Weno7 : public WenoBase {
 public:
  explicit Weno7(Data* data) : WenoBase(data, 7) {}
};
class Weno9 : public WenoBase {
 public:
  explicit Weno9(Data* data) : WenoBase(data, 9) {}
};
class Weno11 : public WenoBase {
 public:
  explicit Weno11(Data* data) : WenoBase(data, 11) {}
};

// ------------------------------------------------------------ flux methods
class FluxMethod {
 public:
  Data* data;
  Model* model;
  FluxMethod(Data* data, Model* model) : data(data), model(model) {}
  virtual ~FluxMethod() {}
  virtual void F(double* cons, double* prims, double* aux, double* f, double* fnet) = 0;
};

// Flux vector splitting with WENO reconstruction (fluxVectorSplitting.h:68-126).
class FVS : public FluxMethod {
 public:
  WenoBase* weno;
  FVS(Data* data, WenoBase* weno, Model* model);
  virtual ~FVS() {}
  void F(double* cons, double* prims, double* aux, double* f, double* fnet) override;
};

// ---------------------------------------------------- boundary conditions
class Bcs {
 public:
  Data* data;
  explicit Bcs(Data* data);
  virtual ~Bcs() {}
  virtual int bcId() const = 0;
  virtual void apply(double* cons, double* prims = NULL, double* aux = NULL);
};
class Outflow : public Bcs {
 public:
  explicit Outflow(Data* data) : Bcs(data) {}
  int bcId() const override { return MTH_OUTFLOW; }
};
class Periodic : public Bcs {
 public:
  explicit Periodic(Data* data) : Bcs(data) {}
  int bcId() const override { return MTH_PERIODIC; }
};
class Flow : public Bcs {
 public:
  explicit Flow(Data* data) : Bcs(data) {}
  int bcId() const override { return MTH_FLOW; }
};

// ---------------------------------------------------------- model extensions
// A source an integrator adds to the model's (modelExtension.h:13-50).
class ModelExtension {
 public:
  Data* data = nullptr;
  bool sourceExists = false;
  bool fluxExists = false;
  ModelExtension() {}
  explicit ModelExtension(Data* data) : data(data) {}
  virtual ~ModelExtension() {}
  // 0: none this library evaluates; 1: REGIME.
  virtual int extensionId() const { return 0; }
};
// REGIME, the resistive extension of ideal SRMHD (REGIME.h:81-160).  Only
// RKSplit applies a model extension (rkSplit.cc:15-16), and it does so on
// the device; REGIME with another model is rejected.
class REGIME : public ModelExtension {
 public:
  FluxMethod* fluxMethod = nullptr;
  REGIME() {}
  REGIME(Data* data, FluxMethod* fluxMethod) : ModelExtension(data), fluxMethod(fluxMethod) {
    sourceExists = true;
  }
  int extensionId() const override { return 1; }
};

// --------------------------------------------------------- time integrators
class TimeIntegrator {
 public:
  Data* data;
  Model* model;
  Bcs* bcs;
  FluxMethod* fluxMethod;
  ModelExtension* modelExtension = nullptr;
  TimeIntegrator(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod);
  virtual ~TimeIntegrator() {}
  virtual int integratorId() const = 0;
  // One step on host arrays (timeInt.h:61); dt <= 0 means data->dt.
  virtual void step(double* cons, double* prims, double* aux, double dt = 0);
  // C2P, model finalise and boundary conditions (timeInt.h:117-132).
  void finalise(double* cons, double* prims, double* aux);
};
class RK2 : public TimeIntegrator {
 public:
  RK2(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod,
      ModelExtension* modelExtension = NULL)
      : TimeIntegrator(data, model, bcs, fluxMethod) {
    this->modelExtension = modelExtension;
  }
  int integratorId() const override { return MTH_RK2; }
};
class RKSplit : public RK2 {
 public:
  RKSplit(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod,
          ModelExtension* modelExtension = NULL)
      : RK2(data, model, bcs, fluxMethod, modelExtension) {}
  int integratorId() const override { return MTH_RKSPLIT; }
};
// Second-order (Strang) split: half source, RK2, half source
// (rkSplit2ndOrder.h:42-76).
class RKSplit2 : public RK2 {
 public:
  RKSplit2(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod,
           ModelExtension* modelExtension = NULL)
      : RK2(data, model, bcs, fluxMethod, modelExtension) {}
  int integratorId() const override { return MTH_RKSPLIT2; }
};
class SSP2 : public TimeIntegrator {
 public:
  SSP2(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod)
      : TimeIntegrator(data, model, bcs, fluxMethod) {}
  int integratorId() const override { return MTH_SSP2; }
};
// IMEX SSP3(332) (SSP3.h:34) and SSP2(322) (SSP2322.h:34), both derived from
// SSP2 as in the reference.
class SSP3 : public SSP2 {
 public:
  SSP3(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod)
      : SSP2(data, model, bcs, fluxMethod) {}
  int integratorId() const override { return MTH_SSP3; }
};
class SSP2322 : public SSP2 {
 public:
  SSP2322(Data* data, Model* model, Bcs* bcs, FluxMethod* fluxMethod)
      : SSP2(data, model, bcs, fluxMethod) {}
  int integratorId() const override { return MTH_SSP2322; }
};

// ------------------------------------------------------------ initial data
// The base class zeroes the state (initFunc.cc:10-40); subclasses set
// d->prims in every cell, ghosts included.
class InitialFunc {
 public:
  Data* data;
  explicit InitialFunc(Data* data);
  virtual ~InitialFunc() {}
};
// Reference Orszag-Tang set-up (initFunc.cc:229-272).
class OTVortexSingleFluid : public InitialFunc {
 public:
  explicit OTVortexSingleFluid(Data* data);
};
// Measured workloads (not reference classes): see method_b200/initial.py.
class KHShearLayerSingleFluid : public InitialFunc {  // SRMHD/SRRMHD KH, seeded vy noise
 public:
  KHShearLayerSingleFluid(Data* data, int seed = 1234, double shear = 0.5);
};
class OrszagTangUnit : public InitialFunc {  // rho = p = 1 Orszag-Tang
 public:
  explicit OrszagTangUnit(Data* data);
};
class HarrisCurrentSheet : public InitialFunc {  // SRRMHD sheet By = tanh(x / 0.01), p = 50
 public:
  HarrisCurrentSheet(Data* data, int seed = 1234);
};

// ------------------------------------------------------------------ output
// SaveData (saveData.h:17-95) and SerialSaveData (serialSaveData.h:23-86):
// the same members, file layout and text format.  The cons / prims / aux
// files are formatted on the device (mth_save_text); domain and constants
// are written from Data.
class SaveData {
 public:
  Data* d = nullptr;
  int Nouts = 0, Ncount = 0, test = 0;
  char dir[50], app[50];
  SaveData() { dir[0] = app[0] = '\0'; }
  SaveData(Data* data, int test = 0);
  virtual ~SaveData() {}
  virtual void saveAll(bool timeSeries = false) {}
  virtual void saveVar(std::string variable, int num = 1) {}
};
class SerialSaveData : public SaveData {
 public:
  SerialEnv* env = nullptr;
  SerialSaveData(Data* data, SerialEnv* env, int test = 0) : SaveData(data, test), env(env) {}
  virtual ~SerialSaveData() {}
  void saveCons();
  void savePrims();
  void saveAux();
  void saveDomain();
  void saveConsts();
  // All of the above into Data/Final, or Data/TimeSeries with app = Nouts++
  // (serialSaveData.cc:8-29).
  void saveAll(bool timeSeries = false) override;
  // One variable, every cell, into Data/TimeSeries/UserDef (serialSaveData.cc:248-361).
  void saveVar(std::string variable, int num = 1) override;
};

// -------------------------------------------------------------- simulation
class Simulation {
 public:
  Data* data;
  PlatformEnv* env;
  InitialFunc* init = nullptr;
  Model* model = nullptr;
  TimeIntegrator* timeInt = nullptr;
  Bcs* bcs = nullptr;
  FluxMethod* fluxMethod = nullptr;
  SaveData* save = nullptr;
  Simulation(Data* data, PlatformEnv* env);
  ~Simulation();
  void set(InitialFunc* init, Model* model, TimeIntegrator* timeInt, Bcs* bcs,
           FluxMethod* fluxMethod, SaveData* save = NULL);
  void updateTime();
  void evolve(bool output = false, int safety = -1);
  // Copies the device state into d->cons/prims/aux (no-op when current).
  void syncHost();
};

#endif  // METHOD_B200_METHOD_HPP
