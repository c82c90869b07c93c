// A reference-style driver (the wiring of
// Examples/KelvinHelmholtz/SingleFluidIdealSerial/main.cc) built against the
// drop-in headers of include/method_b200/ and linked with libmethod_b200.so.
// Runs the SRMHD Kelvin-Helmholtz shear-layer workload for a few steps and
// writes the final cons and prims as raw doubles to argv[1] and the initial
// prims (after Simulation::set) to argv[2] (when given); with argv[3], also the
// final state as SerialSaveData text files in that directory.
#include "simData.h"
#include "simulation.h"
#include "initFunc.h"
#include "srmhd.h"
#include "boundaryConds.h"
#include "RK2.h"
#include "fluxVectorSplitting.h"
#include "serialEnv.h"
#include "serialSaveData.h"
#include "weno.h"
#include <cstdio>
#include <cstring>

int main(int argc, char* argv[]) {
  int Ng(4), nx(64), ny(128), nz(0);
  double xmin(-0.5), xmax(0.5), ymin(-1.0), ymax(1.0), zmin(0.0), zmax(1.0);
  double endTime(3.0), cfl(0.4), gamma(4.0 / 3.0), sigma(0), cp(0.1);
  SerialEnv env(&argc, &argv, 1, 1, 1);
  Data data(nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax, endTime, &env, cfl, Ng, gamma, sigma,
            cp, -1e4, 1e4, 10, 1 << 30);
  SRMHD model(&data);
  Weno3 weno(&data);
  FVS fluxMethod(&data, &weno, &model);
  Flow bcs(&data);
  Simulation sim(&data, &env);
  KHShearLayerSingleFluid init(&data, 1234);
  RK2 timeInt(&data, &model, &bcs, &fluxMethod);
  sim.set(&init, &model, &timeInt, &bcs, &fluxMethod, NULL);
  FILE* f0 = argc > 2 ? std::fopen(argv[2], "wb") : NULL;
  if (f0) {
    std::fwrite(data.prims, sizeof(double), (size_t)data.Nprims * data.Ntot, f0);
    std::fclose(f0);
  }
  for (int s = 0; s < 20; ++s) sim.updateTime();
  std::printf("t = %.17g iters = %d rho[center] = %.17g\n", data.t, data.iters,
              data.prims[data.id(0, data.Nx / 2, data.Ny / 2, 0)]);
  if (argc > 1) {
    FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(data.cons, sizeof(double), (size_t)data.Ncons * data.Ntot, f);
    std::fwrite(data.prims, sizeof(double), (size_t)data.Nprims * data.Ntot, f);
    std::fclose(f);
  }
  if (argc > 3) {
    SerialSaveData save(&data, &env);
    std::strcpy(save.dir, argv[3]);
    save.saveCons();
    save.savePrims();
    save.saveAux();
    save.saveDomain();
    save.saveConsts();
  }
  return 0;
}
