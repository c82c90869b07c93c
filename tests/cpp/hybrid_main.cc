// A reference-style Hybrid driver (the wiring of Examples/Hybrid/*/main.cc:
// Hybrid model, FVS, model.setupREGIME(&fluxMethod), RKSplit2) built against
// the drop-in headers of include/method_b200/ and linked with
// libmethod_b200.so.  Orszag-Tang on the unit square, WENO3, periodic,
// sigma 170 (inside the blend band), eight steps; writes the final cons and
// prims as raw doubles to argv[1] and the initial prims to argv[2].
#include "simData.h"
#include "simulation.h"
#include "initFunc.h"
#include "hybrid.h"
#include "boundaryConds.h"
#include "rkSplit2ndOrder.h"
#include "fluxVectorSplitting.h"
#include "serialEnv.h"
#include "weno.h"
#include <cstdio>

int main(int argc, char* argv[]) {
  int Ng(4), nx(32), ny(32), nz(0);
  double xmin(0.0), xmax(1.0), ymin(0.0), ymax(1.0), zmin(0.0), zmax(1.0);
  double endTime(1.0), cfl(0.3), gamma(2.0), sigma(170), cp(1.0);
  double sigmaCrossOver(150), sigmaSpan(50);
  bool useREGIME(true);
  SerialEnv env(&argc, &argv, 1, 1, 1);
  Data data(nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax, endTime, &env, cfl, Ng, gamma, sigma,
            cp, -1e4, 1e4, 10, 1 << 30);
  Hybrid model(&data, sigmaCrossOver, sigmaSpan, useREGIME);
  Weno3 weno(&data);
  FVS fluxMethod(&data, &weno, &model);
  model.setupREGIME(&fluxMethod);
  Periodic bcs(&data);
  Simulation sim(&data, &env);
  OTVortexSingleFluid init(&data);
  RKSplit2 timeInt(&data, &model, &bcs, &fluxMethod, NULL);
  sim.set(&init, &model, &timeInt, &bcs, &fluxMethod, NULL);
  if (argc > 2) {
    FILE* f0 = std::fopen(argv[2], "wb");
    std::fwrite(data.prims, sizeof(double), (size_t)data.Nprims * data.Ntot, f0);
    std::fclose(f0);
  }
  for (int s = 0; s < 8; ++s) sim.updateTime();
  std::printf("t = %.17g iters = %d\n", data.t, data.iters);
  if (argc > 1) {
    FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(data.cons, sizeof(double), (size_t)data.Ncons * data.Ntot, f);
    std::fwrite(data.prims, sizeof(double), (size_t)data.Nprims * data.Ntot, f);
    std::fclose(f);
  }
  return 0;
}
