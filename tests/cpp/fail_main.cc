// Failure paths of the drop-in classes, driven the way a reference main.cc
// would meet them: each case prints one line "<case> <outcome>" where the
// outcome is the exception type the call threw ("runtime_error",
// "invalid_argument") or "ok".  The reference throws std::runtime_error for
// non-convergence (srrmhd.cc:576-579, srmhd.cc:345, SSP2.cc:89-98) and
// std::invalid_argument for a bad configuration (simData.cc:100-106).
#include "simData.h"
#include "simulation.h"
#include "initFunc.h"
#include "srmhd.h"
#include "srrmhd.h"
#include "boundaryConds.h"
#include "SSP2.h"
#include "RK2.h"
#include "fluxVectorSplitting.h"
#include "serialEnv.h"
#include "weno.h"
#include <cmath>
#include <cstdio>
#include <limits>
#include <stdexcept>

template <class F>
void run(const char* name, F f) {
  const char* outcome = "ok";
  try {
    f();
  } catch (const std::invalid_argument&) {
    outcome = "invalid_argument";
  } catch (const std::runtime_error&) {
    outcome = "runtime_error";
  } catch (...) {
    outcome = "other";
  }
  std::printf("%s %s\n", name, outcome);
}

int main(int argc, char* argv[]) {
  SerialEnv env(&argc, &argv, 1, 1, 1);
  const double nan = std::numeric_limits<double>::quiet_NaN();

  // SRRMHD grid C2P of a state with one NaN cell: the secant fails and throws.
  run("srrmhd_c2p_nan", [&] {
    Data d(16, 32, 0, -0.5, 0.5, -1.0, 1.0, 0.0, 1.0, 1.0, &env, 0.4, 4, 4.0 / 3.0, 1e3);
    SRRMHD model(&d);
    Weno3 weno(&d);
    FVS flux(&d, &weno, &model);
    Outflow bcs(&d);
    Simulation sim(&d, &env);
    HarrisCurrentSheet init(&d, 5);
    SSP2 ti(&d, &model, &bcs, &flux);
    sim.set(&init, &model, &ti, &bcs, &flux, NULL);
    d.cons[d.id(0, 9, 20, 0)] = nan;
    model.getPrimitiveVars(d.cons, d.prims, d.aux);
  });
  // The same state, unchanged: recovers.
  run("srrmhd_c2p_clean", [&] {
    Data d(16, 32, 0, -0.5, 0.5, -1.0, 1.0, 0.0, 1.0, 1.0, &env, 0.4, 4, 4.0 / 3.0, 1e3);
    SRRMHD model(&d);
    Weno3 weno(&d);
    FVS flux(&d, &weno, &model);
    Outflow bcs(&d);
    Simulation sim(&d, &env);
    HarrisCurrentSheet init(&d, 5);
    SSP2 ti(&d, &model, &bcs, &flux);
    sim.set(&init, &model, &ti, &bcs, &flux, NULL);
    model.getPrimitiveVars(d.cons, d.prims, d.aux);
  });
  // One SSP2 step of a state with a NaN cell: the implicit stage fails.
  run("ssp2_step_nan", [&] {
    Data d(16, 32, 0, -0.5, 0.5, -1.0, 1.0, 0.0, 1.0, 1.0, &env, 0.4, 4, 4.0 / 3.0, 1e3);
    SRRMHD model(&d);
    Weno3 weno(&d);
    FVS flux(&d, &weno, &model);
    Outflow bcs(&d);
    Simulation sim(&d, &env);
    HarrisCurrentSheet init(&d, 5);
    SSP2 ti(&d, &model, &bcs, &flux);
    sim.set(&init, &model, &ti, &bcs, &flux, NULL);
    d.cons[d.id(4, 10, 12, 0)] = nan;
    ti.step(d.cons, d.prims, d.aux, 1e-4);
  });
  // SRMHD single-cell C2P with a guess it cannot leave (v^2 > 1): throws.
  run("srmhd_single_cell_bad", [&] {
    Data d(8, 8, 0, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 1.0, &env, 0.4, 4, 4.0 / 3.0, 0.0);
    SRMHD model(&d);
    double cons[9] = {1.2, 0.3, 0.1, 0.0, 2.0, 0.5, 0.2, 0.1, 0.0};
    double prims[8] = {1.0, 1.2, 0.1, 0.0, 1.0, 0.5, 0.2, 0.1};
    double aux[13] = {5.0};
    model.getPrimitiveVarsSingleCell(cons, prims, aux);
  });
  // Negative conductivity is a configuration error.
  run("negative_sigma", [&] {
    Data d(8, 8, 0, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 1.0, &env, 0.4, 4, 4.0 / 3.0, -1.0);
  });
  return 0;
}
