// Factory for the reference's SSP2322 integrator, in a translation unit of
// its own: the reference's SSP2322.h and SSP3.h share one include guard
// (SSP3_H), so the two headers cannot be included together.  Test
// infrastructure only (see ref_driver.cc).
#include "SSP2322.h"

TimeIntegrator* mref_new_ssp2322(Data* data, Model* model, Bcs* bcs, FluxMethod* flux) {
  return new SSP2322(data, model, bcs, flux);
}
