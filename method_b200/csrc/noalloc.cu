// SRMHD primitive recovery for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to call cudaMalloc: a host
// application that hands out all device memory from its own fixed-budget
// pool, or a latency-critical stepping loop in which an allocation (and the
// device synchronisation cudaMalloc may imply) is not acceptable.  They still
// own the arrays of the state, so they pass inputs and outputs; the only
// memory this entry point needs beyond those arrays -- the queue of cells
// whose Powell-hybrid solve failed and the per-call counters -- lives in the
// file-scope array below, which every GPU that loads the library holds until
// the process exits (about 4 MiB).
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "launch.h"
#include "../../include/method_b200.h"

namespace {

constexpr long long kMaxCells = MTH_NOALLOC_MAX_CELLS;  // interior cells per call
constexpr size_t kListBytes = sizeof(int) * (size_t)kMaxCells;
constexpr size_t kCountOffset = kListBytes;         // one int, padded to 256 B
constexpr size_t kCountersOffset = kListBytes + 256;  // 16 long long
constexpr size_t kScratchBytes = kCountersOffset + 16 * sizeof(long long);

// Shared by every call on a device; keeps the previous call's contents.
static __device__ __align__(256) unsigned char g_c2p_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of g_c2p_scratch on the current device, looked up once per
// device.  In host code the name g_c2p_scratch is only a host-side stand-in,
// so kernels must receive this address, never the name.
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_c2p_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" mth_status mth_c2p_srmhd_noalloc(int nx, int ny, int nz, int Ng, double gamma,
                                            const double* cons, const double* prims_guess,
                                            const double* aux_guess, double* prims, double* aux,
                                            double* solution, void* stream) {
  using namespace mth;
  if (nx <= 0 || ny < 0 || nz < 0 || (ny == 0 && nz != 0) || Ng < 1 || !cons || !prims_guess ||
      !aux_guess || !prims || !aux || !solution)
    return MTH_ERR_INVALID;
  Grid g{};
  g.nx = nx; g.ny = ny; g.nz = nz; g.Ng = Ng;
  g.Nx = nx + 2 * Ng; g.Ny = ny + 2 * Ng; g.Nz = nz + 2 * Ng;
  g.dims = 3;
  if (nz == 0) { g.Nz = 1; g.dims = 2; }
  if (ny == 0) { g.Nz = g.Ny = 1; g.dims = 1; }
  g.is = Ng; g.ie = g.Nx - Ng;
  g.js = Ng; g.je = g.Ny - Ng;
  g.ks = Ng; g.ke = g.Nz - Ng;
  if (g.dims < 3) { g.ks = 0; g.ke = 1; }
  if (g.dims < 2) { g.js = 0; g.je = 1; }
  g.gamma = gamma;
  g.Ntot = (long long)g.Nx * g.Ny * g.Nz;
  const long long n = (long long)(g.ie - g.is) * (g.je - g.js) * (g.ke - g.ks);
  if (n > kMaxCells) {
    std::fprintf(stderr,
                 "mth_c2p_srmhd_noalloc: %lld interior cells exceed the fixed scratch capacity "
                 "of %lld cells\n",
                 n, kMaxCells);
    return MTH_ERR_INVALID;
  }
  void* base = nullptr;
  if (scratch_address(&base) != cudaSuccess) return MTH_ERR_CUDA;
  unsigned char* b = static_cast<unsigned char*>(base);
  C2PWork w{reinterpret_cast<int*>(b), reinterpret_cast<int*>(b + kCountOffset),
            reinterpret_cast<long long*>(b + kCountersOffset)};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the failure count and the counters must start at zero in every call
  if (cudaMemsetAsync(b + kCountOffset, 0, kScratchBytes - kCountOffset, st) != cudaSuccess)
    return MTH_ERR_CUDA;
  if (launch_c2p_srmhd(g, cons, prims_guess, aux_guess, prims, aux, solution, w, st) !=
      cudaSuccess)
    return MTH_ERR_CUDA;
  return MTH_OK;
}
