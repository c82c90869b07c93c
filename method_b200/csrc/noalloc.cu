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
//
// The array's device address belongs to a CUDA context, not to a device
// number: after cudaDeviceReset, or when a caller makes a context of its own
// current through the driver API, the same device has a new address.  The
// address is therefore cached per context, keyed on the context's
// process-unique id (cuCtxGetId), and looked up by cudaGetSymbolAddress the
// first time a context calls.
#include <climits>
#include <cstdio>
#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "launch.h"
#include "../../include/method_b200.h"

namespace {

constexpr long long kMaxCells = MTH_NOALLOC_MAX_CELLS;  // interior cells per call
constexpr size_t kListBytes = sizeof(int) * (size_t)kMaxCells;
constexpr size_t kCountOffset = kListBytes;         // one int, padded to 256 B
constexpr size_t kCountersOffset = kListBytes + 256;  // 16 long long
constexpr size_t kScratchBytes = kCountersOffset + 16 * sizeof(long long);

// Shared by every call in a context; keeps the previous call's contents.
static __device__ __align__(256) unsigned char g_c2p_scratch[kScratchBytes];

typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

struct CachedAddress {
  unsigned long long ctx_id;  // 0: empty slot
  void* addr;
};

constexpr int kSlots = 64;
std::mutex g_mu;
CachedAddress g_cache[kSlots] = {};
int g_next_slot = 0;
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;

// Id of the calling thread's current context (0 when none is current).  The
// two driver functions are resolved through the runtime, so the library does
// not link libcuda itself.  Caller holds g_mu.
cudaError_t current_context_id(unsigned long long* id) {
  *id = 0;
  if (!g_ctx_get_current || !g_ctx_get_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    void *f1 = nullptr, *f2 = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    if (e != cudaSuccess || q1 != cudaDriverEntryPointSuccess || !f1)
      return e != cudaSuccess ? e : cudaErrorSymbolNotFound;
    e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e != cudaSuccess || q2 != cudaDriverEntryPointSuccess || !f2)
      return e != cudaSuccess ? e : cudaErrorSymbolNotFound;
    g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
    g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f2);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  if (!ctx) return cudaSuccess;
  if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  return cudaSuccess;
}

// Device address of g_c2p_scratch in the current context.  In host code the
// name g_c2p_scratch is only a host-side stand-in, so kernels must receive
// this address, never the name.  The first call in a context runs
// cudaGetSymbolAddress (which also makes the device's primary context current
// if no context is); later calls in that context only read the cache.
cudaError_t scratch_address(void** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  unsigned long long id = 0;
  cudaError_t e = current_context_id(&id);
  if (e != cudaSuccess) return e;
  if (id) {
    for (const CachedAddress& c : g_cache)
      if (c.ctx_id == id) {
        *out = c.addr;
        return cudaSuccess;
      }
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_c2p_scratch);
  if (e != cudaSuccess) return e;
  e = current_context_id(&id);  // a context exists now
  if (e != cudaSuccess) return e;
  if (!id) return cudaErrorDeviceUninitialized;
  g_cache[g_next_slot] = CachedAddress{id, p};
  g_next_slot = (g_next_slot + 1) % kSlots;
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" mth_status mth_c2p_srmhd_noalloc(int nx, int ny, int nz, int Ng, double gamma,
                                            const double* cons, const double* prims_guess,
                                            const double* aux_guess, double* prims, double* aux,
                                            double* solution, void* stream,
                                            long long* unconverged) {
  using namespace mth;
  if (nx <= 0 || ny < 0 || nz < 0 || (ny == 0 && nz != 0) || Ng < 1 || !cons || !prims_guess ||
      !aux_guess || !prims || !aux || !solution)
    return MTH_ERR_INVALID;
  // ghost-inclusive extents and cell ids are ints on the device
  const long long Nx = (long long)nx + 2LL * Ng;
  const long long Ny = ny == 0 ? 1 : (long long)ny + 2LL * Ng;
  const long long Nz = nz == 0 ? 1 : (long long)nz + 2LL * Ng;
  if (Nx > INT_MAX || Ny > INT_MAX || Nz > INT_MAX || Nx * Ny > INT_MAX || Nx * Ny * Nz > INT_MAX) {
    std::fprintf(stderr,
                 "mth_c2p_srmhd_noalloc: a grid of %lld x %lld x %lld cells (ghosts included) "
                 "has cell ids beyond the int range\n",
                 Nx, Ny, Nz);
    return MTH_ERR_INVALID;
  }
  Grid g{};
  g.nx = nx; g.ny = ny; g.nz = nz; g.Ng = Ng;
  g.Nx = (int)Nx; g.Ny = (int)Ny; g.Nz = (int)Nz;
  g.dims = nz == 0 ? (ny == 0 ? 1 : 2) : 3;
  g.is = Ng; g.ie = g.Nx - Ng;
  g.js = Ng; g.je = g.Ny - Ng;
  g.ks = Ng; g.ke = g.Nz - Ng;
  if (g.dims < 3) { g.ks = 0; g.ke = 1; }
  if (g.dims < 2) { g.js = 0; g.je = 1; }
  g.gamma = gamma;
  g.Ntot = Nx * Ny * Nz;
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
  long long* counters = reinterpret_cast<long long*>(b + kCountersOffset);
  C2PWork w{reinterpret_cast<int*>(b), reinterpret_cast<int*>(b + kCountOffset), counters};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the failure count and the counters must start at zero in every call
  if (cudaMemsetAsync(b + kCountOffset, 0, kScratchBytes - kCountOffset, st) != cudaSuccess)
    return MTH_ERR_CUDA;
  if (launch_c2p_srmhd(g, cons, prims_guess, aux_guess, prims, aux, solution, w, st) !=
      cudaSuccess)
    return MTH_ERR_CUDA;
  if (unconverged) {
    // counters[2]: cells the neighbour-average retry left unconverged
    if (cudaMemcpyAsync(unconverged, counters + 2, sizeof(long long), cudaMemcpyDeviceToHost,
                        st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return MTH_ERR_CUDA;
  }
  return MTH_OK;
}
