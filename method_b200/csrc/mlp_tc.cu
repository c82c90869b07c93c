// Guess network inference on the fifth-generation tensor cores (tcgen05).
//
// The same network, weights and rounding points as the warp-level path of
// mlp.cu (BF16 weights and activations, FP32 accumulation, ReLU between
// layers), computed as four M = 128 matrix products per tile of 128 cells.
// Each warpgroup of a CTA (two per CTA, sharing the weights) owns a tile:
//   * one thread per cell stages the cell's standardised features as BF16 in
//     shared memory (row m of the warpgroup's A operand);
//   * one thread issues `tcgen05.mma.cta_group::1.kind::f16` with A and the
//     layer's weights (B) read from shared memory through matrix
//     descriptors, the FP32 product accumulating in tensor memory (TMEM,
//     64 columns per warpgroup), and `tcgen05.commit` signals the
//     warpgroup's mbarrier;
//   * every thread then reads its own row back from TMEM (`tcgen05.ld`, warp
//     w owns TMEM lanes 32 (w mod 4) .. 32 (w mod 4) + 31), adds the bias,
//     applies ReLU, rounds to BF16 and writes the next layer's A row.
// Operands use the K-major layout without swizzle: 8-row x 16-byte core
// matrices, the two 8-element K halves of a 16-wide K slab 128 bytes apart
// (leading byte offset), 8-row groups 256 bytes apart (stride byte offset),
// K slabs one after another; the descriptor and instruction-descriptor
// fields follow the PTX ISA's tcgen05 matrix and instruction descriptors.
//
// Every wait on an mbarrier is bounded; a wait that runs out stops the
// warpgroup's remaining tiles, sets the error word and still frees the CTA's
// TMEM.  The solver uses the warp-level path of mlp.cu by default (faster for
// this small network on B200, mlp.cu: kTcInference).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "common.cuh"
#include "ensemble.h"
#include "launch.h"
#include "mlp.cuh"
#include "../../include/method_b200.h"

namespace mth {
namespace mlp {
namespace tc {

constexpr int TM = 128;              // cells per tile: the MMA's M, one thread each
constexpr int WG = 2;                // warpgroups per CTA, one tile in flight each
constexpr int THREADS = WG * TM;
constexpr int TMEM_COLS = 64 * WG;   // FP32 accumulator columns per CTA, 64 per warpgroup
constexpr int KN = H / 16;     // 16-wide K slabs of a hidden layer

// Offset (in BF16 elements) of element (r, k) of a K-major operand of `rows`
// rows.
__host__ __device__ constexpr int kmaj(int rows, int r, int k) {
  return (k >> 4) * (rows / 8 * 128) + (r >> 3) * 128 + ((k >> 3) & 1) * 64 + (r & 7) * 8 +
         (k & 7);
}

struct Smem {
  __nv_bfloat16 w1[H * INP];     // B of layer 1: N 64 x K 16 (K 8..15 zero)
  __nv_bfloat16 w2[H * H];       // N 64 x K 64
  __nv_bfloat16 w3[H * H];
  __nv_bfloat16 w4[16 * H];      // N 16 (outputs 2..15 zero) x K 64
  __nv_bfloat16 a[WG][TM * H];   // A per warpgroup: its tile's activations, K up to 64
  float b1[H], b2[H], b3[H], b4[16];
  float stats[NSTAT];
  unsigned long long mbar[WG];
  uint32_t tmem;
  int abort;
};
static_assert(offsetof(Smem, w2) % 16 == 0 && offsetof(Smem, w3) % 16 == 0 &&
                  offsetof(Smem, w4) % 16 == 0 && offsetof(Smem, a) % 16 == 0 &&
                  (TM * H * sizeof(__nv_bfloat16)) % 16 == 0 &&
                  offsetof(Smem, mbar) % 8 == 0,
              "operands need 16-byte alignment, the mbarrier 8");

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N / 8 in
// bits 17-22, M / 16 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading byte offset 128
// and stride byte offset 256 (each >> 4), descriptor version 1 (bits 46-47),
// no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t sdesc(const void* p) {
  return (uint64_t)((smem_addr(p) >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id,
                                    uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::
                   "r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes visible to the tensor cores' reads
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait for the mbarrier phase with parity `parity`.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 20); ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Barrier and OR-reduction over the 128 threads of warpgroup `wg` (named
// barriers 1 and 2; 0 is the CTA's).
__device__ __forceinline__ void wg_sync(int wg) {
  if (wg == 0)
    asm volatile("bar.sync 1, 128;" ::: "memory");
  else
    asm volatile("bar.sync 2, 128;" ::: "memory");
}
__device__ __forceinline__ bool wg_any(int wg, bool v) {
  uint32_t r;
  if (wg == 0)
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 2, 128, q;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
  return r != 0;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(addr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void load_weights(Smem& s, const float* __restrict__ P,
                                             const float* __restrict__ st) {
  for (int i = threadIdx.x; i < H * INP; i += blockDim.x) {
    const int n = i / INP, k = i % INP;  // W1 is [in][out]
    s.w1[kmaj(H, n, k)] = __float2bfloat16(P[OFF_W1 + k * H + n]);
  }
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    const int n = i / H, k = i % H;
    s.w2[kmaj(H, n, k)] = __float2bfloat16(P[OFF_W2 + k * H + n]);
    s.w3[kmaj(H, n, k)] = __float2bfloat16(P[OFF_W3 + k * H + n]);
  }
  for (int i = threadIdx.x; i < 16 * H; i += blockDim.x) {
    const int n = i / H, k = i % H;
    s.w4[kmaj(16, n, k)] = __float2bfloat16(n < OUTP ? P[OFF_W4 + k * OUTP + n] : 0.f);
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.b1[i] = P[OFF_B1 + i];
    s.b2[i] = P[OFF_B2 + i];
    s.b3[i] = P[OFF_B3 + i];
  }
  for (int i = threadIdx.x; i < 16; i += blockDim.x) s.b4[i] = i < OUTP ? P[OFF_B4 + i] : 0.f;
  for (int i = threadIdx.x; i < NSTAT; i += blockDim.x) s.stats[i] = st ? st[i] : 0.f;
}

// Row `row` of A: 16 BF16 values (one K slab) from v[0 .. 15].
__device__ __forceinline__ void store_row16(__nv_bfloat16* a, int row, int k0, const float* v,
                                            bool relu, const float* bias) {
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float lo = v[2 * i], hi = v[2 * i + 1];
    if (bias) {
      lo += bias[2 * i];
      hi += bias[2 * i + 1];
    }
    if (relu) {
      lo = fmaxf(lo, 0.f);
      hi = fmaxf(hi, 0.f);
    }
    w[i] = pack_bf16(__float2bfloat16(lo), __float2bfloat16(hi));
  }
  *reinterpret_cast<uint4*>(a + kmaj(TM, row, k0)) = make_uint4(w[0], w[1], w[2], w[3]);
  *reinterpret_cast<uint4*>(a + kmaj(TM, row, k0 + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
}

// Warpgroup wg: its A (layer-1 input, staged by the caller) -> y[2] of this
// thread's row.  The two warpgroups of a CTA run their tiles independently
// (their own A, mbarrier and TMEM columns; the weights are shared), so one's
// products overlap the other's loads and epilogues.  Returns false when a
// wait ran out (the warpgroup then stops).
__device__ __forceinline__ bool infer_tile(Smem& s, int wg, uint32_t& phase, float* y) {
  const int row = threadIdx.x - wg * TM, warp = threadIdx.x >> 5;
  __nv_bfloat16* a = s.a[wg];
  const uint32_t bar = smem_addr(&s.mbar[wg]);
  const uint32_t d = s.tmem + (uint32_t)(wg * 64);  // column offset in the low half
  const uint32_t lane_addr = d + ((uint32_t)((warp & 3) * 32) << 16);
  bool ok = true;
#pragma unroll 1
  for (int layer = 0; layer < 4; ++layer) {
    fence_async_smem();
    fence_before();
    wg_sync(wg);
    fence_after();
    if (row == 0) {
      if (layer == 0) {
        mma(d, sdesc(a), sdesc(s.w1), idesc(TM, H), 0);
      } else {
        const __nv_bfloat16* w = layer == 1 ? s.w2 : layer == 2 ? s.w3 : s.w4;
        const int n = layer == 3 ? 16 : H;
#pragma unroll
        for (int kk = 0; kk < KN; ++kk)
          mma(d, sdesc(a + kk * (TM / 8 * 128)), sdesc(w + kk * (n / 8 * 128)), idesc(TM, n),
              kk > 0 ? 1u : 0u);
      }
      commit(bar);
    }
    ok = mbar_wait(bar, phase);
    phase ^= 1u;
    if (wg_any(wg, !ok)) return false;
    fence_after();
    if (layer < 3) {
      const float* b = layer == 0 ? s.b1 : layer == 1 ? s.b2 : s.b3;
#pragma unroll 1
      for (int c = 0; c < H / 16; ++c) {
        float v[16];
        tmem_ld16(lane_addr + c * 16, v);
        store_row16(a, row, c * 16, v, true, b + c * 16);
      }
    } else {
      float v[16];
      tmem_ld16(lane_addr, v);
      y[0] = v[0] + s.b4[0];
      y[1] = v[1] + s.b4[1];
    }
  }
  return true;
}

// Set-up shared by the kernels: weights, mbarrier, TMEM.
__device__ __forceinline__ void setup(Smem& s, const float* P, const float* st) {
  load_weights(s, P, st);
  if (threadIdx.x == 0) {
    for (int w = 0; w < WG; ++w)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s.mbar[w])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s.abort = 0;
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s.tmem)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
}

__device__ __forceinline__ void teardown(Smem& s, long long* err) {
  fence_before();
  __syncthreads();
  fence_after();
  if (threadIdx.x == 0 && s.abort && err)
    atomicOr(reinterpret_cast<unsigned long long*>(err), (unsigned long long)ERR_DEVICE);
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem),
                 "r"(TMEM_COLS));
}

// y[n][2] (standardised outputs) from standardised features x[n][8].
__global__ void __launch_bounds__(THREADS) k_forward_tc(const float* __restrict__ P, long long n,
                                                        const float* __restrict__ x,
                                                        float* __restrict__ y, long long* err) {
  extern __shared__ __align__(128) unsigned char raw[];
  Smem& s = *reinterpret_cast<Smem*>(raw);
  setup(s, P, nullptr);
  const int wg = threadIdx.x / TM, row = threadIdx.x % TM;
  uint32_t phase = 0;
  for (long long tile = (long long)blockIdx.x * WG + wg; tile * TM < n;
       tile += (long long)gridDim.x * WG) {
    const long long q = tile * TM + row;
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = (k < IN && q < n) ? x[q * IN + k] : 0.f;
    store_row16(s.a[wg], row, 0, f, false, nullptr);
    float out[2];
    if (!infer_tile(s, wg, phase, out)) {
      s.abort = 1;
      mbar_wait(smem_addr(&s.mbar[wg]), phase ^ 1u);  // the product still in flight, if it ends
      break;
    }
    if (q < n) {
      y[q * OUT] = out[0];
      y[q * OUT + 1] = out[1];
    }
  }
  teardown(s, err);
}

// Guess (Z, v^2) of every interior cell of a grid, or of the n cells of a
// variable-major batch (batch = 1), as k_mlp_zguess.
template <int MODEL>
__global__ void __launch_bounds__(THREADS) k_zguess_tc(Grid g, long long n_cells, int batch,
                                                  const double* __restrict__ cons,
                                                  const float* __restrict__ P,
                                                  const float* __restrict__ st,
                                                  double* __restrict__ zguess, long long* err) {
  extern __shared__ __align__(128) unsigned char raw[];
  Smem& s = *reinterpret_cast<Smem*>(raw);
  setup(s, P, st);
  const int wg = threadIdx.x / TM, row = threadIdx.x % TM;
  uint32_t phase = 0;
  const long long N = batch ? n_cells : g.Ntot;
  for (long long tile = (long long)blockIdx.x * WG + wg; tile * TM < n_cells;
       tile += (long long)gridDim.x * WG) {
    const long long t = tile * TM + row;
    long long cell = -1;
    if (t < n_cells) {
      if (batch) {
        cell = t;
      } else {
        int i, j, k;
        interior_ijk(g, t, i, j, k);
        cell = cell_id(g, i, j, k);
      }
    }
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.f;
    double D = 1.0;
    if (cell >= 0) {
      double c[Net<MODEL>::NC];
#pragma unroll
      for (int v = 0; v < Net<MODEL>::NC; ++v) c[v] = cons[v * N + cell];
      D = c[0];
      Net<MODEL>::features(c, f);
#pragma unroll
      for (int k = 0; k < IN; ++k) f[k] = (f[k] - s.stats[k]) * s.stats[IN + k];
    }
    store_row16(s.a[wg], row, 0, f, false, nullptr);
    float out[2];
    if (!infer_tile(s, wg, phase, out)) {
      s.abort = 1;
      mbar_wait(smem_addr(&s.mbar[wg]), phase ^ 1u);  // the product still in flight, if it ends
      break;
    }
    if (cell >= 0) {
      const float y0 = out[0] * s.stats[2 * IN + 2] + s.stats[2 * IN];
      const float y1 = out[1] * s.stats[2 * IN + 3] + s.stats[2 * IN + 1];
      zguess[cell] = D * (double)exp10f(y0);
      zguess[N + cell] = fmin(fmax((double)y1, 0.0), 0.999999);
    }
  }
  teardown(s, err);
}

// Ensembles: the guess for the cells of every member of one model into the
// members' EA_ZG planes, one 128-cell work item per tile (as k_ens_mlp_zguess).
template <int MODEL>
__global__ void __launch_bounds__(THREADS) k_ens_zguess_tc(const Member* __restrict__ mem,
                                                      const Item* __restrict__ items,
                                                      int n_items, int ic,
                                                      const float* __restrict__ P,
                                                      const float* __restrict__ st) {
  extern __shared__ __align__(128) unsigned char raw[];
  Smem& s = *reinterpret_cast<Smem*>(raw);
  setup(s, P, st);
  const int wg = threadIdx.x / TM, row = threadIdx.x % TM;
  uint32_t phase = 0;
  long long* err = nullptr;
  for (int it = blockIdx.x * WG + wg; it < n_items; it += gridDim.x * WG) {
    const Item w = items[it];
    const Member& d = mem[w.m];
    const Grid& g = d.g;
    err = d.counters + 3;
    const long long t = w.a + row;
    long long cell = -1;
    if (t < n_interior(g)) {
      int i, j, k;
      interior_ijk(g, t, i, j, k);
      cell = cell_id(g, i, j, k);
    }
    float f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = 0.f;
    double D = 1.0;
    if (cell >= 0) {
      const double* cons = d.a[ic];
      double c[Net<MODEL>::NC];
#pragma unroll
      for (int v = 0; v < Net<MODEL>::NC; ++v) c[v] = cons[v * g.Ntot + cell];
      D = c[0];
      Net<MODEL>::features(c, f);
#pragma unroll
      for (int k = 0; k < IN; ++k) f[k] = (f[k] - s.stats[k]) * s.stats[IN + k];
    }
    store_row16(s.a[wg], row, 0, f, false, nullptr);
    float out[2];
    if (!infer_tile(s, wg, phase, out)) {
      s.abort = 1;
      mbar_wait(smem_addr(&s.mbar[wg]), phase ^ 1u);  // the product still in flight, if it ends
      break;
    }
    if (cell >= 0) {
      const float y0 = out[0] * s.stats[2 * IN + 2] + s.stats[2 * IN];
      const float y1 = out[1] * s.stats[2 * IN + 3] + s.stats[2 * IN + 1];
      double* zg = d.a[EA_ZG];
      zg[cell] = D * (double)exp10f(y0);
      zg[g.Ntot + cell] = fmin(fmax((double)y1, 0.0), 0.999999);
    }
  }
  teardown(s, err);
}

int grid_for(long long rows) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms < 1) sms = 148;
  }
  // 4 CTAs per SM: 4 x 128 TMEM columns of the 512, ~54 KB shared memory each
  const long long need = (rows + WG * TM - 1) / (WG * TM);
  return (int)std::max(1LL, std::min(need, (long long)sms * 4));
}

cudaError_t configure() {
  static bool done = false;
  if (done) return cudaSuccess;
  const int b = (int)sizeof(Smem);
  cudaError_t e = cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_zguess_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_zguess_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ens_zguess_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ens_zguess_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  done = e == cudaSuccess;
  return e;
}

}  // namespace tc

cudaError_t launch_forward_tc(const float* P, long long n, const float* x, float* y, long long* err,
                              cudaStream_t st) {
  cudaError_t e = tc::configure();
  if (e != cudaSuccess) return e;
  tc::k_forward_tc<<<tc::grid_for(n), tc::THREADS, sizeof(tc::Smem), st>>>(P, n, x, y, err);
  return cudaGetLastError();
}

cudaError_t launch_zguess_tc(const Grid& g, long long n_cells, bool batch, const double* cons,
                             const float* P, const float* stats, double* zguess, long long* err,
                             cudaStream_t st, int model) {
  cudaError_t e = tc::configure();
  if (e != cudaSuccess) return e;
  if (model == 0)
    tc::k_zguess_tc<0><<<tc::grid_for(n_cells), tc::THREADS, sizeof(tc::Smem), st>>>(
        g, n_cells, batch ? 1 : 0, cons, P, stats, zguess, err);
  else
    tc::k_zguess_tc<1><<<tc::grid_for(n_cells), tc::THREADS, sizeof(tc::Smem), st>>>(
        g, n_cells, batch ? 1 : 0, cons, P, stats, zguess, err);
  return cudaGetLastError();
}

cudaError_t ens_zguess_tc(const Member* mem, const Item* items, int n_items, int ic,
                          const float* P, const float* stats, cudaStream_t st, int model) {
  cudaError_t e = tc::configure();
  if (e != cudaSuccess) return e;
  const int blocks = tc::grid_for((long long)n_items * tc::TM);
  if (model == 0)
    tc::k_ens_zguess_tc<0><<<blocks, tc::THREADS, sizeof(tc::Smem), st>>>(mem, items, n_items, ic, P,
                                                                     stats);
  else
    tc::k_ens_zguess_tc<1><<<blocks, tc::THREADS, sizeof(tc::Smem), st>>>(mem, items, n_items, ic, P,
                                                                     stats);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace mth

namespace {
struct TcBuf {
  void* p = nullptr;
  ~TcBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

extern "C" mth_status mth_mlp_forward_tc(const float* params, int n, const float* x, float* y,
                                         int device) {
  using namespace mth;
  if (!params || n <= 0 || !x || !y) return MTH_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return MTH_ERR_CUDA;
  TcBuf P, dx, dy, de;
  if (cudaMalloc(&P.p, sizeof(float) * mlp::NPARAM) != cudaSuccess ||
      cudaMalloc(&dx.p, sizeof(float) * n * mlp::IN) != cudaSuccess ||
      cudaMalloc(&dy.p, sizeof(float) * n * mlp::OUT) != cudaSuccess ||
      cudaMalloc(&de.p, sizeof(long long)) != cudaSuccess)
    return MTH_ERR_CUDA;
  if (cudaMemcpy(P.p, params, sizeof(float) * mlp::NPARAM, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(dx.p, x, sizeof(float) * n * mlp::IN, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(de.p, 0, sizeof(long long)) != cudaSuccess)
    return MTH_ERR_CUDA;
  if (mlp::launch_forward_tc((const float*)P.p, n, (const float*)dx.p, (float*)dy.p, (long long*)de.p,
                             0) != cudaSuccess)
    return MTH_ERR_CUDA;
  long long err = 0;
  if (cudaMemcpy(y, dy.p, sizeof(float) * n * mlp::OUT, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&err, de.p, sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    return MTH_ERR_CUDA;
  return err ? MTH_ERR_CUDA : MTH_OK;
}
