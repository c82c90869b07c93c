// Text output in the reference's SerialSaveData format, formatted on the GPU.
//
// SerialSaveData (serialSaveData.cc:31-246) writes every interior value with
// printf's "%.16f " and one line per (var, i, j) row.  Here the numbers are
// converted on the device: each value's decimal expansion is computed with
// exact integer arithmetic (a double is m 2^e; its 16-decimal rounding is
// (m 5^16) shifted by e + 16 with round-half-even on the bits shifted out, in
// 128-bit integers; integer parts beyond 64 bits use 32-bit limb division),
// which is what a correctly rounding printf prints.  A length pass, a scan
// and a write pass produce the file body in device memory; the host adds the
// header line and writes the bytes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace mth {
namespace text {

constexpr unsigned long long kPow5_16 = 152587890625ull;       // 5^16
constexpr unsigned long long kPow10_16 = 10000000000000000ull;  // 10^16
constexpr int kTile = 1024;                                     // values per scan tile
constexpr int kScanThreads = 128;                               // kTile / 8 values each

struct Parts {
  int kind;                 // 0 finite, 1 inf, 2 nan
  bool neg;
  bool big;                 // integer part m 2^e beyond 64 bits
  unsigned long long ip;    // integer part (when !big)
  unsigned long long frac;  // the 16 fractional digits
  unsigned long long m;     // big: mantissa
  int e;                    // big: exponent (>= 11)
};

__device__ __forceinline__ Parts decompose(double v) {
  Parts p{};
  const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
  p.neg = (bits >> 63) != 0;
  const int ex = (int)((bits >> 52) & 0x7ff);
  const unsigned long long mant = bits & ((1ull << 52) - 1);
  if (ex == 0x7ff) {
    p.kind = mant ? 2 : 1;
    return p;
  }
  p.kind = 0;
  const unsigned long long m = ex ? (mant | (1ull << 52)) : mant;
  const int e = ex ? ex - 1075 : -1074;
  if (e >= 0) {
    if (e <= 10) {
      p.ip = m << e;
    } else {
      p.big = true;
      p.m = m;
      p.e = e;
    }
    p.frac = 0;
    return p;
  }
  const int s = -e;  // value = m / 2^s
  unsigned long long fm;
  if (s < 64) {
    p.ip = m >> s;
    fm = m & ((1ull << s) - 1);
  } else {
    p.ip = 0;
    fm = m;
  }
  if (s <= 16) {
    p.frac = (fm * kPow5_16) << (16 - s);  // exact: fm < 2^s
  } else {
    const unsigned __int128 q = (unsigned __int128)fm * kPow5_16;  // < 2^91
    const int t = s - 16;
    unsigned long long r;
    if (t >= 128) {
      r = 0;  // q < 2^91 <= 2^(t-1): below one half
    } else {
      r = (unsigned long long)(q >> t);
      const unsigned __int128 rem = q & ((((unsigned __int128)1) << t) - 1);
      const unsigned __int128 half = ((unsigned __int128)1) << (t - 1);
      if (rem > half || (rem == half && (r & 1))) ++r;
    }
    p.frac = r;
  }
  if (p.frac == kPow10_16) {  // rounding carried into the integer part
    p.frac = 0;
    p.ip += 1;
  }
  return p;
}

__device__ __forceinline__ int u64_digits(unsigned long long x) {
  int n = 1;
  while (x >= 10) {
    x /= 10;
    ++n;
  }
  return n;
}

// Decimal digits of m 2^e (e >= 11) into buf (most significant first); returns
// the count.  32-bit limbs, repeated division by 10^9.
__device__ int big_digits(unsigned long long m, int e, char* buf) {
  unsigned int L[36];
  for (int q = 0; q < 36; ++q) L[q] = 0;
  const int w = e / 32, b = e % 32;  // w <= 30
  const unsigned __int128 sh = ((unsigned __int128)m) << b;
  L[w] = (unsigned int)sh;
  L[w + 1] = (unsigned int)(sh >> 32);
  L[w + 2] = (unsigned int)(sh >> 64);
  int nl = w + 3;
  while (nl > 0 && L[nl - 1] == 0) --nl;
  unsigned int chunks[40];
  int nc = 0;
  while (nl > 0) {
    unsigned long long r = 0;
    for (int q = nl - 1; q >= 0; --q) {
      const unsigned long long cur = (r << 32) | L[q];
      L[q] = (unsigned int)(cur / 1000000000ull);
      r = cur % 1000000000ull;
    }
    chunks[nc++] = (unsigned int)r;
    while (nl > 0 && L[nl - 1] == 0) --nl;
  }
  int n = 0;
  for (int c = nc - 1; c >= 0; --c) {
    unsigned int x = chunks[c];
    char tmp[9];
    int k = 0;
    do {
      tmp[k++] = (char)('0' + x % 10);
      x /= 10;
    } while (x);
    if (c != nc - 1)
      while (k < 9) tmp[k++] = '0';
    while (k > 0) buf[n++] = tmp[--k];
  }
  return n;
}

// Length of printf("%.16f", v).
__device__ int f16_len(double v) {
  const Parts p = decompose(v);
  if (p.kind) return 3 + (p.neg ? 1 : 0);
  int nd;
  if (p.big) {
    char buf[320];
    nd = big_digits(p.m, p.e, buf);
  } else {
    nd = u64_digits(p.ip);
  }
  return (p.neg ? 1 : 0) + nd + 17;
}

// printf("%.16f", v) into o; returns the length.
__device__ int f16_write(double v, char* o) {
  const Parts p = decompose(v);
  int n = 0;
  if (p.neg) o[n++] = '-';
  if (p.kind == 1) {
    o[n++] = 'i';
    o[n++] = 'n';
    o[n++] = 'f';
    return n;
  }
  if (p.kind == 2) {
    o[n++] = 'n';
    o[n++] = 'a';
    o[n++] = 'n';
    return n;
  }
  if (p.big) {
    n += big_digits(p.m, p.e, o + n);
  } else {
    char tmp[20];
    int k = 0;
    unsigned long long x = p.ip;
    do {
      tmp[k++] = (char)('0' + x % 10);
      x /= 10;
    } while (x);
    while (k > 0) o[n++] = tmp[--k];
  }
  o[n++] = '.';
  unsigned long long f = p.frac;
  for (int q = 15; q >= 0; --q) {
    o[n + q] = (char)('0' + f % 10);
    f /= 10;
  }
  return n + 16;
}

// Value t of the body (var-major, then interior i, j, k) and whether a
// newline follows it: after every value in 1D / 2D, after each k row in 3D
// (serialSaveData.cc:55-83).
__device__ __forceinline__ double body_value(const Grid& g, const double* arr, long long t,
                                             bool& eol) {
  const long long nI = n_interior(g);
  const long long v = t / nI, r = t - v * nI;
  int i, j, k;
  interior_ijk(g, r, i, j, k);
  eol = (g.dims < 3) || (k == g.ke - 1);
  return arr[v * g.Ntot + cell_id(g, i, j, k)];
}

// Per tile of kTile values: the offset of each value within its tile, and the
// tile's byte count.
__global__ void __launch_bounds__(kScanThreads)
    k_text_scan(Grid g, const double* __restrict__ arr, long long n,
                unsigned int* __restrict__ local, unsigned long long* __restrict__ tile_sum) {
  constexpr int PER = kTile / kScanThreads;
  __shared__ unsigned int warp_tot[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kTile;
  unsigned int len[PER];
  unsigned int sum = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const long long t = base + (long long)threadIdx.x * PER + q;
    unsigned int l = 0;
    if (t < n) {
      bool eol;
      const double v = body_value(g, arr, t, eol);
      l = (unsigned int)f16_len(v) + 1 + (eol ? 1 : 0);
    }
    len[q] = l;
    sum += l;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned int x = sum;  // inclusive warp scan
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  unsigned int before = 0;
  for (int w = 0; w < wid; ++w) before += warp_tot[w];
  unsigned int off = before + x - sum;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const long long t = base + (long long)threadIdx.x * PER + q;
    if (t < n) local[t] = off;
    off += len[q];
  }
  if (threadIdx.x == blockDim.x - 1) tile_sum[blockIdx.x] = off;
}

// Exclusive scan of the tile sums in place (one block of 1024 threads, the
// tiles in chunks of 1024); the grand total into *total.
__global__ void __launch_bounds__(1024)
    k_text_scan_tiles(unsigned long long* __restrict__ s, long long n_tiles,
                      unsigned long long* __restrict__ total) {
  __shared__ unsigned long long wsum[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (long long c0 = 0; c0 < n_tiles; c0 += blockDim.x) {
    const long long t = c0 + threadIdx.x;
    const unsigned long long v = t < n_tiles ? s[t] : 0;
    unsigned long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    unsigned long long before = 0;
    for (int w = 0; w < wid; ++w) before += wsum[w];
    const unsigned long long incl = before + x;
    if (t < n_tiles) s[t] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_text_write(Grid g, const double* __restrict__ arr, long long n,
                             const unsigned int* __restrict__ local,
                             const unsigned long long* __restrict__ tile_off,
                             char* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  bool eol;
  const double v = body_value(g, arr, t, eol);
  char* o = out + tile_off[t / kTile] + local[t];
  int len = f16_write(v, o);
  o[len++] = ' ';
  if (eol) o[len] = '\n';
}

}  // namespace text

cudaError_t format_body(const Grid& g, const double* arr, int nvars, std::string& out,
                        cudaStream_t st) {
  const long long n = n_interior_host(g) * nvars;
  const long long tiles = (n + text::kTile - 1) / text::kTile;
  unsigned int* local = nullptr;
  unsigned long long *tsum = nullptr, *total = nullptr;
  char* dbuf = nullptr;
  unsigned long long bytes = 0;
  cudaError_t e = cudaMalloc(&local, sizeof(unsigned int) * (size_t)std::max(n, 1LL));
  if (e == cudaSuccess)
    e = cudaMalloc(&tsum, sizeof(unsigned long long) * (size_t)std::max(tiles, 1LL));
  if (e == cudaSuccess) e = cudaMalloc(&total, sizeof(unsigned long long));
  if (e == cudaSuccess && n > 0) {
    text::k_text_scan<<<(unsigned)tiles, text::kScanThreads, 0, st>>>(g, arr, n, local, tsum);
    text::k_text_scan_tiles<<<1, 1024, 0, st>>>(tsum, tiles, total);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&bytes, total, sizeof bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (e == cudaSuccess && bytes > 0) e = cudaMalloc(&dbuf, bytes);
  if (e == cudaSuccess && n > 0) {
    text::k_text_write<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, arr, n, local, tsum,
                                                                      dbuf);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    out.resize(bytes);
    if (bytes) e = cudaMemcpyAsync(&out[0], dbuf, bytes, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(local);
  cudaFree(tsum);
  cudaFree(total);
  cudaFree(dbuf);
  return e;
}

}  // namespace mth
