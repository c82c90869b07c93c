// Guess network for primitive recovery: 8 -> 64 -> 64 -> 64 -> 2, ReLU.
//
// BF16 weights and activations, FP32 accumulation on the tensor cores
// through warp-level mma.sync m16n8k16 tiles.  One CTA of 8 warps owns 128
// samples (16 per warp); activations live in shared memory as BF16 so that
// the backward pass can read them transposed.
//
// Parameter vector (FP32 master copy, packed): W1[16][64] (input rows 8..15
// are zero padding), b1[64], W2[64][64], b2[64], W3[64][64], b3[64],
// W4[64][8] (output columns 2..7 are zero padding), b4[8].  W is stored
// [in][out], so a layer computes h_out = h_in W + b.
//
// Features of an SRMHD conserved state (all scale-free, FP32):
//   f0 = log10(tau/D)          f4 = log10(1 + tau/D)
//   f1 = log10(S^2/D^2)        f5 = |S| / (tau + D)
//   f2 = log10(B^2/D)          f6 = B^2 / (tau + D)
//   f3 = (B.S)^2 / (B^2 S^2)   f7 = log10(S^2 / (tau + D)^2)
// standardised with per-feature mean / inverse std.  Outputs: y0 =
// log10(Z / D) with Z = rho h W^2, y1 = v^2, standardised the same way.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace mth {
namespace mlp {

constexpr int IN = 8, INP = 16, H = 64, OUT = 2, OUTP = 8;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + INP * H;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H * H;
constexpr int OFF_W4 = OFF_B3 + H;
constexpr int OFF_B4 = OFF_W4 + H * OUTP;
constexpr int NPARAM = OFF_B4 + OUTP;  // 9928 packed parameters
constexpr int ROWS = 128;              // samples per CTA
constexpr int WARPS = 8;

// Normalisation: mean[8], inv_std[8] of the features, mean[2], std[2] of the targets.
constexpr int NSTAT = 20;

__device__ __forceinline__ void features_srmhd(const double* c, float* f) {
  const double D = c[0];
  const double S2 = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
  const double tau = c[4];
  const double B2 = c[5] * c[5] + c[6] * c[6] + c[7] * c[7];
  const double BS = c[5] * c[1] + c[6] * c[2] + c[7] * c[3];
  const double E = tau + D;
  // sums and ratios in FP64, logarithms in FP32 (the network's precision)
  f[0] = log10f(fmaxf((float)(tau / D), 1e-30f));
  f[1] = log10f((float)(S2 / (D * D)) + 1e-30f);
  f[2] = log10f((float)(B2 / D) + 1e-30f);
  f[3] = (float)(BS * BS / (B2 * S2 + 1e-300));
  f[4] = log10f(1.f + fmaxf((float)(tau / D), 0.f));
  f[5] = (float)(sqrt(S2) / E);
  f[6] = (float)(B2 / E);
  f[7] = log10f((float)(S2 / (E * E)) + 1e-30f);
}

// Features of an SRRMHD conserved state (D, S, tau, B, E, psi, phi, q): its
// primitive recovery depends on S-bar = S - E x B and tau-bar = tau -
// (B^2 + E^2)/2 only (srrmhd.cc:256-301), so the map uses those:
//   f0 = log10(tau-bar/D)        f4 = log10(S-bar^2 / (tau-bar + D)^2)
//   f1 = log10(S-bar^2/D^2)      f5 = S-bar^2 / (tau-bar + D)^2
//   f2 = log10(1 + tau-bar/D)    f6 = D / (tau-bar + D)
//   f3 = |S-bar| / (tau-bar + D) f7 = 0
// Outputs as for SRMHD: log10(Z/D) with Z = rho h W^2, and v^2.
__device__ __forceinline__ void features_srrmhd(const double* c, float* f) {
  const double D = c[0];
  const double sx = c[1] - (c[9] * c[7] - c[10] * c[6]);
  const double sy = c[2] - (c[10] * c[5] - c[8] * c[7]);
  const double sz = c[3] - (c[8] * c[6] - c[9] * c[5]);
  const double S2 = sx * sx + sy * sy + sz * sz;
  const double tb = c[4] - 0.5 * (c[5] * c[5] + c[6] * c[6] + c[7] * c[7] + c[8] * c[8] +
                                  c[9] * c[9] + c[10] * c[10]);
  const double E = tb + D;
  f[0] = log10f(fmaxf((float)(tb / D), 1e-30f));
  f[1] = log10f((float)(S2 / (D * D)) + 1e-30f);
  f[2] = log10f(1.f + fmaxf((float)(tb / D), 0.f));
  f[3] = (float)(sqrt(S2) / E);
  f[4] = log10f((float)(S2 / (E * E)) + 1e-30f);
  f[5] = (float)(S2 / (E * E));
  f[6] = (float)(D / E);
  f[7] = 0.f;
}

// Conserved variables per model and the feature map of a model.
template <int MODEL>
struct Net;
template <>
struct Net<0> {
  static constexpr int NC = 9;
  __device__ __forceinline__ static void features(const double* c, float* f) {
    features_srmhd(c, f);
  }
};
template <>
struct Net<1> {
  static constexpr int NC = 14;
  __device__ __forceinline__ static void features(const double* c, float* f) {
    features_srrmhd(c, f);
  }
};

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  uint32_t l = (uint32_t)__bfloat16_as_ushort(lo), h = (uint32_t)__bfloat16_as_ushort(hi);
  return l | (h << 16);
}

// D = A (16x16, bf16, row) * B (16x8, bf16, col) + C, FP32.
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One 16x8 output tile: C += sum_k A(r, k) B(k, n) for K a multiple of 16.
// a_at(r, k) / b_at(k, n) return bf16 operands from shared memory; the
// fragment ownership follows the m16n8k16 layout (PTX ISA, mma.m16n8k16):
// g = lane / 4 owns rows g and g + 8, t = lane % 4 owns columns 2t, 2t+1
// (+8).
template <int K, class FA, class FB>
__device__ __forceinline__ void tile_mma(float* c, FA a_at, FB b_at) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t a[4], b[2];
    a[0] = pack_bf16(a_at(g, k0 + 2 * t), a_at(g, k0 + 2 * t + 1));
    a[1] = pack_bf16(a_at(g + 8, k0 + 2 * t), a_at(g + 8, k0 + 2 * t + 1));
    a[2] = pack_bf16(a_at(g, k0 + 2 * t + 8), a_at(g, k0 + 2 * t + 9));
    a[3] = pack_bf16(a_at(g + 8, k0 + 2 * t + 8), a_at(g + 8, k0 + 2 * t + 9));
    b[0] = pack_bf16(b_at(k0 + 2 * t, g), b_at(k0 + 2 * t + 1, g));
    b[1] = pack_bf16(b_at(k0 + 2 * t + 8, g), b_at(k0 + 2 * t + 9, g));
    mma_bf16(c, a, b);
  }
}

}  // namespace mlp
}  // namespace mth
