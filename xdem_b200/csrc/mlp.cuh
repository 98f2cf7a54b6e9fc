// mlp.cuh — the learned warm start of the closest-approach Newton iteration.
//
// A multilayer perceptron maps an ellipse pair's relative pose and semi-axes,
//   x = [dx/b_i, dy/b_i (centre offset in ellipse i's frame), cos Δθ, sin Δθ,
//        a_i/b_i, a_j/b_i, b_j/b_i]   (Δθ = θ_j - θ_i),
// through three hidden layers of width 64 with SiLU to two outputs:
//   y0  the root of the reference's quartic (EllipticParticle.cpp:92-100,163)
//       as a fraction of Newton's analytic start sqrt(δ + 1),
//   y1  a contact logit.
// Weights are BF16 and every product accumulates in FP32 on the tensor cores.
// Inference (the world's warm start and xdem_mlp_forward) runs tcgen05 MMAs
// with the accumulator in tensor memory, 128 rows per CTA (mlp_tc.cuh).  The
// training kernels (learn.cu) keep a warp-level form built from the helpers
// below (mma.sync m16n8k16): a warp evaluates 16 samples at a time, and a
// layer's accumulator fragments (rows = samples, columns = units) are exactly
// the A-operand fragments of the next layer, so the backward pass finds every
// activation it needs in registers.
//
// Parameters live in one FP32 vector (the training master copy) with the
// layout of MlpLayout; BF16 copies of the weight matrices, row-major
// [out][in] and transposed for the backward pass, are made from it after
// every update.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace xdem {

constexpr int kMlpIn = 7;
constexpr int kMlpK1 = 16;  // input width padded to one k-step
constexpr int kMlpH = 64;
constexpr int kMlpOut = 2;
constexpr int kMlpOutPad = 8;  // output width padded to one n-tile

// FP32 parameter vector: W1 [64][16], b1[64], W2 [64][64], b2[64],
// W3 [64][64], b3[64], W4 [8][64] (rows 2..7 zero), b4[8]
struct MlpLayout {
  static constexpr int W1 = 0;
  static constexpr int B1 = W1 + kMlpH * kMlpK1;
  static constexpr int W2 = B1 + kMlpH;
  static constexpr int B2 = W2 + kMlpH * kMlpH;
  static constexpr int W3 = B2 + kMlpH;
  static constexpr int B3 = W3 + kMlpH * kMlpH;
  static constexpr int W4 = B3 + kMlpH;
  static constexpr int B4 = W4 + kMlpOutPad * kMlpH;
  static constexpr int COUNT = B4 + kMlpOutPad;
};

// BF16 weight copies: W1, W2, W3, W4 as [out][in], then W2ᵀ, W3ᵀ as [in][out]
struct MlpBf16Layout {
  static constexpr int W1 = 0;
  static constexpr int W2 = W1 + kMlpH * kMlpK1;
  static constexpr int W3 = W2 + kMlpH * kMlpH;
  static constexpr int W4 = W3 + kMlpH * kMlpH;
  static constexpr int W2T = W4 + kMlpOutPad * kMlpH;
  static constexpr int W3T = W2T + kMlpH * kMlpH;
  static constexpr int COUNT = W3T + kMlpH * kMlpH;
};

// what a kernel needs to evaluate the network
struct MlpDev {
  const __nv_bfloat16* wb;  // MlpBf16Layout
  const float* theta;       // MlpLayout (biases read from here)
  float scale[kMlpIn];      // input scaling (x_k * scale_k)
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// D += A (16x16, row) * B (16x8, col); BF16 inputs, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// B fragment of n-tile j, k-step s from a row-major [n][kdim] BF16 matrix:
// (k = 16s + 2t, +1) and (k = 16s + 2t + 8, +9) of row n = 8j + g
__device__ __forceinline__ void load_b(const __nv_bfloat16* W, int kdim, int j, int s, int g, int t,
                                       uint32_t& b0, uint32_t& b1) {
  const __nv_bfloat16* row = W + (size_t)(8 * j + g) * kdim + 16 * s + 2 * t;
  b0 = *reinterpret_cast<const uint32_t*>(row);
  b1 = *reinterpret_cast<const uint32_t*>(row + 8);
}

// One hidden layer of 64 units: acc (8 n-tiles) = bias + A (4 k-steps) * Wᵀ.
__device__ __forceinline__ void mlp_hidden(const __nv_bfloat16* W, const float* bias,
                                           const uint32_t (&A)[4][4], int g, int t,
                                           float (&acc)[8][4]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float b0 = bias[8 * j + 2 * t], b1 = bias[8 * j + 2 * t + 1];
    acc[j][0] = b0;
    acc[j][1] = b1;
    acc[j][2] = b0;
    acc[j][3] = b1;
  }
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t b0, b1;
      load_b(W, kMlpH, j, s, g, t, b0, b1);
      mma_bf16(acc[j], A[s], b0, b1);
    }
}

// SiLU of accumulator fragments, repacked as the next layer's A fragments:
// k-step s takes n-tiles 2s (columns 16s..16s+7) and 2s+1 (16s+8..16s+15)
__device__ __forceinline__ void act_to_a(const float (&acc)[8][4], uint32_t (&A)[4][4]) {
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    A[s][0] = pack_bf16(silu(acc[2 * s][0]), silu(acc[2 * s][1]));
    A[s][1] = pack_bf16(silu(acc[2 * s][2]), silu(acc[2 * s][3]));
    A[s][2] = pack_bf16(silu(acc[2 * s + 1][0]), silu(acc[2 * s + 1][1]));
    A[s][3] = pack_bf16(silu(acc[2 * s + 1][2]), silu(acc[2 * s + 1][3]));
  }
}

// The features of a closest-approach pair (see the file comment), FP32,
// scaled.  d = p_j + offset - p_i; (c1, s1), (c2, s2): cos/sin of θ_i, θ_j.
__device__ __forceinline__ void mlp_features(const MlpDev& net, double dx, double dy, double c1,
                                             double s1, double c2, double s2, double a_i,
                                             double asp_i, double a_j, double asp_j, float* f) {
  const double b_i = a_i / asp_i;
  f[0] = (float)((c1 * dx + s1 * dy) / b_i);
  f[1] = (float)((-s1 * dx + c1 * dy) / b_i);
  f[2] = (float)(c1 * c2 + s1 * s2);
  f[3] = (float)(c1 * s2 - s1 * c2);
  f[4] = (float)asp_i;
  f[5] = (float)(a_j / b_i);
  f[6] = (float)((a_j / asp_j) / b_i);
#pragma unroll
  for (int k = 0; k < kMlpIn; ++k) f[k] *= net.scale[k];
}

}  // namespace xdem
