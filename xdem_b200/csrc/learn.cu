// learn.cu — training and evaluation of the warm-start network (mlp.cuh) on
// the GPU: forward and backward passes on the tensor cores (mma.sync BF16,
// FP32 accumulate), deterministic gradient reduction, Adam.  C-ABI: the
// xdem_mlp_* entry points of include/xdem_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "../../include/xdem_gpu.h"
#include "mlp_host.h"
#include "mlp_tc.cuh"

using namespace xdem;

namespace {

constexpr int kTrainWarps = 4;
constexpr int kTrainRows = 16 * kTrainWarps;  // samples per block
constexpr float kLogitWeight = 0.1f;          // weight of the contact term in the loss

// ---- parameter copies ------------------------------------------------------------
__global__ void k_mlp_publish(const float* theta, __nv_bfloat16* wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kMlpH * kMlpK1) wb[MlpBf16Layout::W1 + i] = __float2bfloat16_rn(theta[MlpLayout::W1 + i]);
  if (i < kMlpH * kMlpH) {
    const int n = i / kMlpH, k = i % kMlpH;
    const float w2 = theta[MlpLayout::W2 + i], w3 = theta[MlpLayout::W3 + i];
    wb[MlpBf16Layout::W2 + i] = __float2bfloat16_rn(w2);
    wb[MlpBf16Layout::W3 + i] = __float2bfloat16_rn(w3);
    wb[MlpBf16Layout::W2T + k * kMlpH + n] = __float2bfloat16_rn(w2);
    wb[MlpBf16Layout::W3T + k * kMlpH + n] = __float2bfloat16_rn(w3);
  }
  if (i < kMlpOutPad * kMlpH) wb[MlpBf16Layout::W4 + i] = __float2bfloat16_rn(theta[MlpLayout::W4 + i]);
}

// ---- evaluation ---------------------------------------------------------------------
// rows of x through the network on the tensor cores (mlp_tc.cuh), 128 per
// tile; *failed = 1 when a completion barrier timed out
__global__ void __launch_bounds__(128) k_mlp_forward(MlpDev net, int64_t n, const float* x,
                                                     float* y, int32_t* failed) {
  __shared__ MlpTcSmem s;
  mlp_tc_setup(s, net);
  uint32_t phase = 0;
  const int64_t tiles = (n + kTcRows - 1) / kTcRows;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row = tile * kTcRows + threadIdx.x;
    float f[kMlpIn];
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c) f[c] = row < n ? x[row * kMlpIn + c] * net.scale[c] : 0.0f;
    float o0, o1;
    if (!mlp_tc_tile(s, f, phase, o0, o1)) {
      if (threadIdx.x == 0) *failed = 1;
      break;
    }
    if (row < n) {
      y[row * 2] = o0;
      y[row * 2 + 1] = o1;
    }
  }
  mlp_tc_teardown(s);
}

// a completion barrier that nothing arrives on: the bounded wait gives up
__global__ void k_selftest_wait(int32_t* timed_out) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0);
  if (threadIdx.x == 0) *timed_out = ok ? 0 : 1;
}

// ---- training ----------------------------------------------------------------------------
// shared memory of one training block (4 warps x 16 samples)
struct TrainSmem {
  float x[kTrainRows][16];           // scaled inputs (FP32)
  __nv_bfloat16 xb[kTrainRows][16];  // as the MMA saw them
  float z[3][kTrainRows][kMlpH];     // pre-activations of layers 1-3
  __nv_bfloat16 h[3][kTrainRows][kMlpH];  // activations of layers 1-3 (BF16, MMA inputs)
  __nv_bfloat16 dz[3][kTrainRows][kMlpH];  // dL/dz of layers 1-3 (BF16, MMA inputs)
  float dy[kTrainRows][2];           // dL/dy
  float loss[kTrainRows];
};

__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// A fragment (rows r0..r0+15 of a [rows][64] BF16 matrix, k-step s)
__device__ __forceinline__ void load_a_rows(const __nv_bfloat16 (*M)[kMlpH], int r0, int s, int g,
                                            int t, uint32_t (&a)[4]) {
  const int c = 16 * s + 2 * t;
  a[0] = pack2(M[r0 + g][c], M[r0 + g][c + 1]);
  a[1] = pack2(M[r0 + g + 8][c], M[r0 + g + 8][c + 1]);
  a[2] = pack2(M[r0 + g][c + 8], M[r0 + g][c + 9]);
  a[3] = pack2(M[r0 + g + 8][c + 8], M[r0 + g + 8][c + 9]);
}

// Weight gradient of one layer for the block: rows n = 16*warp .. +15 of
// dW[n][k] = sum over the 64 samples of dZ[m][n] * H[m][k], kdim columns of H
// (ntiles = kdim / 8); A'(n, m) = dZ[m][n], B'(m, k) = H[m][k].
template <int NT, class HT>
__device__ __forceinline__ void weight_grad(const __nv_bfloat16 (*dZ)[kMlpH], const HT* H, int hstride,
                                            int warp, int g, int t, float* out, int kdim) {
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
  const int n0 = 16 * warp;
#pragma unroll
  for (int s = 0; s < 4; ++s) {  // samples 16s .. 16s+15
    const int m0 = 16 * s + 2 * t;
    uint32_t a[4];
    a[0] = pack2(dZ[m0][n0 + g], dZ[m0 + 1][n0 + g]);
    a[1] = pack2(dZ[m0][n0 + g + 8], dZ[m0 + 1][n0 + g + 8]);
    a[2] = pack2(dZ[m0 + 8][n0 + g], dZ[m0 + 9][n0 + g]);
    a[3] = pack2(dZ[m0 + 8][n0 + g + 8], dZ[m0 + 9][n0 + g + 8]);
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int k = 8 * j + g;
      const uint32_t b0 = pack2(H[(size_t)m0 * hstride + k], H[(size_t)(m0 + 1) * hstride + k]);
      const uint32_t b1 = pack2(H[(size_t)(m0 + 8) * hstride + k], H[(size_t)(m0 + 9) * hstride + k]);
      mma_bf16(acc[j], a, b0, b1);
    }
  }
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int k = 8 * j + 2 * t;
    out[(n0 + g) * kdim + k] = acc[j][0];
    out[(n0 + g) * kdim + k + 1] = acc[j][1];
    out[(n0 + g + 8) * kdim + k] = acc[j][2];
    out[(n0 + g + 8) * kdim + k + 1] = acc[j][3];
  }
}

// Forward and backward pass of 64 samples perm[first + 64*block ..] (rows past
// `count` are masked); writes the block's gradient (MlpLayout) and loss sum.
// Loss per sample: valid * (y0 - target)^2 + 0.1 * BCE(y1, contact), averaged
// over `count`; valid = the target is finite (the Newton root exists).
__global__ void __launch_bounds__(128) k_mlp_train(MlpDev net, const float* x, const float* target,
                                                   const float* contact, const int32_t* perm,
                                                   int64_t first, int64_t count, float* gpart,
                                                   float* lpart) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = 16 * warp;
  const float inv_count = 1.0f / (float)count;
  // inputs
  for (int e = threadIdx.x; e < kTrainRows * 16; e += blockDim.x) {
    const int r = e >> 4, c = e & 15;
    const int64_t pos = (int64_t)blockIdx.x * kTrainRows + r;
    float v = 0.0f;
    if (c < kMlpIn && pos < count) v = x[(int64_t)perm[first + pos] * kMlpIn + c] * net.scale[c];
    S.x[r][c] = v;
    S.xb[r][c] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  const float* th = net.theta;
  const __nv_bfloat16* wb = net.wb;
  // ---- forward, keeping z and h ----
  float acc[8][4];
  uint32_t A[4][4];
  {
    uint32_t a1[4];
    const int c = 2 * t;
    a1[0] = pack2(S.xb[r0 + g][c], S.xb[r0 + g][c + 1]);
    a1[1] = pack2(S.xb[r0 + g + 8][c], S.xb[r0 + g + 8][c + 1]);
    a1[2] = pack2(S.xb[r0 + g][c + 8], S.xb[r0 + g][c + 9]);
    a1[3] = pack2(S.xb[r0 + g + 8][c + 8], S.xb[r0 + g + 8][c + 9]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float b0 = th[MlpLayout::B1 + 8 * j + 2 * t], b1 = th[MlpLayout::B1 + 8 * j + 2 * t + 1];
      acc[j][0] = b0;
      acc[j][1] = b1;
      acc[j][2] = b0;
      acc[j][3] = b1;
      uint32_t w0, w1;
      load_b(wb + MlpBf16Layout::W1, kMlpK1, j, 0, g, t, w0, w1);
      mma_bf16(acc[j], a1, w0, w1);
    }
  }
  for (int L = 0; L < 3; ++L) {
    // store z and h of layer L+1, then form the next A operand
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      S.z[L][r0 + g][c] = acc[j][0];
      S.z[L][r0 + g][c + 1] = acc[j][1];
      S.z[L][r0 + g + 8][c] = acc[j][2];
      S.z[L][r0 + g + 8][c + 1] = acc[j][3];
    }
    act_to_a(acc, A);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      // A[s] regs: (row g, cols 16s+2t..), (row g+8, ..), (row g, +8), (row g+8, +8)
      const int c = 16 * s + 2 * t;
      *reinterpret_cast<uint32_t*>(&S.h[L][r0 + g][c]) = A[s][0];
      *reinterpret_cast<uint32_t*>(&S.h[L][r0 + g + 8][c]) = A[s][1];
      *reinterpret_cast<uint32_t*>(&S.h[L][r0 + g][c + 8]) = A[s][2];
      *reinterpret_cast<uint32_t*>(&S.h[L][r0 + g + 8][c + 8]) = A[s][3];
    }
    if (L < 2) {
      const __nv_bfloat16* W = wb + (L == 0 ? MlpBf16Layout::W2 : MlpBf16Layout::W3);
      mlp_hidden(W, th + (L == 0 ? MlpLayout::B2 : MlpLayout::B3), A, g, t, acc);
    }
  }
  // output layer
  float o[4];
  o[0] = th[MlpLayout::B4 + 2 * t];
  o[1] = th[MlpLayout::B4 + 2 * t + 1];
  o[2] = o[0];
  o[3] = o[1];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    uint32_t w0, w1;
    load_b(wb + MlpBf16Layout::W4, kMlpH, 0, s, g, t, w0, w1);
    mma_bf16(o, A[s], w0, w1);
  }
  if (t == 0) {
    for (int half = 0; half < 2; ++half) {
      const int r = r0 + g + 8 * half;
      const float y0 = o[2 * half], y1 = o[2 * half + 1];
      const int64_t pos = (int64_t)blockIdx.x * kTrainRows + r;
      float d0 = 0.0f, d1 = 0.0f, l = 0.0f;
      if (pos < count) {
        const int64_t src = perm[first + pos];
        const float tg = target[src], ct = contact[src];
        if (isfinite(tg)) {
          d0 = 2.0f * (y0 - tg) * inv_count;
          l += (y0 - tg) * (y0 - tg);
        }
        const float sg = 1.0f / (1.0f + __expf(-y1));
        d1 = kLogitWeight * (sg - ct) * inv_count;
        // BCE with logits: softplus(y1) - ct * y1
        const float sp = y1 > 0.0f ? y1 + log1pf(__expf(-y1)) : log1pf(__expf(y1));
        l += kLogitWeight * (sp - ct * y1);
      }
      S.dy[r][0] = d0;
      S.dy[r][1] = d1;
      S.loss[r] = l;
    }
  }
  __syncwarp();
  // ---- backward through the warp's rows ----
  // dH3 = dY W4 (two outputs, CUDA cores), dZ3 = dH3 * silu'(z3)
  for (int e = lane; e < 16 * kMlpH; e += 32) {
    const int r = r0 + e / kMlpH, k = e % kMlpH;
    const float w40 = __bfloat162float(wb[MlpBf16Layout::W4 + k]);
    const float w41 = __bfloat162float(wb[MlpBf16Layout::W4 + kMlpH + k]);
    const float dh = S.dy[r][0] * w40 + S.dy[r][1] * w41;
    S.dz[2][r][k] = __float2bfloat16_rn(dh * dsilu(S.z[2][r][k]));
  }
  __syncwarp();
  // dH(L) = dZ(L+1) W(L+1) via the transposed copies, then dZ(L) = dH * silu'(z)
  for (int L = 1; L >= 0; --L) {
    const __nv_bfloat16* WT = wb + (L == 1 ? MlpBf16Layout::W3T : MlpBf16Layout::W2T);
    uint32_t a[4][4];
#pragma unroll
    for (int s = 0; s < 4; ++s) load_a_rows(S.dz[L + 1], r0, s, g, t, a[s]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        uint32_t w0, w1;
        load_b(WT, kMlpH, j, s, g, t, w0, w1);
        mma_bf16(acc[j], a[s], w0, w1);
      }
      const int c = 8 * j + 2 * t;
      S.dz[L][r0 + g][c] = __float2bfloat16_rn(acc[j][0] * dsilu(S.z[L][r0 + g][c]));
      S.dz[L][r0 + g][c + 1] = __float2bfloat16_rn(acc[j][1] * dsilu(S.z[L][r0 + g][c + 1]));
      S.dz[L][r0 + g + 8][c] = __float2bfloat16_rn(acc[j][2] * dsilu(S.z[L][r0 + g + 8][c]));
      S.dz[L][r0 + g + 8][c + 1] = __float2bfloat16_rn(acc[j][3] * dsilu(S.z[L][r0 + g + 8][c + 1]));
    }
    __syncwarp();
  }
  __syncthreads();
  // ---- weight gradients of the block (64 samples) ----
  float* G = gpart + (size_t)blockIdx.x * MlpLayout::COUNT;
  weight_grad<2>(S.dz[0], &S.xb[0][0], 16, warp, g, t, G + MlpLayout::W1, kMlpK1);
  weight_grad<8>(S.dz[1], &S.h[0][0][0], kMlpH, warp, g, t, G + MlpLayout::W2, kMlpH);
  weight_grad<8>(S.dz[2], &S.h[1][0][0], kMlpH, warp, g, t, G + MlpLayout::W3, kMlpH);
  // output layer and biases on the CUDA cores, fixed summation order
  for (int e = threadIdx.x; e < kMlpOutPad * kMlpH; e += blockDim.x) {
    const int n = e / kMlpH, k = e % kMlpH;
    float s = 0.0f;
    if (n < kMlpOut)
      for (int m = 0; m < kTrainRows; ++m) s += S.dy[m][n] * __bfloat162float(S.h[2][m][k]);
    G[MlpLayout::W4 + e] = s;
  }
  for (int e = threadIdx.x; e < 3 * kMlpH + kMlpOutPad; e += blockDim.x) {
    float s = 0.0f;
    if (e < 3 * kMlpH) {
      const int L = e / kMlpH, n = e % kMlpH;
      for (int m = 0; m < kTrainRows; ++m) s += __bfloat162float(S.dz[L][m][n]);
      const int off = L == 0 ? MlpLayout::B1 : (L == 1 ? MlpLayout::B2 : MlpLayout::B3);
      G[off + n] = s;
    } else {
      const int n = e - 3 * kMlpH;
      if (n < kMlpOut)
        for (int m = 0; m < kTrainRows; ++m) s += S.dy[m][n];
      G[MlpLayout::B4 + n] = s;
    }
  }
  if (threadIdx.x == 0) {
    float l = 0.0f;
    for (int m = 0; m < kTrainRows; ++m) l += S.loss[m];
    lpart[blockIdx.x] = l;
  }
}

// sums the blocks' partial gradients in block order (deterministic)
__global__ void k_mlp_reduce(const float* gpart, int nblocks, float* grad, const float* lpart,
                             float* loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < MlpLayout::COUNT) {
    float s = 0.0f;
    for (int b = 0; b < nblocks; ++b) s += gpart[(size_t)b * MlpLayout::COUNT + p];
    grad[p] = s;
  }
  if (p == 0 && loss) {
    float s = 0.0f;
    for (int b = 0; b < nblocks; ++b) s += lpart[b];
    *loss = s;
  }
}

// Adam (Kingma and Ba 2015) on the FP32 master parameters; the padding
// entries (inputs 7..15 of W1, outputs 2..7 of W4) stay zero
__global__ void k_mlp_adam(float* theta, float* m, float* v, const float* grad, float lr, float b1,
                           float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MlpLayout::COUNT) return;
  if (p < MlpLayout::B1 && (p % kMlpK1) >= kMlpIn) return;
  if (p >= MlpLayout::W4 && p < MlpLayout::B4 && (p - MlpLayout::W4) / kMlpH >= kMlpOut) return;
  if (p >= MlpLayout::B4 + kMlpOut) return;
  const float gr = grad[p];
  const float mm = b1 * m[p] + (1.0f - b1) * gr;
  const float vv = b2 * v[p] + (1.0f - b2) * gr * gr;
  m[p] = mm;
  v[p] = vv;
  theta[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

}  // namespace

cudaError_t mlp_reserve(xdem_mlp_s* m, int64_t need) {
  if (need <= m->cap) return cudaSuccess;
  int64_t cap = std::max<int64_t>(need, 2 * m->cap);
  float *x = nullptr, *t = nullptr, *c = nullptr;
  cudaError_t e = cudaMalloc(&x, sizeof(float) * kMlpIn * cap);
  if (e == cudaSuccess) e = cudaMalloc(&t, sizeof(float) * cap);
  if (e == cudaSuccess) e = cudaMalloc(&c, sizeof(float) * cap);
  if (e == cudaSuccess && m->size > 0) {
    e = cudaMemcpyAsync(x, m->x, sizeof(float) * kMlpIn * m->size, cudaMemcpyDeviceToDevice, m->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(t, m->target, sizeof(float) * m->size, cudaMemcpyDeviceToDevice, m->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c, m->contact, sizeof(float) * m->size, cudaMemcpyDeviceToDevice, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  }
  if (e != cudaSuccess) {
    cudaFree(x);
    cudaFree(t);
    cudaFree(c);
    return e;
  }
  cudaFree(m->x);
  cudaFree(m->target);
  cudaFree(m->contact);
  m->x = x;
  m->target = t;
  m->contact = c;
  m->cap = cap;
  return cudaSuccess;
}

namespace {

cudaError_t publish(xdem_mlp_s* m) {
  k_mlp_publish<<<(kMlpH * kMlpH + 127) / 128, 128, 0, m->stream>>>(m->theta, m->wb);
  return cudaGetLastError();
}

cudaError_t ensure_gpart(xdem_mlp_s* m, int blocks) {
  if (blocks <= m->gpart_blocks) return cudaSuccess;
  cudaFree(m->gpart);
  cudaFree(m->lpart);
  m->gpart = nullptr;
  m->lpart = nullptr;
  cudaError_t e = cudaMalloc(&m->gpart, sizeof(float) * MlpLayout::COUNT * (size_t)blocks);
  if (e == cudaSuccess) e = cudaMalloc(&m->lpart, sizeof(float) * (size_t)blocks);
  if (e == cudaSuccess) m->gpart_blocks = blocks;
  return e;
}

// one forward/backward over perm[first, first + count) into m->grad; loss
// (device, may be NULL) receives the summed loss
cudaError_t gradient(xdem_mlp_s* m, const float* x, const float* tg, const float* ct,
                     const int32_t* perm, int64_t first, int64_t count, float* loss) {
  const int blocks = (int)((count + kTrainRows - 1) / kTrainRows);
  cudaError_t e = ensure_gpart(m, blocks);
  if (e != cudaSuccess) return e;
  const size_t smem = sizeof(TrainSmem);
  e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_mlp_train<<<blocks, 128, smem, m->stream>>>(m->dev(), x, tg, ct, perm, first, count, m->gpart,
                                                 m->lpart);
  k_mlp_reduce<<<(MlpLayout::COUNT + 255) / 256, 256, 0, m->stream>>>(m->gpart, blocks, m->grad,
                                                                        m->lpart, loss);
  return cudaGetLastError();
}

}  // namespace

extern "C" {

int32_t xdem_mlp_param_count(void) { return MlpLayout::COUNT; }

int32_t xdem_mlp_create(uint64_t seed, xdem_mlp* out) {
  if (!out) return XDEM_ERR_ARGUMENT;
  *out = nullptr;
  xdem_mlp_s* m = new (std::nothrow) xdem_mlp_s();
  if (!m) return XDEM_ERR_ARGUMENT;
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->theta, sizeof(float) * MlpLayout::COUNT);
  if (e == cudaSuccess) e = cudaMalloc(&m->adam_m, sizeof(float) * MlpLayout::COUNT);
  if (e == cudaSuccess) e = cudaMalloc(&m->adam_v, sizeof(float) * MlpLayout::COUNT);
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, sizeof(float) * MlpLayout::COUNT);
  if (e == cudaSuccess) e = cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * MlpBf16Layout::COUNT);
  if (e != cudaSuccess) {
    xdem_mlp_destroy(m);
    return XDEM_ERR_CUDA;
  }
  // He-uniform initial weights (seeded), zero biases and padding
  std::vector<float> th(MlpLayout::COUNT, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols, int fan_in) {
    const float lim = std::sqrt(6.0f / (float)fan_in);
    std::uniform_real_distribution<float> u(-lim, lim);
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) th[off + r * cols + c] = (r < used_rows && c < used_cols) ? u(rng) : 0.0f;
  };
  fill(MlpLayout::W1, kMlpH, kMlpK1, kMlpH, kMlpIn, kMlpIn);
  fill(MlpLayout::W2, kMlpH, kMlpH, kMlpH, kMlpH, kMlpH);
  fill(MlpLayout::W3, kMlpH, kMlpH, kMlpH, kMlpH, kMlpH);
  fill(MlpLayout::W4, kMlpOutPad, kMlpH, kMlpOut, kMlpH, kMlpH);
  e = cudaMemcpyAsync(m->theta, th.data(), sizeof(float) * MlpLayout::COUNT, cudaMemcpyHostToDevice,
                      m->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->adam_m, 0, sizeof(float) * MlpLayout::COUNT, m->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->adam_v, 0, sizeof(float) * MlpLayout::COUNT, m->stream);
  if (e == cudaSuccess) e = publish(m);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) {
    xdem_mlp_destroy(m);
    return XDEM_ERR_CUDA;
  }
  *out = m;
  return XDEM_OK;
}

int32_t xdem_mlp_destroy(xdem_mlp m) {
  if (!m) return XDEM_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->theta);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->grad);
  cudaFree(m->wb);
  cudaFree(m->gpart);
  cudaFree(m->lpart);
  cudaFree(m->x);
  cudaFree(m->target);
  cudaFree(m->contact);
  cudaFree(m->perm);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return XDEM_OK;
}

int32_t xdem_mlp_get_params(xdem_mlp m, float* theta, float* scale) {
  if (!m) return XDEM_ERR_ARGUMENT;
  if (theta) {
    if (cudaMemcpyAsync(theta, m->theta, sizeof(float) * MlpLayout::COUNT, cudaMemcpyDeviceToHost,
                        m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess)
      return XDEM_ERR_CUDA;
  }
  if (scale) std::memcpy(scale, m->scale, sizeof(float) * kMlpIn);
  return XDEM_OK;
}

int32_t xdem_mlp_set_params(xdem_mlp m, const float* theta, const float* scale) {
  if (!m) return XDEM_ERR_ARGUMENT;
  if (scale) std::memcpy(m->scale, scale, sizeof(float) * kMlpIn);
  if (theta) {
    if (cudaMemcpyAsync(m->theta, theta, sizeof(float) * MlpLayout::COUNT, cudaMemcpyHostToDevice,
                        m->stream) != cudaSuccess ||
        publish(m) != cudaSuccess || cudaStreamSynchronize(m->stream) != cudaSuccess)
      return XDEM_ERR_CUDA;
  }
  return XDEM_OK;
}

int32_t xdem_mlp_forward(xdem_mlp m, int64_t n, const float* x, float* y) {
  if (!m || n <= 0 || !x || !y) return XDEM_ERR_ARGUMENT;
  float *dx = nullptr, *dy = nullptr;
  int32_t* dfail = nullptr;
  int32_t failed = 0;
  cudaError_t e = cudaMalloc(&dx, sizeof(float) * kMlpIn * n);
  if (e == cudaSuccess) e = cudaMalloc(&dy, sizeof(float) * 2 * n);
  if (e == cudaSuccess) e = cudaMalloc(&dfail, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(dfail, 0, sizeof(int32_t), m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dx, x, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) {
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const int blocks = (int)std::min<int64_t>(tiles, 148 * 4);
    k_mlp_forward<<<blocks, 128, 0, m->stream>>>(m->dev(), n, dx, dy, dfail);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&failed, dfail, sizeof(int32_t), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dfail);
  if (e != cudaSuccess) return XDEM_ERR_CUDA;
  return failed ? XDEM_ERR_TIMEOUT : XDEM_OK;
}

int32_t xdem_selftest_bounded_wait(double* ms) {
  int32_t* d = nullptr;
  int32_t h = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t e = cudaMalloc(&d, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaEventCreate(&ev[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
  if (e == cudaSuccess) e = cudaEventRecord(ev[0]);
  if (e == cudaSuccess) {
    k_selftest_wait<<<1, 32>>>(d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev[1]);
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int32_t), cudaMemcpyDeviceToHost);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev[0], ev[1]);
  if (ms) *ms = t;
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  cudaFree(d);
  if (e != cudaSuccess) return XDEM_ERR_CUDA;
  return h ? XDEM_ERR_TIMEOUT : XDEM_OK;
}

int32_t xdem_mlp_gradient(xdem_mlp m, int64_t n, const float* x, const float* target,
                          const float* contact, float* grad, float* loss) {
  if (!m || n <= 0 || !x || !target || !contact || !grad) return XDEM_ERR_ARGUMENT;
  float *dx = nullptr, *dt = nullptr, *dc = nullptr, *dl = nullptr;
  int32_t* dp = nullptr;
  std::vector<int32_t> ident(n);
  for (int64_t i = 0; i < n; ++i) ident[i] = (int32_t)i;
  cudaError_t e = cudaMalloc(&dx, sizeof(float) * kMlpIn * n);
  if (e == cudaSuccess) e = cudaMalloc(&dt, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dc, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dl, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dp, sizeof(int32_t) * n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dt, target, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dc, contact, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, ident.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = gradient(m, dx, dt, dc, dp, 0, n, dl);
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad, m->grad, sizeof(float) * MlpLayout::COUNT, cudaMemcpyDeviceToHost, m->stream);
  float l = 0.0f;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&l, dl, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (loss) *loss = l / (float)n;
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(dc);
  cudaFree(dl);
  cudaFree(dp);
  return e == cudaSuccess ? XDEM_OK : XDEM_ERR_CUDA;
}

int32_t xdem_mlp_add_samples(xdem_mlp m, int64_t n, const float* x, const float* target,
                             const float* contact) {
  if (!m || n <= 0 || !x || !target || !contact) return XDEM_ERR_ARGUMENT;
  if (mlp_reserve(m, m->size + n) != cudaSuccess) return XDEM_ERR_CUDA;
  cudaError_t e = cudaMemcpyAsync(m->x + kMlpIn * m->size, x, sizeof(float) * kMlpIn * n,
                                  cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->target + m->size, target, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->contact + m->size, contact, sizeof(float) * n, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return XDEM_ERR_CUDA;
  m->size += n;
  return XDEM_OK;
}

int32_t xdem_mlp_dataset(xdem_mlp m, int64_t* size, float* x, float* target, float* contact) {
  if (!m || !size) return XDEM_ERR_ARGUMENT;
  const int64_t n = m->size;
  *size = n;
  cudaError_t e = cudaSuccess;
  if (x && n) e = cudaMemcpyAsync(x, m->x, sizeof(float) * kMlpIn * n, cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess && target && n)
    e = cudaMemcpyAsync(target, m->target, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess && contact && n)
    e = cudaMemcpyAsync(contact, m->contact, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  return e == cudaSuccess ? XDEM_OK : XDEM_ERR_CUDA;
}

int32_t xdem_mlp_clear_dataset(xdem_mlp m) {
  if (!m) return XDEM_ERR_ARGUMENT;
  m->size = 0;
  return XDEM_OK;
}

int32_t xdem_mlp_train(xdem_mlp m, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                       int64_t max_samples, float* epoch_loss) {
  if (!m || epochs <= 0 || batch < kTrainRows || !(lr > 0.0f)) return XDEM_ERR_ARGUMENT;
  const int64_t n = max_samples > 0 ? std::min(max_samples, m->size) : m->size;
  if (n <= 0) return XDEM_ERR_ARGUMENT;
  if (n > m->perm_cap) {
    cudaFree(m->perm);
    m->perm = nullptr;
    if (cudaMalloc(&m->perm, sizeof(int32_t) * n) != cudaSuccess) return XDEM_ERR_CUDA;
    m->perm_cap = n;
  }
  std::vector<int32_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = (int32_t)i;
  std::mt19937_64 rng(seed);
  float* dloss = nullptr;
  const int64_t nbatches = (n + batch - 1) / batch;
  if (cudaMalloc(&dloss, sizeof(float) * (size_t)nbatches) != cudaSuccess) return XDEM_ERR_CUDA;
  cudaError_t e = cudaSuccess;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    e = cudaMemcpyAsync(m->perm, order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, m->stream);
    for (int64_t b = 0; b < nbatches && e == cudaSuccess; ++b) {
      const int64_t first = b * batch, count = std::min<int64_t>(batch, n - first);
      e = gradient(m, m->x, m->target, m->contact, m->perm, first, count, dloss + b);
      if (e != cudaSuccess) break;
      m->adam_t += 1;
      const float c1 = 1.0f - std::pow(b1, (float)m->adam_t), c2 = 1.0f - std::pow(b2, (float)m->adam_t);
      k_mlp_adam<<<(MlpLayout::COUNT + 255) / 256, 256, 0, m->stream>>>(m->theta, m->adam_m, m->adam_v,
                                                                         m->grad, lr, b1, b2, eps, c1, c2);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = publish(m);
    }
    if (e == cudaSuccess && epoch_loss) {
      std::vector<float> hl(nbatches);
      e = cudaMemcpyAsync(hl.data(), dloss, sizeof(float) * nbatches, cudaMemcpyDeviceToHost, m->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
      double s = 0.0;
      for (float v : hl) s += v;
      epoch_loss[ep] = (float)(s / (double)n);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  cudaFree(dloss);
  return e == cudaSuccess ? XDEM_OK : XDEM_ERR_CUDA;
}

}  // extern "C"
