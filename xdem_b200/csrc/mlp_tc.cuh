// mlp_tc.cuh — inference of the warm-start network (mlp.cuh) on the
// fifth-generation tensor cores: tcgen05.mma with the accumulator in tensor
// memory.
//
// A CTA of 128 threads evaluates tiles of 128 rows (one row per thread, the
// MMA's M).  Per tile:
//   features  each thread writes its row's 7 scaled inputs, rounded to BF16,
//             into the activation tile in shared memory;
//   layers    one thread issues the layer's MMAs (M=128, N=64, K=16 each;
//             layer 1 one, layers 2 and 3 four) reading the activation tile
//             and the layer's weights from shared memory, accumulating in
//             FP32 in 64 columns of tensor memory, and commits them to an
//             mbarrier; every warp then loads its 32 rows from tensor memory,
//             adds the bias, applies SiLU, and writes the BF16 activations
//             back as the next layer's A operand;
//   output    the two output units (64 → 2) in FP32 on the CUDA cores from the
//             BF16 activations, as the tensor cores would compute them.
// Weights, biases and the barrier are set up once per CTA, which then walks
// the tiles grid-stride.  Shared-memory operands use the canonical K-major
// layout without swizzle: element (r, k) of an R-row operand sits at byte
// (k / 8)·16R + 16r + 2(k % 8), so a core matrix (8 rows × 16 bytes) is
// contiguous, the 8-row groups are 128 bytes apart (the descriptor's stride
// offset) and the K chunks 16R bytes apart (its leading offset).
//
// Waits are bounded: a barrier that does not complete within kTcWaitLimit
// non-blocking polls makes every thread leave the tile loop, the tensor
// memory is freed and ST_TIMEOUT is raised.
#pragma once
#include "mlp.cuh"

namespace xdem {

constexpr int kTcRows = 128;       // rows per tile = MMA M
constexpr int kTcCols = 64;        // tensor-memory columns (FP32 accumulator, N = 64)
constexpr int kTcWaitLimit = 1 << 20;  // polls of 32 ns or more: about 0.1 s at most

struct MlpTcSmem {
  alignas(128) __nv_bfloat16 a[kTcRows * kMlpH];  // activation tile, 16 KB
  alignas(128) __nv_bfloat16 w1[kMlpH * kMlpK1];
  alignas(128) __nv_bfloat16 w2[kMlpH * kMlpH];
  alignas(128) __nv_bfloat16 w3[kMlpH * kMlpH];
  float b1[kMlpH], b2[kMlpH], b3[kMlpH];
  float w4[kMlpOut][kMlpH];
  float b4[kMlpOut];
  alignas(8) uint64_t bar;
  uint32_t tmem;
};

// element offset of (r, k) in an R-row canonical K-major operand
__device__ __forceinline__ int kmajor(int rows, int r, int k) {
  return (k >> 3) * (rows * 8) + r * 8 + (k & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start, leading (K-chunk) and stride
// (8-row group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((smem_u32(p) >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N = 64, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTcCols >> 3) << 17) |
                              ((uint32_t)(kTcRows >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate), "r"(mask0), "r"(mask1),
        "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t b = smem_u32(bar);
  for (int i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void async_proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's row (the warp's lane quarter)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// One CTA's copy of the network (weights in the canonical layout), the
// barrier and 64 columns of tensor memory.  Every thread must call.
__device__ __forceinline__ void mlp_tc_setup(MlpTcSmem& s, const MlpDev& net) {
  const int t = threadIdx.x;
  for (int i = t; i < kMlpH * kMlpK1; i += blockDim.x)
    s.w1[kmajor(kMlpH, i / kMlpK1, i % kMlpK1)] = net.wb[MlpBf16Layout::W1 + i];
  for (int i = t; i < kMlpH * kMlpH; i += blockDim.x) {
    s.w2[kmajor(kMlpH, i / kMlpH, i % kMlpH)] = net.wb[MlpBf16Layout::W2 + i];
    s.w3[kmajor(kMlpH, i / kMlpH, i % kMlpH)] = net.wb[MlpBf16Layout::W3 + i];
  }
  for (int i = t; i < kMlpH; i += blockDim.x) {
    s.b1[i] = net.theta[MlpLayout::B1 + i];
    s.b2[i] = net.theta[MlpLayout::B2 + i];
    s.b3[i] = net.theta[MlpLayout::B3 + i];
    s.w4[0][i] = __bfloat162float(net.wb[MlpBf16Layout::W4 + i]);
    s.w4[1][i] = __bfloat162float(net.wb[MlpBf16Layout::W4 + kMlpH + i]);
  }
  if (t < kMlpOut) s.b4[t] = net.theta[MlpLayout::B4 + t];
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (t < 32) {  // one whole warp allocates
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  async_proxy_fence();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void mlp_tc_teardown(MlpTcSmem& s) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(kTcCols)
                 : "memory");
}

// SiLU for the epilogue, z·σ(z) with σ(z) = (1 + tanh(z/2))/2 on the
// hardware tanh (relative error about 2^-11, below the BF16 rounding that
// follows); the exact quotient costs an order of magnitude more issue slots
// and made the epilogue the kernel's bottleneck
__device__ __forceinline__ float silu_fast(float z) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
  return z * fmaf(0.5f, t, 0.5f);
}

// this thread's 64 activations of a finished layer: tensor memory -> +bias
// -> SiLU -> BF16 (h, as the next layer reads them)
__device__ __forceinline__ void tc_epilogue(const MlpTcSmem& s, const float* bias, float* h) {
  const int warp = threadIdx.x >> 5;
  const uint32_t taddr = s.tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
  for (int c = 0; c < kTcCols; c += 16) tmem_ld16(taddr + c, h + c);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < kMlpH; ++k) h[k] = __bfloat162float(__float2bfloat16_rn(silu_fast(h[k] + bias[k])));
}

// row r's activations h into the activation tile (eight 16-byte chunks)
__device__ __forceinline__ void tc_store_row(MlpTcSmem& s, int r, const float* h) {
#pragma unroll
  for (int c = 0; c < kMlpH / 8; ++c) {
    uint4 q;
    q.x = pack_bf16(h[8 * c + 0], h[8 * c + 1]);
    q.y = pack_bf16(h[8 * c + 2], h[8 * c + 3]);
    q.z = pack_bf16(h[8 * c + 4], h[8 * c + 5]);
    q.w = pack_bf16(h[8 * c + 6], h[8 * c + 7]);
    *reinterpret_cast<uint4*>(s.a + kmajor(kTcRows, r, 8 * c)) = q;
  }
}

// Issues one layer (K = 16 * ksteps) and waits for it.  false: the barrier
// timed out in some thread (then every thread returns false).
__device__ __forceinline__ bool tc_layer(MlpTcSmem& s, const __nv_bfloat16* w, int ksteps,
                                         uint32_t& phase) {
  async_proxy_fence();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    for (int k = 0; k < ksteps; ++k)
      umma_bf16(s.tmem, umma_desc(s.a + kmajor(kTcRows, 0, 16 * k), kTcRows * 16, 128),
                umma_desc(w + kmajor(kMlpH, 0, 16 * k), kMlpH * 16, 128), k > 0 ? 1u : 0u);
    umma_commit(&s.bar);
  }
  const bool ok = mbar_wait(&s.bar, phase);
  phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// The network on the features f (7 scaled inputs) of this thread's row;
// (o0, o1) = its two outputs.  Every thread of the CTA must call, once per
// tile.  false: a barrier timed out.
__device__ __forceinline__ bool mlp_tc_tile(MlpTcSmem& s, const float* f, uint32_t& phase,
                                            float& o0, float& o1) {
  const int r = threadIdx.x;
  {
    uint4 q;
    q.x = pack_bf16(f[0], f[1]);
    q.y = pack_bf16(f[2], f[3]);
    q.z = pack_bf16(f[4], f[5]);
    q.w = pack_bf16(f[6], 0.0f);
    *reinterpret_cast<uint4*>(s.a + kmajor(kTcRows, r, 0)) = q;
    *reinterpret_cast<uint4*>(s.a + kmajor(kTcRows, r, 8)) = make_uint4(0u, 0u, 0u, 0u);
  }
  float h[kMlpH];
  if (!tc_layer(s, s.w1, kMlpK1 / 16, phase)) return false;
  tc_epilogue(s, s.b1, h);
  tc_store_row(s, r, h);
  if (!tc_layer(s, s.w2, kMlpH / 16, phase)) return false;
  tc_epilogue(s, s.b2, h);
  tc_store_row(s, r, h);
  if (!tc_layer(s, s.w3, kMlpH / 16, phase)) return false;
  tc_epilogue(s, s.b3, h);
  float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
  for (int k = 0; k < kMlpH; ++k) {
    y0 = fmaf(h[k], s.w4[0][k], y0);
    y1 = fmaf(h[k], s.w4[1][k], y1);
  }
  o0 = y0 + s.b4[0];
  o1 = y1 + s.b4[1];
  return true;
}

}  // namespace xdem
