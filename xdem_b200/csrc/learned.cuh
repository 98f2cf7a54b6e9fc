// learned.cuh — the world side of the learned warm start (mlp.cuh):
//
//   k_mlp_warm    one warp per 16 listed closest-approach pairs: the pair's
//                 features from the FP64 state, the network on the tensor
//                 cores, and (root fraction, contact logit) into w.warm for
//                 the pair kernel that follows;
//   k_harvest     training pairs from the last candidate list: features, the
//                 root the plain FP64 Newton iteration converges to (as a
//                 fraction of its analytic start) and whether the pair touches.
#pragma once
#include "mlp.cuh"
#include "pairs.cuh"

namespace xdem {

// features of listed pair e (d = p_j + offset - p_i in ellipse i's frame)
template <bool FOLD_BG>
__device__ __forceinline__ void pair_features(const DevWorld& w, const MlpDev& net, const PairEntry& e,
                                              double2 csa, double2 csb, float* f) {
  const WorldScalars& ws = w.ws[sys_at(w, e.m)];
  const double2 pa = w.pos[e.m], pb = w.pos[e.mj];
  vec2<double> off, ovel;
  image_offset(ws, e.code & 0xff, pa, pb, off, ovel);
  const double dx = (pb.x + off.x) - pa.x, dy = (pb.y + off.y) - pa.y;
  mlp_features(net, dx, dy, csa.x, csa.y, csb.x, csb.y, w.rad[e.m], w.asp[e.m], w.rad[e.mj],
               w.asp[e.mj], f);
}

// warm starts of the entries [0, *count) of a pair list: entry i is pair
// list ? list[i] : i.  LAW_CLOSEST worlds read the orientation cosines of
// k_candidates.
template <int LAW>
__global__ void __launch_bounds__(128) k_mlp_warm(DevWorld w, MlpDev net, const int32_t* count,
                                                  const int32_t* list) {
  if (stopped(w)) return;
  __shared__ float feat[4][16 * 16];
  __shared__ float out[4][16 * 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = *count;
  const int tiles = (n + 15) / 16;
  for (int tile = blockIdx.x * 4 + warp; tile < tiles; tile += gridDim.x * 4) {
    const int i = tile * 16 + lane;
    if (lane < 16) {
      float f[kMlpIn] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
      if (i < n) {
        const PairEntry e = w.pairs[list ? list[i] : i];
        double2 csa, csb;
        if (LAW == LAW_CLOSEST) {
          csa = w.body[e.m].cs;
          csb = w.body[e.mj].cs;
        } else {
          csa = make_double2(cos(w.rot[e.m]), sin(w.rot[e.m]));
          csb = make_double2(cos(w.rot[e.mj]), sin(w.rot[e.mj]));
        }
        pair_features<false>(w, net, e, csa, csb, f);
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) feat[warp][lane * 16 + k] = k < kMlpIn ? f[k] : 0.0f;
    }
    __syncwarp();
    mlp_forward_tile(net, feat[warp], out[warp]);
    if (lane < 16 && i < n) w.warm[i] = make_float2(out[warp][lane * 2], out[warp][lane * 2 + 1]);
    __syncwarp();
  }
}

// Training pairs: every `stride`-th entry of the last candidate list whose two
// bodies are ellipses, appended to (x, target, contact) from index base; the
// number appended (capped at cap - base) accumulates in *added.
__global__ void __launch_bounds__(128) k_harvest(DevWorld w, MlpDev net, int stride, float* x,
                                                 float* target, float* contact, int64_t base,
                                                 int64_t cap, unsigned long long* added) {
  const int n = w.ws->last_pairs;
  const int lane = threadIdx.x & 31;
  for (int t0 = (blockIdx.x * blockDim.x + threadIdx.x - lane); t0 < n; t0 += gridDim.x * blockDim.x) {
    const int t = t0 + lane;
    bool keep = false;
    float f[kMlpIn];
    float tg = 0.0f, ct = 0.0f;
    if (t < n && t % stride == 0) {
      const PairEntry e = w.pairs[t];
      if (w.shape[e.m] == SHAPE_ELLIPSE && w.shape[e.mj] == SHAPE_ELLIPSE) {
        const WorldScalars& ws = w.ws[sys_at(w, e.m)];
        const PState a = load_state<false>(w, ws, e.m);
        const PState b = load_state<false>(w, ws, e.mj);
        vec2<double> off, ovel;
        image_offset(ws, e.code & 0xff, make_double2(a.x, a.y), make_double2(b.x, b.y), off, ovel);
        const double2 csa = make_double2(cos(a.rot), sin(a.rot));
        const double2 csb = make_double2(cos(b.rot), sin(b.rot));
        // features without the input scaling (the network applies it)
        MlpDev unit = net;
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) unit.scale[k] = 1.0f;
        const double dx = (b.x + off.x) - a.x, dy = (b.y + off.y) - a.y;
        mlp_features(unit, dx, dy, csa.x, csa.y, csb.x, csb.y, a.r, a.asp, b.r, b.asp, f);
        Geom g = Geom{};
        uint32_t st = 0;
        const bool touching = ellipse_closest(a, b, off, ovel, csa.x, csa.y, csb.x, csb.y, g, st);
        // a target exists when Newton ran, converged, and its root lies in the
        // interval between 1 and the analytic start that the warm start uses
        const double lo = fmin(1.0, g.q_start), hi = fmax(1.0, g.q_start);
        const bool root = g.iters > 0 && g.iters < kNewtonCap && g.q_start > 0.0 &&
                          g.q >= lo * (1.0 - 1e-9) && g.q <= hi * (1.0 + 1e-9);
        tg = root ? (float)(g.q / g.q_start) : __int_as_float(0x7fc00000);
        ct = touching ? 1.0f : 0.0f;
        keep = true;
      }
    }
    const unsigned take = __ballot_sync(0xffffffffu, keep);
    if (take == 0) continue;
    unsigned long long at = 0;
    if (lane == __ffs(take) - 1) at = atomicAdd(added, (unsigned long long)__popc(take));
    at = __shfl_sync(0xffffffffu, at, __ffs(take) - 1);
    if (keep) {
      const int64_t idx = base + (int64_t)at + __popc(take & ((1u << lane) - 1u));
      if (idx < cap) {
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) x[idx * kMlpIn + k] = f[k];
        target[idx] = tg;
        contact[idx] = ct;
      }
    }
  }
}

}  // namespace xdem
