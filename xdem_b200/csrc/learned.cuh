// learned.cuh — the world side of the learned warm start (mlp.cuh):
//
//   k_mlp_warm    tiles of 128 listed closest-approach pairs: the pair's
//                 features from the FP64 state, the network on the tensor
//                 cores (tcgen05, mlp_tc.cuh), and (root fraction, contact
//                 logit) into w.warm for the pair kernel that follows;
//   k_harvest     training pairs from the last candidate list: features, the
//                 root the plain FP64 Newton iteration converges to (as a
//                 fraction of its analytic start) and whether the pair touches.
#pragma once
#include "mlp_tc.cuh"
#include "pairs.cuh"

namespace xdem {

// warm starts of the entries [0, *count) of a pair list: entry i is pair
// list ? list[i] : i.  Tiles of 128 entries go through the network on the
// tensor cores (mlp_tc.cuh); the features come from the pair's body records.
template <int LAW>
__global__ void __launch_bounds__(128) k_mlp_warm(DevWorld w, MlpDev net, const int32_t* count,
                                                  const int32_t* list) {
  if (stopped(w)) return;
  __shared__ MlpTcSmem s;
  mlp_tc_setup(s, net);
  uint32_t phase = 0;
  const int n = *count;
  const int tiles = (n + kTcRows - 1) / kTcRows;
  bool failed = false;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int i = tile * kTcRows + threadIdx.x;
    float f[kMlpIn] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (i < n) {
      const PairEntry e = w.pairs[list ? list[i] : i];
      const BodyRec ba = w.body[e.m], bb = w.body[e.mj];
      const WorldScalars& ws = w.ws[sys_at(w, e.m)];
      vec2<double> off, ovel;
      image_offset(ws, e.code & 0xff, ba.pos, bb.pos, off, ovel);
      const double dx = (bb.pos.x + off.x) - ba.pos.x, dy = (bb.pos.y + off.y) - ba.pos.y;
      mlp_features(net, dx, dy, ba.cs.x, ba.cs.y, bb.cs.x, bb.cs.y, ba.r, ba.asp, bb.r, bb.asp, f);
    }
    float o0, o1;
    if (!mlp_tc_tile(s, f, phase, o0, o1)) {
      failed = true;
      break;
    }
    if (i < n) w.warm[i] = make_float2(o0, o1);
  }
  mlp_tc_teardown(s);
  if (failed && threadIdx.x == 0) raise(w.status, ST_TIMEOUT);
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
      // carried-over records are no candidate pairs
      if (!(e.code & kCarryFlag) && w.shape[e.m] == SHAPE_ELLIPSE &&
          w.shape[e.mj] == SHAPE_ELLIPSE) {
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
        const bool root = g.iters > 0 && !g.stuck && g.q_start > 0.0 &&
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
