// analysis.cuh — rattler-free coordination number and solid fraction on the
// device (QuadronAnalysis.cpp:663-668,980-986,144-165,703-713,724-732): the
// particles without contacts are dropped, then, repeatedly, the particles
// left with exactly one contact together with that contact (open chains);
// Z = 2 x remaining contacts / remaining particles, φ = their volume over the
// box area.  What remains is the 2-core of the contact graph, which does not
// depend on the order of removal, so the removal runs in parallel rounds:
// every remaining particle with at most one remaining contact leaves in the
// same round.
#pragma once
#include "kernels.cuh"

namespace xdem {

// every contact of the current record set starts active; each end counts it
// (deg must start at zero)
__global__ void k_core_init(DevWorld w, int par, int32_t* deg, uint8_t* eact) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  const int n = w.n, K = w.K;
  const Slots& cur = w.slots[par];
  const int cnt = min(cur.count[m], K);
  const int base = cnt > 0 ? cur.base[m] : 0;
  int own = 0;
  // eact: one flag per (slot, owner), slot-major scratch
  for (int s = 0; s < K; ++s) {
    const size_t e = (size_t)s * n + m;
    const int partner = s < cnt ? cur.partner[base + s] : -1;
    const bool on = partner >= 0;
    eact[e] = on ? 1 : 0;
    if (on) {
      own++;
      atomicAdd(&deg[w.mpos[partner]], 1);
    }
  }
  if (own) atomicAdd(&deg[m], own);
}

__global__ void k_core_active(DevWorld w, const int32_t* deg, uint8_t* active) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < w.n) active[m] = deg[m] > 0 ? 1 : 0;
}

// one round: the remaining particles with at most one remaining contact leave
__global__ void k_core_mark(DevWorld w, const int32_t* deg, uint8_t* active, uint8_t* leave,
                            int32_t* changed) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  const bool go = active[m] && deg[m] <= 1;
  leave[m] = go ? 1 : 0;
  if (go) {
    active[m] = 0;
    *changed = 1;
  }
}

// contacts of a leaving particle leave too; the other end loses a contact
__global__ void k_core_edges(DevWorld w, int par, int32_t* deg, const uint8_t* leave,
                             uint8_t* eact) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  const int n = w.n, K = w.K;
  const Slots& cur = w.slots[par];
  const int cnt = min(cur.count[m], K);
  const int base = cnt > 0 ? cur.base[m] : 0;
  for (int s = 0; s < cnt; ++s) {
    const size_t e = (size_t)s * n + m;
    if (!eact[e]) continue;
    const int p = w.mpos[cur.partner[base + s]];
    if (!leave[m] && !leave[p]) continue;
    eact[e] = 0;
    if (!leave[m]) atomicSub(&deg[m], 1);
    if (!leave[p]) atomicSub(&deg[p], 1);
  }
}

// per system: remaining particles, remaining contacts, their volume; one
// block per system over its memory range, fixed-order tree (deterministic)
__global__ void __launch_bounds__(256) k_core_sums(DevWorld w, const uint8_t* active,
                                                   const uint8_t* eact, double* out) {
  __shared__ double sv[256];
  __shared__ long long sp[256], se[256];
  const WorldScalars& ws = w.ws[blockIdx.x];
  const int n = w.n, K = w.K, t = threadIdx.x;
  double vol = 0.0;
  long long np = 0, ne = 0;
  for (int m = ws.first + t; m < ws.first + ws.count; m += 256) {
    if (active[m]) {
      np++;
      vol += w.vol[m];
    }
    for (int s = 0; s < K; ++s) ne += eact[(size_t)s * n + m];
  }
  sv[t] = vol;
  sp[t] = np;
  se[t] = ne;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (t < off) {
      sv[t] += sv[t + off];
      sp[t] += sp[t + off];
      se[t] += se[t + off];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[3 * blockIdx.x + 0] = sp[0] == 0 ? 0.0 : (double)se[0] / (double)sp[0] * 2.0;
    out[3 * blockIdx.x + 1] = sv[0] / (ws.xlen * ws.ylen);
    out[3 * blockIdx.x + 2] = (double)sp[0];
  }
}

}  // namespace xdem
