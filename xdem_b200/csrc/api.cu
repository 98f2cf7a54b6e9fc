// api.cu — the C-ABI of include/xdem_gpu.h: world lifetime, host<->device
// transfers, and the launch sequences of each reference step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/xdem_gpu.h"
#include "kernels.cuh"
#include "pairs.cuh"
#include "pairs_mixed.cuh"
#include "learned.cuh"
#include "verlet.cuh"
#include "analysis.cuh"
#include "mlp_host.h"
#include "resort.cuh"

using namespace xdem;

namespace {

constexpr int kBlock = 128;
constexpr int kDefaultSlots = 24;
// default steps between memory-order refreshes; odd, so that a captured
// chunk (one re-sort + kResortEvery steps) swaps the record sets an even number
// of times.  On the 1M shear a re-sort costs ~1.5 ms and every 63 steps keeps
// the neighbour gathers as local as every 31 (0.863 against 0.909 ms/step;
// 127: 0.859)
constexpr int kResortEvery = 63;
// since_resort value that makes the next step refresh the memory order
constexpr int kResortDue = 1 << 30;
constexpr double kPi = 3.14159265358979323846;

inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

struct DeviceBuffers {
  std::vector<void*> ptrs;
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return cudaSuccess;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

}  // namespace

struct xdem_world_s {
  xdem_params prm{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  DevWorld dw{};
  DeviceBuffers particle_bufs;
  WorldScalars* ws = nullptr;
  uint32_t* status = nullptr;
  int par = 0;            // record set holding the latest contacts
  int nsys = 1;           // systems (batched worlds: more than one)
  int partial_blocks = 0;
  uint32_t host_status = 0;
  double total_volume = 0.0;
  std::vector<double> control_mass{0.0};  // per system
  // per-kernel timing
  bool prof_on = false;
  std::vector<cudaEvent_t> prof_events;  // pairs (begin, end)
  std::vector<int> prof_kind;            // kind of each pair
  size_t prof_used = 0;                  // pairs recorded
  int64_t launches = 0;
  cudaEvent_t timer[2] = {nullptr, nullptr};
  int since_resort = kResortDue;  // steps since the memory order was refreshed
  // steps between memory-order refreshes (odd), 0 = never
  // (xdem_set_memory_order_refresh)
  int resort_every = kResortEvery;
  int law = LAW_ANY;                // contact-kernel specialisation for the shapes present
  bool has_clumps = false;          // a clump's time integral reads its sub-particles' sums
  bool list_decided = false;        // the step's list-rebuild decision is already enqueued
  bool body_written = false;        // the step's body records are written by its binning
  xdem_mlp_s* mlp = nullptr;        // learned warm start of the closest-approach Newton iteration
  PermList perm{};                  // particle arrays moved by a re-sort
  // launch configuration (xdem_set_launch_config / xdem_autotune): blocks per
  // SM of the pair kernels (their grid-stride loop gives each thread
  // npairs / (blocks * 128) pairs) and the cell size as a multiple of each
  // system's base cell size
  int pair_blocks_per_sm = 16;
  double cell_factor = 1.0;
  std::vector<double> base_maxsize;
  // candidate lists (verlet.cuh): entries per particle (0 = full scan every
  // step) and the skin as a fraction of the smallest base cell size
  int vl_capacity = 48;
  double skin_fraction = 0.1;
};

namespace {

inline uint32_t cuda_check(xdem_world_s* w, cudaError_t e) {
  if (e == cudaSuccess) return 0;
  if (w) w->host_status |= XDEM_ERR_CUDA;
  return XDEM_ERR_CUDA;
}

#define CK(w, call)                                    \
  do {                                                 \
    if (uint32_t _s = cuda_check((w), (call))) return (int32_t)_s; \
  } while (0)

double factor_of(double kn, double e) {
  // ContactModel_LinearDissipativeFrictioanl ctor (…Frictional.h:18-23)
  double lg = std::log(e);
  return 2.0 * std::sqrt(kn) * std::fabs(lg) / std::sqrt(kPi * kPi + lg * lg);
}

cudaError_t read_scalars(xdem_world_s* w, WorldScalars* out) {
  cudaError_t e = cudaMemcpyAsync(out, w->ws, sizeof(WorldScalars), cudaMemcpyDeviceToHost, w->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(w->stream);
}

cudaError_t write_scalars(xdem_world_s* w, const WorldScalars* in) {
  cudaError_t e = cudaMemcpyAsync(w->ws, in, sizeof(WorldScalars), cudaMemcpyHostToDevice, w->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(w->stream);
}

// applies f to the scalars of every system of the world
template <class F>
cudaError_t modify_all(xdem_world_s* w, F f) {
  std::vector<WorldScalars> all(w->nsys);
  cudaError_t e = cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys,
                                  cudaMemcpyDeviceToHost, w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return e;
  for (int s = 0; s < w->nsys; ++s) f(all[s], s);
  e = cudaMemcpyAsync(w->ws, all.data(), sizeof(WorldScalars) * w->nsys, cudaMemcpyHostToDevice,
                      w->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(w->stream);
}

template <class T>
cudaError_t upload(T* dst, const T* src, size_t count, cudaStream_t s) {
  return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s);
}
template <class T>
cudaError_t download(T* dst, const T* src, size_t count, cudaStream_t s) {
  return cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s);
}

// ---- per-kernel timing ------------------------------------------------------
enum KernelKind {
  KK_MODIFY = 0, KK_BIN, KK_SCAN, KK_SCATTER, KK_CANDIDATES, KK_PAIRS, KK_COLLECT_INTEGRATE, KK_COLLECT,
  KK_INTEGRATE, KK_RATTLERS, KK_STRESS_PARTIAL, KK_STRESS_FINAL, KK_END_OF_STEP, KK_SCALE,
  KK_BACKGROUND, KK_KE, KK_RESORT, KK_STAGE, KK_FALLBACK, KK_WARM, KK_VL_CHECK, KK_VL_BUILD,
  KK_DEEP, KK_COUNT
};
const char* const kKindNames[KK_COUNT] = {
    "k_modify_position", "k_bin", "k_scan", "k_scatter", "k_candidates", "k_pair_forces",
    "k_collect_integrate", "k_collect", "k_integrate", "k_rattlers", "k_stress_partial",
    "k_stress_final", "k_end_of_step", "k_scale_positions", "k_background_velocity",
    "k_kinetic_energy", "k_resort", "k_stage", "k_pair_fallback", "k_mlp_warm", "k_vl_check",
    "k_vl_build", "k_pair_deep"};

void prof_begin(xdem_world_s* w, int kind) {
  if (!w->prof_on) return;
  size_t need = 2 * (w->prof_used + 1);
  while (w->prof_events.size() < need) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) {
      w->host_status |= XDEM_ERR_CUDA;
      w->prof_on = false;
      return;
    }
    w->prof_events.push_back(e);
  }
  if (w->prof_kind.size() <= w->prof_used) w->prof_kind.resize(w->prof_used + 1);
  w->prof_kind[w->prof_used] = kind;
  cudaEventRecord(w->prof_events[2 * w->prof_used], w->stream);
}

void prof_end(xdem_world_s* w) {
  if (!w->prof_on) return;
  cudaEventRecord(w->prof_events[2 * w->prof_used + 1], w->stream);
  w->prof_used++;
}

#define LAUNCH(w, kind, ...)  \
  do {                        \
    prof_begin((w), (kind));  \
    __VA_ARGS__;              \
    prof_end((w));            \
    (w)->launches++;          \
  } while (0)

// ---- launch helpers -------------------------------------------------------
// A step kernel as a programmatic dependent launch: it may become resident
// while the kernel before it runs and waits in its pdl_begin until that one
// has completed, so that its launch and its blocks' start overlap the other's
// tail.  While the kernels are timed one by one it is an ordinary launch.
template <typename... KArgs, typename... Args>
void launch_chain(xdem_world_s* w, int kind, void (*kernel)(KArgs...), int grid, int block,
                  size_t smem, Args... args) {
  prof_begin(w, kind);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = w->prof_on ? 0 : 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = w->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cuda_check(w, cudaLaunchKernelEx(&cfg, kernel, args...));
  prof_end(w);
  w->launches++;
}

void launch_modify(xdem_world_s* w) {
  int n = w->dw.n;
  LAUNCH(w, KK_MODIFY, k_modify_position<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw));
}

// whether this step rebuilds the candidate lists (a grid-stride pass over the
// path lengths, few blocks, so that the last one has few maxima to combine)
void launch_list_decision(xdem_world_s* w) {
  const int vb = std::min(blocks_for(w->dw.n, kVlBlock), 148 * 4);
  launch_chain(w, KK_VL_CHECK, k_vl_maxdisp, vb, kVlBlock, 0, w->dw);
}

// findPossibleContacts' binning; modify: the step's position move first, in
// the binning kernel
// decided: the step's list-rebuild decision is taken between the scan and the
// scatter, which then writes the cell records only where a scan reads them
void launch_find(xdem_world_s* w, bool modify = false, bool decided = false) {
  int n = w->dw.n;
  if (modify)
    launch_chain(w, KK_BIN, k_bin<true>, blocks_for(n, kBlock), kBlock, 0, w->dw);
  else
    launch_chain(w, KK_BIN, k_bin<false>, blocks_for(n, kBlock), kBlock, 0, w->dw);
  int cells = w->dw.ncell_total;
  int tiles = std::min(blocks_for(cells, kScanTile), 2 * 148 * 8);
  launch_chain(w, KK_SCAN, k_scan_tiles, tiles, kScanThreads, 0, w->dw);
  launch_chain(w, KK_SCAN, k_scan_apply, tiles, kScanThreads, 0, w->dw);
  int nb = std::max(blocks_for(n, kBlock), std::min(blocks_for(cells, kBlock), 1184));
  if (decided) launch_list_decision(w);
  launch_chain(w, KK_SCATTER, k_scatter, nb, kBlock, 0, w->dw, decided ? 1 : 0);
}

// A pair kernel (DevWorld, slot-set parity, record) on the world's stream as
// a programmatic dependent launch: it may start while the kernel before it
// (which signals with griddepcontrol.launch_dependents) still runs.  The
// launch after it is an ordinary one and waits for both.
void launch_dependent(xdem_world_s* w, int blocks, void (*kernel)(DevWorld, int, int, int),
                      int record) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = w->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cuda_check(w, cudaLaunchKernelEx(&cfg, kernel, w->dw, w->par, record, 0));
  w->launches++;
}

// updateContacts as candidate scan, per-pair forces, and history carry-over
// (pairs.cuh); the pair kernel runs a grid-stride loop over the listed pairs
// dynamic shared memory of k_candidates_vl: the kept entries of a block's 128
// owners, partner positions and codes, K slots each
static size_t candidates_smem(const xdem_world_s* w) {
  return (size_t)2 * w->dw.K * 128 * sizeof(int32_t);
}

template <bool FOLD_BG, int LAW>
void launch_update_phases(xdem_world_s* w, int record) {
  const int nb = blocks_for(w->dw.n, 128);
  const int pb = 148 * w->pair_blocks_per_sm;
  // the learned warm start applies to closest-approach worlds
  const bool warm = w->mlp != nullptr && w->dw.warm != nullptr && LAW == LAW_CLOSEST;
  if (w->dw.V > 0) {
    if (!w->list_decided) launch_list_decision(w);
    launch_chain(w, KK_VL_BUILD, k_vl_build<LAW>, nb, 128, 0, w->dw);
    launch_chain(w, KK_CANDIDATES, k_candidates_vl<LAW>, nb, 128, candidates_smem(w), w->dw, w->par,
                 w->body_written ? 0 : 1);
  } else {
    LAUNCH(w, KK_CANDIDATES, k_candidates<LAW><<<nb, 128, 0, w->stream>>>(w->dw, w->par));
  }
  // the launch that ends the pair phase (finish = 1) also resets the pair
  // counters for the next update (finish_pairs)
  // deep pairs are listed apart where the closest-approach law applies
  const bool deep_lists = LAW == LAW_CLOSEST || (LAW == LAW_ANY && w->prm.ellipse_method ==
                                                                       XDEM_ELLIPSE_CLOSEST_APPROACH);
  if (w->prm.precision == XDEM_PRECISION_MIXED && deep_lists && !warm) {
    // The deep pairs first, then the regular pair pass as a programmatic
    // dependent launch: every block of k_pair_deep_m signals at its start, so
    // the regular pass starts once the deep pass is on the GPU and runs
    // beside it (in whatever order the blocks would otherwise be dispatched).
    // The regular pass uses nothing the deep pass writes; the deferred pass
    // after it is an ordinary launch and waits for both.  While the kernels
    // are timed one by one the regular pass is an ordinary launch too.
    launch_chain(w, KK_DEEP, k_pair_deep_m<FOLD_BG, LAW>, 148 * 2, 128, 0, w->dw, w->par, record);
    if (w->prof_on) {
      LAUNCH(w, KK_PAIRS, k_pair_forces_m<FOLD_BG, LAW, PASS_REGULAR><<<pb, 128, 0, w->stream>>>(
                              w->dw, w->par, record, 0));
    } else {
      launch_dependent(w, pb, k_pair_forces_m<FOLD_BG, LAW, PASS_REGULAR>, record);
    }
    LAUNCH(w, KK_FALLBACK, k_pair_fallback_m<FOLD_BG, LAW><<<148 * 4, 128, 0, w->stream>>>(
                               w->dw, w->par, record, 1));
  } else if (w->prm.precision == XDEM_PRECISION_MIXED) {
    const bool deferred = LAW == LAW_CLOSEST || LAW == LAW_ANY;
    LAUNCH(w, KK_PAIRS, k_pair_forces_m<FOLD_BG, LAW><<<pb, 128, 0, w->stream>>>(
                            w->dw, w->par, record, deferred ? 0 : 1));
    if (deferred) {
      if (warm) {
        LAUNCH(w, KK_WARM, k_mlp_warm<LAW><<<148 * 4, 128, 0, w->stream>>>(
                               w->dw, w->mlp->dev(), w->dw.nfallback, w->dw.fallback));
        LAUNCH(w, KK_FALLBACK, k_pair_fallback_m<FOLD_BG, LAW, true><<<148 * 4, 128, 0, w->stream>>>(
                                   w->dw, w->par, record, 1));
      } else {
        LAUNCH(w, KK_FALLBACK, k_pair_fallback_m<FOLD_BG, LAW><<<148 * 4, 128, 0, w->stream>>>(
                                   w->dw, w->par, record, 1));
      }
    }
  } else if (warm) {
    LAUNCH(w, KK_WARM,
           k_mlp_warm<LAW><<<148 * 4, 128, 0, w->stream>>>(w->dw, w->mlp->dev(), w->dw.npairs, nullptr));
    LAUNCH(w, KK_PAIRS,
           k_pair_forces<FOLD_BG, LAW, true><<<pb, 128, 0, w->stream>>>(w->dw, w->par, record, 1));
  } else {
    LAUNCH(w, KK_PAIRS,
           k_pair_forces<FOLD_BG, LAW><<<pb, 128, 0, w->stream>>>(w->dw, w->par, record, 1));
  }
}

template <bool FOLD_BG>
void launch_update_law(xdem_world_s* w, int record) {
  switch (w->law) {
    case LAW_CIRCLE: launch_update_phases<FOLD_BG, LAW_CIRCLE>(w, record); break;
    case LAW_CLOSEST: launch_update_phases<FOLD_BG, LAW_CLOSEST>(w, record); break;
    case LAW_INTERSECTION: launch_update_phases<FOLD_BG, LAW_INTERSECTION>(w, record); break;
    default: launch_update_phases<FOLD_BG, LAW_ANY>(w, record); break;
  }
}

void launch_update(xdem_world_s* w, bool fold_bg, int record) {
  if (fold_bg) launch_update_law<true>(w, record);
  else launch_update_law<false>(w, record);
  w->par ^= 1;
}

void launch_collect(xdem_world_s* w) {
  int n = w->dw.n;
  LAUNCH(w, KK_COLLECT, k_collect<<<blocks_for(n, 128), 128, 0, w->stream>>>(w->dw, w->par));
}

void launch_integrate(xdem_world_s* w, bool fold_bg, int reset) {
  int n = w->dw.n;
  if (fold_bg)
    LAUNCH(w, KK_INTEGRATE, k_integrate<true><<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, reset));
  else
    LAUNCH(w, KK_INTEGRATE, k_integrate<false><<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, reset));
}

// the force sum and the time integral of a world without clumps in one pass
void launch_collect_integrate(xdem_world_s* w, bool fold_bg, int reset) {
  int n = w->dw.n;
  if (fold_bg)
    launch_chain(w, KK_COLLECT_INTEGRATE, k_collect_integrate<true>, blocks_for(n, 128), 128, 0,
                 w->dw, w->par, reset);
  else
    launch_chain(w, KK_COLLECT_INTEGRATE, k_collect_integrate<false>, blocks_for(n, 128), 128, 0,
                 w->dw, w->par, reset);
}

void launch_stress(xdem_world_s* w) {
  if (w->nsys > 1) {
    LAUNCH(w, KK_STRESS_PARTIAL,
           k_stress_systems<<<w->nsys, kReduceBlock, 0, w->stream>>>(w->dw, w->par));
    return;
  }
  int nb = blocks_for(w->dw.n, kReduceBlock);
  LAUNCH(w, KK_STRESS_PARTIAL, k_stress_partial<<<nb, kReduceBlock, 0, w->stream>>>(w->dw, w->par));
  LAUNCH(w, KK_STRESS_FINAL, k_stress_final<<<1, 1024, 0, w->stream>>>(w->dw, nb));
}

void launch_rattlers(xdem_world_s* w, int reset, double scale) {
  int n = w->dw.n;
  LAUNCH(w, KK_RATTLERS, k_rattlers<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, reset, scale));
}

void launch_end_of_step(xdem_world_s* w, int law, double p0, double p1, int le_update, int stop_on,
                        double stop_p, int count_step) {
  LAUNCH(w, KK_END_OF_STEP,
         k_end_of_step<<<blocks_for(w->nsys, 128), 128, 0, w->stream>>>(
             w->dw, law, p0, p1, le_update, stop_on, stop_p, count_step));
  if (law != BOX_NONE)
    LAUNCH(w, KK_SCALE, k_scale_positions<<<blocks_for(w->dw.n, kBlock), kBlock, 0, w->stream>>>(w->dw));
}

// refresh of the memory order (resort.cuh), after a step's binning
void launch_resort(xdem_world_s* w) {
  int n = w->dw.n;
  int cells = w->dw.ncell_total;
  int cb = std::min(blocks_for(cells, kBlock), 148 * 16);
  LAUNCH(w, KK_RESORT, k_sort_cells<<<cb, kBlock, 0, w->stream>>>(w->dw));
  LAUNCH(w, KK_RESORT, k_permute<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, w->perm));
  LAUNCH(w, KK_RESORT, k_copy_back<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, w->perm));
  LAUNCH(w, KK_RESORT,
         k_permute_history<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, w->par));
  w->par ^= 1;
  LAUNCH(w, KK_RESORT, k_remap_cells<<<std::min(blocks_for(2 * n, kBlock), 148 * 16), kBlock, 0,
                                       w->stream>>>(w->dw));
}

// one step of a control sequence; record: store the full contact record;
// resort: refresh the memory order after the binning
void enqueue_step(xdem_world_s* w, const xdem_control* ctl, int record, bool resort = false) {
  int kind = w->prm.world_kind;
  bool own = ctl->sequence == XDEM_SEQ_TAKE_TIME_STEP;
  bool le = own && kind == XDEM_WORLD_LEES_EDWARDS;
  if (ctl->scale_rattlers) launch_rattlers(w, 0, ctl->rattler_scale);
  // with candidate lists and no re-sort the rebuild decision comes before the
  // scatter, so that the cell records are written only when a scan reads
  // them; a re-sort reorders the records and invalidates the lists, so its
  // step writes them all and decides after it
  const bool decided = w->dw.V > 0 && !resort;
  launch_find(w, true, decided);
  if (resort) launch_resort(w);
  w->list_decided = decided;
  w->body_written = !resort;  // a re-sort moves the particles after the binning wrote them
  launch_update(w, le, record);
  w->list_decided = false;
  w->body_written = false;
  if (w->has_clumps) {
    // a clump's time integral reads its sub-particles' sums: the sum pass
    // first (one thread taking a clump's sub-particles serially measured
    // slower than the two passes)
    launch_collect(w);
    launch_integrate(w, le, own && kind == XDEM_WORLD_PERIODIC_CONTROL);
  } else {
    launch_collect_integrate(w, le, own && kind == XDEM_WORLD_PERIODIC_CONTROL);
  }
  if (ctl->reset_rattlers) launch_rattlers(w, 1, 0.0);
  if (ctl->update_stress) launch_stress(w);
  launch_end_of_step(w, ctl->box_law, ctl->p0, ctl->p1, le ? 1 : 0, ctl->stop_on_pressure,
                     ctl->stop_pressure, 1);
}

// a step with the re-sort policy: the memory order is refreshed every
// resort_every steps (never when it is 0)
void policy_step(xdem_world_s* w, const xdem_control* ctl, int record) {
  bool resort = w->resort_every > 0 && w->since_resort >= w->resort_every;
  if (resort) w->since_resort = 0;
  enqueue_step(w, ctl, record, resort);
  w->since_resort++;
}

// host arrays in id order from device arrays in memory order
template <class T>
cudaError_t download_by_id(xdem_world_s* w, T* dst, const T* src, const std::vector<int32_t>& id_of) {
  const int n = w->dw.n;
  std::vector<T> tmp(n);
  cudaError_t e = download(tmp.data(), src, n, w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return e;
  for (int m = 0; m < n; ++m) dst[id_of[m]] = tmp[m];
  return cudaSuccess;
}

cudaError_t fetch_id_of(xdem_world_s* w, std::vector<int32_t>& id_of) {
  id_of.resize(w->dw.n);
  cudaError_t e = download(id_of.data(), w->dw.id_of, w->dw.n, w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  return e;
}

uint32_t fetch_status(xdem_world_s* w) {
  uint32_t s = 0;
  cudaError_t e = cudaMemcpyAsync(&s, w->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, w->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->status, 0, sizeof(uint32_t), w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) w->host_status |= XDEM_ERR_CUDA;
  s |= w->host_status;
  w->host_status = 0;
  return s;
}

}  // namespace

extern "C" {

int32_t xdem_abi_version(void) { return XDEM_ABI_VERSION; }

const char* xdem_status_string(int32_t bit) {
  switch (bit) {
    case XDEM_OK: return "ok";
    case XDEM_ERR_CAPACITY: return "capacity exceeded (candidate list or contact slots)";
    case XDEM_ERR_NEWTON: return "closest-approach Newton iteration did not converge";
    case XDEM_ERR_NONFINITE: return "non-finite value";
    case XDEM_ERR_UNSUPPORTED_PAIR: return "no contact law for this pair of shapes";
    case XDEM_ERR_ZERO_VECTOR: return "normalisation of a zero-length vector";
    case XDEM_ERR_CUDA: return "CUDA runtime error";
    case XDEM_ERR_ARGUMENT: return "invalid argument";
    case XDEM_ERR_GRID: return "cell grid has fewer than 3 cells along an axis";
    case XDEM_ERR_TIMEOUT: return "a device-side wait ran out of its iteration limit";
    default: return "unknown status";
  }
}

int32_t xdem_device_count(int32_t* out) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (out) *out = (e == cudaSuccess) ? c : 0;
  return (e == cudaSuccess && c > 0) ? XDEM_OK : XDEM_ERR_CUDA;
}

int32_t xdem_create(const xdem_params* prm, xdem_world* out) {
  if (!prm || !out) return XDEM_ERR_ARGUMENT;
  *out = nullptr;
  if (prm->world_kind < 0 || prm->world_kind > 2 || prm->ellipse_method < 0 ||
      prm->ellipse_method > 1 || prm->precision < 0 || prm->precision > 1 ||
      prm->max_contacts < 0 || prm->max_contacts > kMaxSlots || !(prm->dt > 0.0))
    return XDEM_ERR_ARGUMENT;
  xdem_world_s* w = new (std::nothrow) xdem_world_s();
  if (!w) return XDEM_ERR_ARGUMENT;
  w->prm = *prm;
  if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete w;
    return XDEM_ERR_CUDA;
  }
  w->own_stream = true;
  if (cudaMalloc(&w->ws, sizeof(WorldScalars)) != cudaSuccess ||
      cudaMalloc(&w->status, sizeof(uint32_t)) != cudaSuccess) {
    xdem_destroy(w);
    return XDEM_ERR_CUDA;
  }
  WorldScalars s{};
  s.xmin = prm->xmin;
  s.xmax = prm->xmax;
  s.ymin = prm->ymin;
  s.ymax = prm->ymax;
  s.xlen = s.xmax - s.xmin;
  s.ylen = s.ymax - s.ymin;
  s.shift_rate = prm->shift_strain_rate;
  s.shift_vel = s.shift_rate * s.ylen;  // setShiftStrainRate (LeesEdwardsBoundaryWorld.cpp:485-489)
  s.dt = prm->dt;
  s.g = prm->global_damping;
  s.kn = prm->normal_stiffness;
  s.kt = prm->shear_stiffness;
  s.mu = prm->frictional_coeff;
  s.factor = factor_of(prm->normal_stiffness, prm->restitution_coeff);
  s.scale_x = s.scale_y = 1.0;
  if (write_scalars(w, &s) != cudaSuccess || cudaMemset(w->status, 0, sizeof(uint32_t)) != cudaSuccess) {
    xdem_destroy(w);
    return XDEM_ERR_CUDA;
  }
  w->dw.ws = w->ws;
  w->dw.nsys = 1;
  w->dw.status = w->status;
  w->dw.kind = prm->world_kind;
  w->dw.method = prm->ellipse_method;
  w->dw.precision = prm->precision;
  w->dw.K = prm->max_contacts > 0 ? prm->max_contacts : kDefaultSlots;
  *out = w;
  return XDEM_OK;
}

int32_t xdem_destroy(xdem_world w) {
  if (!w) return XDEM_OK;
  if (w->stream) cudaStreamSynchronize(w->stream);
  w->particle_bufs.release();
  for (cudaEvent_t e : w->prof_events) cudaEventDestroy(e);
  for (cudaEvent_t e : w->timer)
    if (e) cudaEventDestroy(e);
  if (w->ws) cudaFree(w->ws);
  if (w->status) cudaFree(w->status);
  if (w->own_stream && w->stream) cudaStreamDestroy(w->stream);
  delete w;
  return XDEM_OK;
}

int32_t xdem_get_stream(xdem_world w, void** s) {
  if (!w || !s) return XDEM_ERR_ARGUMENT;
  *s = static_cast<void*>(w->stream);
  return XDEM_OK;
}

int32_t xdem_set_stream(xdem_world w, void* s) {
  if (!w) return XDEM_ERR_ARGUMENT;
  cudaStreamSynchronize(w->stream);
  if (w->own_stream) cudaStreamDestroy(w->stream);
  if (s) {
    w->stream = static_cast<cudaStream_t>(s);
    w->own_stream = false;
  } else {
    CK(w, cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    w->own_stream = true;
  }
  return XDEM_OK;
}

}  // extern "C"

namespace {

// One system of a world: particles [first, first + count), its box, time step.
struct SysDesc {
  int first, count;
  double box[4];
  double dt;
};

// Uploads the particles P (all systems, ids global) and sizes every device
// array; sys lists the systems in id order (one entry for a single world,
// whose box and time step are then taken from its current scalars).
int32_t set_particles_impl(xdem_world_s* w, const xdem_particles* P, const std::vector<SysDesc>& sys) {
  if (!w || !P || P->n <= 0 || sys.empty()) return XDEM_ERR_ARGUMENT;
  const int n = P->n;
  if ((int64_t)n * w->dw.K >= (int64_t)1 << 31) return XDEM_ERR_ARGUMENT;
  if (!P->shape || !P->up_level || !P->setting || !P->outer_radius || !P->radius ||
      !P->aspect_ratio || !P->x || !P->y || !P->vx || !P->vy || !P->rot || !P->rot_vel ||
      !P->volume || !P->mass || !P->inv_mass || !P->inertia || !P->inv_inertia)
    return XDEM_ERR_ARGUMENT;
  cudaStreamSynchronize(w->stream);
  w->particle_bufs.release();
  DevWorld& d = w->dw;
  d.n = n;
  const int K = d.K;
  DeviceBuffers& B = w->particle_bufs;
  int32_t *shape, *up, *setting, *num_sub;
  double *orad, *rad, *asp, *mass, *im, *I, *iI, *vol;
  CK(w, B.alloc(&shape, n));
  CK(w, B.alloc(&up, n));
  CK(w, B.alloc(&setting, n));
  CK(w, B.alloc(&num_sub, n));
  CK(w, B.alloc(&orad, n));
  CK(w, B.alloc(&rad, n));
  CK(w, B.alloc(&asp, n));
  CK(w, B.alloc(&mass, n));
  CK(w, B.alloc(&im, n));
  CK(w, B.alloc(&I, n));
  CK(w, B.alloc(&iI, n));
  CK(w, B.alloc(&vol, n));
  CK(w, B.alloc(&d.pos, n));
  CK(w, B.alloc(&d.vel, n));
  CK(w, B.alloc(&d.rot, n));
  CK(w, B.alloc(&d.w, n));
  CK(w, B.alloc(&d.branch, n));
  CK(w, B.alloc(&d.rattler, n));
  CK(w, B.alloc(&d.force, n));
  CK(w, B.alloc(&d.torque, n));
  CK(w, B.alloc(&d.ncp, n));
  d.shape = shape;
  d.up = up;
  d.setting = setting;
  d.num_sub = num_sub;
  d.orad = orad;
  d.rad = rad;
  d.asp = asp;
  d.mass = mass;
  d.im = im;
  d.I = I;
  d.iI = iI;
  d.vol = vol;
  // host-side derived data
  std::vector<double2> pos(n), vel(n), br(n);
  std::vector<int32_t> ns(n, 0), rat(n, 0);
  for (int i = 0; i < n; ++i) {
    pos[i] = make_double2(P->x[i], P->y[i]);
    vel[i] = make_double2(P->vx[i], P->vy[i]);
    br[i] = make_double2(P->branch_x ? P->branch_x[i] : 0.0, P->branch_y ? P->branch_y[i] : 0.0);
    if (P->num_sub) ns[i] = P->num_sub[i];
    if (P->is_rattler) rat[i] = P->is_rattler[i];
    if (P->shape[i] < 0 || P->shape[i] > 3) return XDEM_ERR_ARGUMENT;
    if (P->shape[i] == XDEM_SHAPE_SEGMENT && (!P->seg_x1 || !P->seg_y1 || !P->seg_x2 || !P->seg_y2))
      return XDEM_ERR_ARGUMENT;
    if (P->shape[i] == XDEM_SHAPE_CLUMP && (ns[i] < 0 || i + ns[i] >= n)) return XDEM_ERR_ARGUMENT;
  }
  // per system: largest outer radius (updateMaximumParticleSize,
  // BaseWorld.cpp:201-219), particle volume (updateTotalParticleVolume,
  // BaseWorld.cpp:188-199) and mass
  const int nsys = (int)sys.size();
  std::vector<double> sys_maxr(nsys, 0.0), sys_vol(nsys, 0.0), sys_mass(nsys, 0.0);
  std::vector<int32_t> sys_of(n, 0);
  for (int k = 0; k < nsys; ++k) {
    if (sys[k].first < 0 || sys[k].count <= 0 || sys[k].first + sys[k].count > n)
      return XDEM_ERR_ARGUMENT;
    for (int i = sys[k].first; i < sys[k].first + sys[k].count; ++i) {
      sys_of[i] = k;
      // a clump's sub-particles belong to its system
      if (P->shape[i] == XDEM_SHAPE_CLUMP && i + ns[i] >= sys[k].first + sys[k].count)
        return XDEM_ERR_ARGUMENT;
      if (P->outer_radius[i] > sys_maxr[k]) sys_maxr[k] = P->outer_radius[i];
      if (!(P->setting[i] & XDEM_SKIP_MACRO_SUM)) {
        sys_vol[k] += P->volume[i];
        sys_mass[k] += P->mass[i];
      }
    }
  }
  cudaStream_t s = w->stream;
  CK(w, upload(shape, P->shape, n, s));
  CK(w, upload(up, P->up_level, n, s));
  CK(w, upload(setting, P->setting, n, s));
  CK(w, upload(num_sub, ns.data(), n, s));
  CK(w, upload(orad, P->outer_radius, n, s));
  CK(w, upload(rad, P->radius, n, s));
  CK(w, upload(asp, P->aspect_ratio, n, s));
  CK(w, upload(mass, P->mass, n, s));
  CK(w, upload(im, P->inv_mass, n, s));
  CK(w, upload(I, P->inertia, n, s));
  CK(w, upload(iI, P->inv_inertia, n, s));
  CK(w, upload(vol, P->volume, n, s));
  CK(w, upload(d.pos, pos.data(), n, s));
  CK(w, upload(d.vel, vel.data(), n, s));
  CK(w, upload(d.rot, P->rot, n, s));
  CK(w, upload(d.w, P->rot_vel, n, s));
  CK(w, upload(d.branch, br.data(), n, s));
  CK(w, upload(d.rattler, rat.data(), n, s));
  CK(w, cudaMemsetAsync(d.force, 0, sizeof(double2) * n, s));
  CK(w, cudaMemsetAsync(d.torque, 0, sizeof(double) * n, s));
  CK(w, cudaMemsetAsync(d.ncp, 0, sizeof(int32_t) * n, s));
  w->total_volume = sys_vol[0];
  w->control_mass.assign(nsys, 0.0);
  for (int k = 0; k < nsys; ++k)  // setVirtualBoundaryMass (PeriodicControlWorld.cpp:58-66)
    w->control_mass[k] = sys_mass[k] / ((double)sys[k].count * 10.0);
  // one contact law for the whole world when every non-clump body has one shape
  bool any_circle = false, any_ellipse = false, any_segment = false, any_clump = false;
  for (int i = 0; i < n; ++i) {
    any_circle |= P->shape[i] == XDEM_SHAPE_CIRCLE;
    any_ellipse |= P->shape[i] == XDEM_SHAPE_ELLIPSE;
    any_segment |= P->shape[i] == XDEM_SHAPE_SEGMENT;
    any_clump |= P->shape[i] == XDEM_SHAPE_CLUMP;
  }
  w->has_clumps = any_clump;
  if ((any_circle && any_ellipse) || any_segment) w->law = LAW_ANY;
  else if (any_ellipse)
    w->law = w->prm.ellipse_method == XDEM_ELLIPSE_INTERSECTION ? LAW_INTERSECTION : LAW_CLOSEST;
  else w->law = LAW_CIRCLE;
  // scalars of every system: the single world keeps its current ones; a batch
  // takes the contact model and run settings of the world's and its own box
  // and time step
  WorldScalars tmpl;
  CK(w, read_scalars(w, &tmpl));
  if (nsys != w->nsys) {
    WorldScalars* nws = nullptr;
    CK(w, cudaMalloc(&nws, sizeof(WorldScalars) * nsys));
    cudaFree(w->ws);
    w->ws = nws;
    w->dw.ws = nws;
    w->nsys = nsys;
  }
  d.nsys = nsys;
  std::vector<WorldScalars> all(nsys, tmpl);
  std::vector<int32_t> cell_base(nsys + 1, 0);
  size_t cells = 0;
  for (int k = 0; k < nsys; ++k) {
    WorldScalars& ws = all[k];
    if (nsys > 1) {
      ws.xmin = sys[k].box[0];
      ws.xmax = sys[k].box[1];
      ws.ymin = sys[k].box[2];
      ws.ymax = sys[k].box[3];
      ws.xlen = ws.xmax - ws.xmin;
      ws.ylen = ws.ymax - ws.ymin;
      ws.shift_vel = ws.shift_rate * ws.ylen;
      ws.dt = sys[k].dt;
      ws.shift = ws.strain = ws.velX = ws.velY = 0.0;
      for (int c = 0; c < 4; ++c) ws.stress[c] = 0.0;
      if (!(ws.xlen > 0.0) || !(ws.ylen > 0.0) || !(ws.dt > 0.0)) return XDEM_ERR_ARGUMENT;
    }
    ws.maxsize = w->prm.max_particle_size > 0 ? w->prm.max_particle_size : sys_maxr[k] * 2.01;
    w->base_maxsize.resize(nsys);
    w->base_maxsize[k] = ws.maxsize;
    // grid capacity: twice the starting grid of the base cell size per axis,
    // so a growing box keeps its cell size for a while and then coarsens
    int nx0 = (int)std::floor(ws.xlen / ws.maxsize), ny0 = (int)std::floor(ws.ylen / ws.maxsize);
    ws.nx_cap = std::max(3, 2 * nx0 + 4);
    ws.ny_cap = std::max(3, 2 * ny0 + 4);
    ws.maxsize *= w->cell_factor;
    ws.cell_base = (int32_t)cells;
    ws.first = sys[k].first;
    ws.count = sys[k].count;
    ws.vl_valid = 0;  // the first step builds the candidate lists
    ws.vl_travel = 0.0;
    cell_base[k] = (int32_t)cells;
    cells += (size_t)ws.nx_cap * ws.ny_cap + 2 * (size_t)ws.nx_cap;
    if (cells >= ((size_t)1 << 31) - 2) return XDEM_ERR_ARGUMENT;
  }
  cell_base[nsys] = (int32_t)cells;
  d.ncell_total = (int)cells;
  CK(w, cudaMemcpyAsync(w->ws, all.data(), sizeof(WorldScalars) * nsys, cudaMemcpyHostToDevice, s));
  CK(w, B.alloc(&d.sys_cell_base, nsys + 1));
  CK(w, upload(d.sys_cell_base, cell_base.data(), nsys + 1, s));
  d.sys_of = nullptr;
  if (nsys > 1) {
    // a system keeps its memory range through re-sorts, so sys_of never moves
    CK(w, B.alloc(&d.sys_of, n));
    CK(w, upload(d.sys_of, sys_of.data(), n, s));
  }
  CK(w, B.alloc(&d.cell_count, cells + 1));
  CK(w, B.alloc(&d.cell_max, 1));
  CK(w, cudaMemsetAsync(d.cell_max, 0, sizeof(int32_t), s));
  CK(w, B.alloc(&d.cell_start, cells + 1));
  CK(w, B.alloc(&d.tile_sum, cells / kScanTile + 2));
  CK(w, B.alloc(&d.done, 4));
  CK(w, cudaMemsetAsync(d.done, 0, 4 * sizeof(uint32_t), s));
  CK(w, B.alloc(&d.cell_mem, 2 * (size_t)n));
  CK(w, B.alloc(&d.cell_pos, 2 * (size_t)n));
  CK(w, B.alloc(&d.cell_scr, 2 * (size_t)n));
  CK(w, B.alloc(&d.cell_up, 2 * (size_t)n));
  CK(w, B.alloc(&d.body, n));
  // the centre-line screen's axis records (mixed precision only)
  d.axis = nullptr;
  if (w->prm.precision == XDEM_PRECISION_MIXED) CK(w, B.alloc(&d.axis, n));
  d.screen_r = w->law == LAW_CIRCLE ? d.rad : d.orad;
  // wall segments: vertices by id (their screening radius follows from the
  // vertices and the position, screen_radius in kernels.cuh)
  d.seg = nullptr;
  if (any_segment) {
    std::vector<double4> sv(n, double4{0.0, 0.0, 0.0, 0.0});
    for (int i = 0; i < n; ++i)
      if (P->shape[i] == XDEM_SHAPE_SEGMENT)
        sv[i] = double4{P->seg_x1[i], P->seg_y1[i], P->seg_x2[i], P->seg_y2[i]};
    CK(w, B.alloc(&d.seg, n));
    CK(w, upload(d.seg, sv.data(), n, s));
  }
  CK(w, B.alloc(&d.pcell, n));
  CK(w, B.alloc(&d.prank, n));
  CK(w, B.alloc(&d.gcell, n));
  CK(w, B.alloc(&d.grank, n));
  CK(w, cudaMemsetAsync(d.cell_count, 0, sizeof(int32_t) * (cells + 1), s));
  size_t ks = (size_t)K * n;
  for (int b = 0; b < 2; ++b) {
    Slots& S = d.slots[b];
    CK(w, B.alloc(&S.count, n));
    CK(w, B.alloc(&S.base, n));
    CK(w, B.alloc(&S.partner, ks));
    CK(w, B.alloc(&S.n, ks));
    CK(w, B.alloc(&S.s, ks));
    CK(w, B.alloc(&S.damp, ks));
    CK(w, B.alloc(&S.f, ks));
    CK(w, B.alloc(&S.t1, ks));
    CK(w, B.alloc(&S.t2, ks));
    CK(w, B.alloc(&S.b, ks));
    CK(w, B.alloc(&S.cp, ks));
    CK(w, B.alloc(&S.bv1, ks));
    CK(w, B.alloc(&S.bv2, ks));
    CK(w, B.alloc(&S.fn, ks));
    CK(w, B.alloc(&S.ft, ks));
    CK(w, cudaMemsetAsync(S.count, 0, sizeof(int32_t) * n, s));
    CK(w, cudaMemsetAsync(S.base, 0, sizeof(int32_t) * n, s));
  }
  CK(w, B.alloc(&d.incnt, n));
  CK(w, B.alloc(&d.inref, ks));
  CK(w, cudaMemsetAsync(d.incnt, 0, sizeof(int32_t) * n, s));
  CK(w, B.alloc(&d.pairs, ks));
  // the pair and deep-pair counts are the low and high halves of one 64-bit
  // word, so that a warp reserves room in both lists with one atomic
  CK(w, B.alloc(&d.pair_counts, 1));
  CK(w, cudaMemsetAsync(d.pair_counts, 0, sizeof(unsigned long long), s));
  d.npairs = reinterpret_cast<int32_t*>(d.pair_counts);
  d.ndeep = d.npairs + 1;
  CK(w, B.alloc(&d.fallback, w->prm.precision == XDEM_PRECISION_MIXED ? ks : 1));
  CK(w, B.alloc(&d.nfallback, 1));
  CK(w, cudaMemsetAsync(d.nfallback, 0, sizeof(int32_t), s));
  CK(w, B.alloc(&d.deep, w->prm.precision == XDEM_PRECISION_MIXED ? ks : 1));
  d.warm = nullptr;
  if (w->mlp) CK(w, B.alloc(&d.warm, ks));
  // candidate lists: rebuilt by the first step (vl_valid starts at 0)
  d.V = w->vl_capacity;
  {
    double smallest = 1e300;
    for (double b : w->base_maxsize) smallest = std::min(smallest, b);
    d.skin = w->skin_fraction * smallest;
  }
  d.vl = nullptr;
  d.vl_cnt = nullptr;
  d.vl_disp = nullptr;
  d.vl_part = nullptr;
  if (d.V > 0) {
    CK(w, B.alloc(&d.vl, (size_t)d.V * n));
    CK(w, B.alloc(&d.vl_cnt, n));
    CK(w, B.alloc(&d.vl_disp, n));
    CK(w, B.alloc(&d.vl_part, (size_t)blocks_for(n, kVlBlock) + 1));
    CK(w, cudaMemsetAsync(d.vl_cnt, 0, sizeof(int32_t) * n, s));
    CK(w, cudaMemsetAsync(d.vl_disp, 0, sizeof(double) * n, s));
  }
  w->partial_blocks = blocks_for(n, kReduceBlock);
  CK(w, B.alloc(&d.partials, 4 * (size_t)w->partial_blocks + 4));
  // memory order starts as id order
  std::vector<int32_t> ident(n);
  for (int i = 0; i < n; ++i) ident[i] = i;
  CK(w, B.alloc(&d.id_of, n));
  CK(w, B.alloc(&d.mpos, n));
  CK(w, B.alloc(&d.newpos, n));
  CK(w, B.alloc(&d.stage, 6 * (size_t)n));
  CK(w, upload(d.id_of, ident.data(), n, s));
  CK(w, upload(d.mpos, ident.data(), n, s));
  // arrays moved by a re-sort, each with a slab of the scratch buffer
  PermList& L = w->perm;
  L = PermList{};
  auto add = [&](void* p, int esize) {
    if (L.count >= kMaxPermArrays) return;  // sized for the arrays listed below
    L.base[L.count] = p;
    L.esize[L.count] = esize;
    L.count++;
  };
  add(d.id_of, 4);
  add(shape, 4);
  add(up, 4);
  add(setting, 4);
  add(num_sub, 4);
  add(d.rattler, 4);
  add(d.ncp, 4);
  add(orad, 8);
  add(rad, 8);
  add(asp, 8);
  add(mass, 8);
  add(im, 8);
  add(I, 8);
  add(iI, 8);
  add(vol, 8);
  add(d.rot, 8);
  add(d.w, 8);
  add(d.torque, 8);
  add(d.pos, 16);
  add(d.vel, 16);
  add(d.branch, 16);
  add(d.force, 16);
  add(d.pcell, 4);  // read by the candidate scan's history test after a re-sort
  add(d.gcell, 4);
  if (d.axis) add(d.axis, 16);  // written by k_scatter before the re-sort
  size_t off = 0;
  for (int a = 0; a < L.count; ++a) {
    L.offset[a] = off;
    off += (size_t)L.esize[a] * n;
    off = (off + 255) & ~(size_t)255;
  }
  CK(w, B.alloc(&d.scratch, off));
  w->par = 0;
  w->since_resort = kResortDue;
  CK(w, cudaStreamSynchronize(s));
  return XDEM_OK;
}

}  // namespace

extern "C" {

int32_t xdem_set_particles(xdem_world w, const xdem_particles* P) {
  if (!w || !P || P->n <= 0) return XDEM_ERR_ARGUMENT;
  std::vector<SysDesc> sys(1);
  sys[0].first = 0;
  sys[0].count = P->n;
  return set_particles_impl(w, P, sys);
}

// ---- batched systems ------------------------------------------------------------
int32_t xdem_batch_set_particles(xdem_world w, int32_t nsys, const xdem_particles* systems,
                                 const double* boxes, const double* dts) {
  if (!w || nsys <= 0 || !systems || !boxes) return XDEM_ERR_ARGUMENT;
  std::vector<SysDesc> sys(nsys);
  int64_t total = 0;
  for (int k = 0; k < nsys; ++k) {
    const xdem_particles& Q = systems[k];
    if (Q.n <= 0 || !Q.shape || !Q.up_level || !Q.setting || !Q.outer_radius || !Q.radius ||
        !Q.aspect_ratio || !Q.x || !Q.y || !Q.vx || !Q.vy || !Q.rot || !Q.rot_vel || !Q.volume ||
        !Q.mass || !Q.inv_mass || !Q.inertia || !Q.inv_inertia)
      return XDEM_ERR_ARGUMENT;
    sys[k].first = (int)total;
    sys[k].count = Q.n;
    for (int c = 0; c < 4; ++c) sys[k].box[c] = boxes[4 * k + c];
    sys[k].dt = dts ? dts[k] : w->prm.dt;
    total += Q.n;
  }
  if (total >= ((int64_t)1 << 31) / kMaxSlots) return XDEM_ERR_ARGUMENT;
  const int n = (int)total;
  // the concatenation, ids made global
  std::vector<int32_t> shape(n), up(n), setting(n), rattler(n, 0), num_sub(n, 0);
  std::vector<double> orad(n), rad(n), asp(n), x(n), y(n), vx(n), vy(n), rot(n), rv(n), vol(n),
      mass(n), im(n), I(n), iI(n), bx(n, 0.0), by(n, 0.0);
  bool clumps = false, rattlers = false;
  for (int k = 0; k < nsys; ++k) {
    const xdem_particles& Q = systems[k];
    const int f = sys[k].first;
    for (int i = 0; i < Q.n; ++i) {
      const int g = f + i;
      shape[g] = Q.shape[i];
      if (Q.up_level[i] < 0 || Q.up_level[i] >= Q.n) return XDEM_ERR_ARGUMENT;
      up[g] = f + Q.up_level[i];
      setting[g] = Q.setting[i];
      if (Q.is_rattler) {
        rattler[g] = Q.is_rattler[i];
        rattlers = true;
      }
      if (Q.num_sub) {
        num_sub[g] = Q.num_sub[i];
        clumps = true;
      }
      orad[g] = Q.outer_radius[i];
      rad[g] = Q.radius[i];
      asp[g] = Q.aspect_ratio[i];
      x[g] = Q.x[i];
      y[g] = Q.y[i];
      vx[g] = Q.vx[i];
      vy[g] = Q.vy[i];
      rot[g] = Q.rot[i];
      rv[g] = Q.rot_vel[i];
      vol[g] = Q.volume[i];
      mass[g] = Q.mass[i];
      im[g] = Q.inv_mass[i];
      I[g] = Q.inertia[i];
      iI[g] = Q.inv_inertia[i];
      if (Q.branch_x) bx[g] = Q.branch_x[i];
      if (Q.branch_y) by[g] = Q.branch_y[i];
    }
  }
  xdem_particles P{};
  P.n = n;
  P.shape = shape.data();
  P.up_level = up.data();
  P.setting = setting.data();
  P.is_rattler = rattlers ? rattler.data() : nullptr;
  P.outer_radius = orad.data();
  P.radius = rad.data();
  P.aspect_ratio = asp.data();
  P.x = x.data();
  P.y = y.data();
  P.vx = vx.data();
  P.vy = vy.data();
  P.rot = rot.data();
  P.rot_vel = rv.data();
  P.volume = vol.data();
  P.mass = mass.data();
  P.inv_mass = im.data();
  P.inertia = I.data();
  P.inv_inertia = iI.data();
  P.num_sub = clumps ? num_sub.data() : nullptr;
  P.branch_x = clumps ? bx.data() : nullptr;
  P.branch_y = clumps ? by.data() : nullptr;
  return set_particles_impl(w, &P, sys);
}

int32_t xdem_batch_info(xdem_world w, int32_t* nsys, int32_t* first) {
  if (!w || !nsys) return XDEM_ERR_ARGUMENT;
  *nsys = w->nsys;
  if (first) {
    std::vector<WorldScalars> all(w->nsys);
    CK(w, cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys, cudaMemcpyDeviceToHost,
                          w->stream));
    CK(w, cudaStreamSynchronize(w->stream));
    for (int k = 0; k < w->nsys; ++k) first[k] = all[k].first;
    first[w->nsys] = w->dw.n;
  }
  return XDEM_OK;
}

int32_t xdem_batch_get_stress(xdem_world w, double* stress) {
  if (!w || !stress) return XDEM_ERR_ARGUMENT;
  std::vector<WorldScalars> all(w->nsys);
  CK(w, cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys, cudaMemcpyDeviceToHost,
                        w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  for (int k = 0; k < w->nsys; ++k)
    for (int c = 0; c < 4; ++c) stress[4 * k + c] = all[k].stress[c];
  return XDEM_OK;
}

int32_t xdem_batch_get_boundaries(xdem_world w, double* boxes) {
  if (!w || !boxes) return XDEM_ERR_ARGUMENT;
  std::vector<WorldScalars> all(w->nsys);
  CK(w, cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys, cudaMemcpyDeviceToHost,
                        w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  for (int k = 0; k < w->nsys; ++k) {
    boxes[4 * k + 0] = all[k].xmin;
    boxes[4 * k + 1] = all[k].xmax;
    boxes[4 * k + 2] = all[k].ymin;
    boxes[4 * k + 3] = all[k].ymax;
  }
  return XDEM_OK;
}

int32_t xdem_batch_count_contacts(xdem_world w, int64_t* counts) {
  if (!w || !counts || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n, K = w->dw.K;
  std::vector<WorldScalars> all(w->nsys);
  std::vector<int32_t> cnt(n), base(n), partner((size_t)K * n);
  CK(w, cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys, cudaMemcpyDeviceToHost,
                        w->stream));
  CK(w, download(cnt.data(), w->dw.slots[w->par].count, n, w->stream));
  CK(w, download(base.data(), w->dw.slots[w->par].base, n, w->stream));
  CK(w, download(partner.data(), w->dw.slots[w->par].partner, (size_t)K * n, w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  // a system's particles keep its memory range [first, first + count)
  for (int k = 0; k < w->nsys; ++k) {
    int64_t t = 0;
    for (int m = all[k].first; m < all[k].first + all[k].count; ++m)
      for (int s = 0; s < std::min(cnt[m], K); ++s) t += partner[(size_t)base[m] + s] >= 0;
    counts[k] = t;
  }
  return XDEM_OK;
}


int32_t xdem_get_particles(xdem_world w, xdem_particles* P) {
  if (!w || !P || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n;
  const DevWorld& d = w->dw;
  std::vector<int32_t> id_of;
  CK(w, fetch_id_of(w, id_of));
  std::vector<double2> pos(n), vel(n), br(n);
  CK(w, download_by_id(w, pos.data(), d.pos, id_of));
  CK(w, download_by_id(w, vel.data(), d.vel, id_of));
  CK(w, download_by_id(w, br.data(), d.branch, id_of));
  if (P->rot) CK(w, download_by_id(w, P->rot, d.rot, id_of));
  if (P->rot_vel) CK(w, download_by_id(w, P->rot_vel, d.w, id_of));
  if (P->is_rattler) CK(w, download_by_id(w, P->is_rattler, d.rattler, id_of));
  if (P->mass) CK(w, download_by_id(w, P->mass, (const double*)d.mass, id_of));
  if (P->inertia) CK(w, download_by_id(w, P->inertia, (const double*)d.I, id_of));
  if (P->shape) CK(w, download_by_id(w, P->shape, (const int32_t*)d.shape, id_of));
  if (P->setting) CK(w, download_by_id(w, P->setting, (const int32_t*)d.setting, id_of));
  if (P->up_level) CK(w, download_by_id(w, P->up_level, (const int32_t*)d.up, id_of));
  if (P->seg_x1 || P->seg_y1 || P->seg_x2 || P->seg_y2) {
    std::vector<double4> sv(n, double4{0.0, 0.0, 0.0, 0.0});
    if (d.seg) {
      CK(w, download(sv.data(), d.seg, n, w->stream));
      CK(w, cudaStreamSynchronize(w->stream));
    }
    for (int i = 0; i < n; ++i) {
      if (P->seg_x1) P->seg_x1[i] = sv[i].x;
      if (P->seg_y1) P->seg_y1[i] = sv[i].y;
      if (P->seg_x2) P->seg_x2[i] = sv[i].z;
      if (P->seg_y2) P->seg_y2[i] = sv[i].w;
    }
  }
  P->n = n;
  for (int i = 0; i < n; ++i) {
    if (P->x) P->x[i] = pos[i].x;
    if (P->y) P->y[i] = pos[i].y;
    if (P->vx) P->vx[i] = vel[i].x;
    if (P->vy) P->vy[i] = vel[i].y;
    if (P->branch_x) P->branch_x[i] = br[i].x;
    if (P->branch_y) P->branch_y[i] = br[i].y;
  }
  return XDEM_OK;
}

int32_t xdem_set_contacts(xdem_world w, const xdem_contacts* C) {
  if (!w || !C || w->dw.n <= 0 || C->count < 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n, K = w->dw.K;
  const size_t ks = (size_t)K * n;
  std::vector<int32_t> mpos(n);
  CK(w, download(mpos.data(), w->dw.mpos, n, w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  std::vector<int32_t> cnt(n, 0), base(n, 0), fill(n, 0), partner(ks, 0);
  std::vector<double2> nn(ks), sh(ks), f(ks), b(ks), cp(ks), bv1(ks), bv2(ks), fn(ks), ft(ks);
  std::vector<double> damp(ks), t1(ks), t2(ks);
  uint32_t st = 0;
  // records per owner (the first K in input order), then each owner's
  // consecutive records in memory order
  for (int64_t k = 0; k < C->count; ++k) {
    int i = C->id_i[k], j = C->id_j[k];
    if (i < 0 || i >= n || j < 0 || j >= n || i >= j) return XDEM_ERR_ARGUMENT;
    int m = mpos[i];
    if (cnt[m] >= K) {
      st |= XDEM_ERR_CAPACITY;
      continue;
    }
    cnt[m]++;
  }
  for (int m = 1; m < n; ++m) base[m] = base[m - 1] + cnt[m - 1];
  for (int64_t k = 0; k < C->count; ++k) {
    int i = C->id_i[k], j = C->id_j[k];
    int m = mpos[i];
    if (fill[m] >= cnt[m]) continue;
    size_t ci = (size_t)base[m] + fill[m]++;
    partner[ci] = j;
    nn[ci] = make_double2(C->normal_x[k], C->normal_y[k]);
    sh[ci] = make_double2(C->shear_x[k], C->shear_y[k]);
    damp[ci] = C->damping[k];
    double2 Fn = make_double2(C->fn_x[k], C->fn_y[k]);
    double2 Ft = make_double2(C->ft_x[k], C->ft_y[k]);
    f[ci] = make_double2(Fn.x + Ft.x, Fn.y + Ft.y);  // ContactInformation.h:63
    t1[ci] = C->torque_i[k];
    t2[ci] = C->torque_j[k];
    b[ci] = make_double2(C->branch_x[k], C->branch_y[k]);
    cp[ci] = make_double2(C->point_x[k], C->point_y[k]);
    bv1[ci] = make_double2(C->bv1_x[k], C->bv1_y[k]);
    bv2[ci] = make_double2(C->bv2_x[k], C->bv2_y[k]);
    fn[ci] = Fn;
    ft[ci] = Ft;
  }
  // incoming references, so that a collect without an update sums these
  // contacts as the reference would
  std::vector<int32_t> inc(n, 0);
  std::vector<int32_t> id_at(n);
  for (int i = 0; i < n; ++i) id_at[mpos[i]] = i;
  std::vector<uint64_t> inref(ks, 0);
  for (int m = 0; m < n; ++m)
    for (int s = 0; s < cnt[m]; ++s) {
      const size_t ci = (size_t)base[m] + s;
      int mj = mpos[partner[ci]];
      if (inc[mj] < K)
        inref[(size_t)inc[mj] * n + mj] = ((uint64_t)(uint32_t)id_at[m] << 32) | (uint32_t)ci;
      else st |= XDEM_ERR_CAPACITY;
      inc[mj]++;
    }
  const Slots& S = w->dw.slots[w->par];
  cudaStream_t q = w->stream;
  CK(w, upload(S.count, cnt.data(), n, q));
  CK(w, upload(S.base, base.data(), n, q));
  CK(w, upload(S.partner, partner.data(), ks, q));
  CK(w, upload(S.n, nn.data(), ks, q));
  CK(w, upload(S.s, sh.data(), ks, q));
  CK(w, upload(S.damp, damp.data(), ks, q));
  CK(w, upload(S.f, f.data(), ks, q));
  CK(w, upload(S.t1, t1.data(), ks, q));
  CK(w, upload(S.t2, t2.data(), ks, q));
  CK(w, upload(S.b, b.data(), ks, q));
  CK(w, upload(S.cp, cp.data(), ks, q));
  CK(w, upload(S.bv1, bv1.data(), ks, q));
  CK(w, upload(S.bv2, bv2.data(), ks, q));
  CK(w, upload(S.fn, fn.data(), ks, q));
  CK(w, upload(S.ft, ft.data(), ks, q));
  for (int i = 0; i < n; ++i) inc[i] = std::min(inc[i], K);
  CK(w, upload(w->dw.incnt, inc.data(), n, q));
  CK(w, upload(w->dw.inref, inref.data(), ks, q));
  CK(w, cudaStreamSynchronize(q));
  return (int32_t)st;
}

int32_t xdem_get_contacts(xdem_world w, xdem_contacts* C) {
  if (!w || !C || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n, K = w->dw.K;
  const size_t ks = (size_t)K * n;
  const Slots& S = w->dw.slots[w->par];
  cudaStream_t q = w->stream;
  std::vector<int32_t> cnt(n), base(n), partner(ks), id_of(n), mpos(n);
  CK(w, download(cnt.data(), S.count, n, q));
  CK(w, download(base.data(), S.base, n, q));
  CK(w, download(partner.data(), S.partner, ks, q));
  CK(w, download(id_of.data(), w->dw.id_of, n, q));
  CK(w, download(mpos.data(), w->dw.mpos, n, q));
  CK(w, cudaStreamSynchronize(q));
  int64_t total = 0;
  for (int m = 0; m < n; ++m)
    for (int s = 0; s < std::min(cnt[m], K); ++s) total += partner[(size_t)base[m] + s] >= 0;
  C->count = total;
  if (C->capacity < total) return XDEM_ERR_CAPACITY;
  std::vector<double2> nn(ks), sh(ks), b(ks), cp(ks), bv1(ks), bv2(ks), fn(ks), ft(ks);
  std::vector<double> damp(ks), t1(ks), t2(ks);
  CK(w, download(nn.data(), S.n, ks, q));
  CK(w, download(sh.data(), S.s, ks, q));
  CK(w, download(b.data(), S.b, ks, q));
  CK(w, download(cp.data(), S.cp, ks, q));
  CK(w, download(bv1.data(), S.bv1, ks, q));
  CK(w, download(bv2.data(), S.bv2, ks, q));
  CK(w, download(fn.data(), S.fn, ks, q));
  CK(w, download(ft.data(), S.ft, ks, q));
  CK(w, download(damp.data(), S.damp, ks, q));
  CK(w, download(t1.data(), S.t1, ks, q));
  CK(w, download(t2.data(), S.t2, ks, q));
  CK(w, cudaStreamSynchronize(q));
  int64_t k = 0;
  std::vector<std::pair<int32_t, int32_t>> order;
  for (int i = 0; i < n; ++i) {  // owners in id order
    const int m = mpos[i];
    const int c = std::min(cnt[m], K);
    order.clear();
    for (int s = 0; s < c; ++s)
      if (partner[(size_t)base[m] + s] >= 0) order.push_back({partner[(size_t)base[m] + s], s});
    std::sort(order.begin(), order.end());
    for (auto& o : order) {
      size_t ci = (size_t)base[m] + o.second;
      C->id_i[k] = i;
      C->id_j[k] = o.first;
      C->normal_x[k] = nn[ci].x;
      C->normal_y[k] = nn[ci].y;
      C->point_x[k] = cp[ci].x;
      C->point_y[k] = cp[ci].y;
      C->branch_x[k] = b[ci].x;
      C->branch_y[k] = b[ci].y;
      C->bv1_x[k] = bv1[ci].x;
      C->bv1_y[k] = bv1[ci].y;
      C->bv2_x[k] = bv2[ci].x;
      C->bv2_y[k] = bv2[ci].y;
      C->shear_x[k] = sh[ci].x;
      C->shear_y[k] = sh[ci].y;
      C->fn_x[k] = fn[ci].x;
      C->fn_y[k] = fn[ci].y;
      C->ft_x[k] = ft[ci].x;
      C->ft_y[k] = ft[ci].y;
      C->torque_i[k] = t1[ci];
      C->torque_j[k] = t2[ci];
      C->damping[k] = damp[ci];
      ++k;
    }
  }
  (void)id_of;
  return XDEM_OK;
}

int32_t xdem_get_force_and_torque(xdem_world w, double* fx, double* fy, double* t, int32_t* nc) {
  if (!w || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n;
  std::vector<int32_t> id_of;
  CK(w, fetch_id_of(w, id_of));
  std::vector<double2> f(n);
  CK(w, download_by_id(w, f.data(), w->dw.force, id_of));
  if (t) CK(w, download_by_id(w, t, w->dw.torque, id_of));
  if (nc) CK(w, download_by_id(w, nc, w->dw.ncp, id_of));
  for (int i = 0; i < n; ++i) {
    if (fx) fx[i] = f[i].x;
    if (fy) fy[i] = f[i].y;
  }
  return XDEM_OK;
}

int32_t xdem_count_contacts(xdem_world w, int64_t* out) {
  if (!w || !out || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n, K = w->dw.K;
  std::vector<int32_t> cnt(n), base(n), partner((size_t)K * n);
  CK(w, download(cnt.data(), w->dw.slots[w->par].count, n, w->stream));
  CK(w, download(base.data(), w->dw.slots[w->par].base, n, w->stream));
  CK(w, download(partner.data(), w->dw.slots[w->par].partner, (size_t)K * n, w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  int64_t t = 0;
  for (int m = 0; m < n; ++m)
    for (int s = 0; s < std::min(cnt[m], K); ++s) t += partner[(size_t)base[m] + s] >= 0;
  *out = t;
  return XDEM_OK;
}

// ---- world scalars -------------------------------------------------------
int32_t xdem_get_boundary(xdem_world w, double box[4]) {
  if (!w || !box) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  box[0] = s.xmin;
  box[1] = s.xmax;
  box[2] = s.ymin;
  box[3] = s.ymax;
  return XDEM_OK;
}

int32_t xdem_set_boundary(xdem_world w, const double box[4]) {
  if (!w || !box || w->nsys > 1) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  s.xmin = box[0];
  s.xmax = box[1];
  s.ymin = box[2];
  s.ymax = box[3];
  s.xlen = s.xmax - s.xmin;
  s.ylen = s.ymax - s.ymin;
  s.vl_valid = 0;  // the candidate lists are rebuilt by the next step
  CK(w, write_scalars(w, &s));
  return XDEM_OK;
}

int32_t xdem_get_stress(xdem_world w, double stress[4]) {
  if (!w || !stress) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  for (int c = 0; c < 4; ++c) stress[c] = s.stress[c];
  return XDEM_OK;
}

int32_t xdem_get_lees_edwards(xdem_world w, double out[4]) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  out[0] = s.shift;
  out[1] = s.shift_vel;
  out[2] = s.strain;
  out[3] = s.shift_rate;
  return XDEM_OK;
}

int32_t xdem_set_lees_edwards(xdem_world w, const double in[4]) {
  if (!w || !in || w->nsys > 1) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  s.shift = in[0];
  s.shift_vel = in[1];
  s.strain = in[2];
  s.shift_rate = in[3];
  s.vl_valid = 0;
  CK(w, write_scalars(w, &s));
  return XDEM_OK;
}

int32_t xdem_set_shift_strain_rate(xdem_world w, double rate) {
  if (!w) return XDEM_ERR_ARGUMENT;
  CK(w, modify_all(w, [&](WorldScalars& s, int) {
       s.shift_rate = rate;
       s.shift_vel = rate * s.ylen;
     }));
  return XDEM_OK;
}

int32_t xdem_set_time_increment(xdem_world w, double dt) {
  if (!w || !(dt > 0.0)) return XDEM_ERR_ARGUMENT;
  w->prm.dt = dt;
  CK(w, modify_all(w, [&](WorldScalars& s, int) { s.dt = dt; }));
  return XDEM_OK;
}

int32_t xdem_set_global_damping(xdem_world w, double g) {
  if (!w) return XDEM_ERR_ARGUMENT;
  CK(w, modify_all(w, [&](WorldScalars& s, int) { s.g = g; }));
  return XDEM_OK;
}

int32_t xdem_set_contact_model(xdem_world w, double kn, double kt, double e, double mu) {
  if (!w) return XDEM_ERR_ARGUMENT;
  const double factor = factor_of(kn, e);
  CK(w, modify_all(w, [&](WorldScalars& s, int) {
       s.kn = kn;
       s.kt = kt;
       s.mu = mu;
       s.factor = factor;
     }));
  return XDEM_OK;
}

int32_t xdem_set_virtual_boundary_mass(xdem_world w, double mass) {
  if (!w) return XDEM_ERR_ARGUMENT;
  CK(w, modify_all(w, [&](WorldScalars& s, int k) {
       s.vmass = mass >= 0 ? mass : w->control_mass[k];
     }));
  return XDEM_OK;
}

int32_t xdem_set_max_strain_rate(xdem_world w, double r) {
  if (!w) return XDEM_ERR_ARGUMENT;
  CK(w, modify_all(w, [&](WorldScalars& s, int) { s.max_strain_rate = r; }));
  return XDEM_OK;
}

int32_t xdem_get_newton_stats(xdem_world w, int64_t out[3]) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  out[0] = (int64_t)s.newton_solves;
  out[1] = (int64_t)s.newton_iters;
  out[2] = (int64_t)s.newton_capped;
  return XDEM_OK;
}

int32_t xdem_get_pair_count(xdem_world w, int64_t* out) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  *out = s.last_pairs;
  return XDEM_OK;
}

int32_t xdem_reset_newton_stats(xdem_world w) {
  if (!w) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  s.newton_solves = s.newton_iters = s.newton_capped = 0;
  s.vl_builds = 0;
  s.warm_offered = s.warm_used = s.warm_rejected = s.warm_restarted = s.logit_right = 0;
  CK(w, write_scalars(w, &s));
  return XDEM_OK;
}

// ---- learned warm start ------------------------------------------------------
int32_t xdem_set_warm_start(xdem_world w, xdem_mlp m) {
  if (!w) return XDEM_ERR_ARGUMENT;
  cudaStreamSynchronize(w->stream);
  w->mlp = m;
  if (m && w->dw.n > 0 && !w->dw.warm)
    CK(w, w->particle_bufs.alloc(&w->dw.warm, (size_t)w->dw.K * w->dw.n));
  if (!m) w->dw.warm = nullptr;
  return XDEM_OK;
}

int32_t xdem_get_warm_stats(xdem_world w, int64_t out[5]) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  out[0] = (int64_t)s.warm_offered;
  out[1] = (int64_t)s.warm_used;
  out[2] = (int64_t)s.warm_rejected;
  out[3] = (int64_t)s.warm_restarted;
  out[4] = (int64_t)s.logit_right;
  return XDEM_OK;
}

// ---- binary snapshots ---------------------------------------------------------------
}  // extern "C"
namespace {

// file layout (native byte order): SnapHeader, nsys WorldScalars, the
// particles in id order (5 int32 arrays, then 16 double arrays), the memory
// order (the id at each memory position), the wall-segment vertices when
// has_seg (4 double arrays by id), the contacts (id_i, id_j, then 19 double
// arrays, in xdem_contacts field order).  The memory order and the
// steps since the last re-sort come along because block sums (the stress)
// run in memory order: with both restored, a loaded world repeats the saved
// one bit for bit.
struct SnapHeader {
  char magic[8];
  uint32_t version, nsys;
  int32_t n, K;
  int64_t ncontacts;
  uint32_t scalars_bytes, params_bytes;
  int32_t since_resort, has_seg;
  xdem_params prm;
};
constexpr char kSnapMagic[8] = {'X', 'D', 'E', 'M', 'S', 'N', 'P', '1'};

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

template <class T>
bool put(FILE* f, const T* p, size_t count) {
  return fwrite(p, sizeof(T), count, f) == count;
}
template <class T>
bool get(FILE* f, T* p, size_t count) {
  return fread(p, sizeof(T), count, f) == count;
}

// a device array in memory order, downloaded in id order
template <class T>
cudaError_t by_id(xdem_world_s* w, const T* src, const std::vector<int32_t>& id_of, std::vector<T>& out) {
  out.resize(w->dw.n);
  return download_by_id(w, out.data(), src, id_of);
}

// A snapshot file read into host memory and checked in full before any of
// it reaches the device: the header's sizes against the file's length, the
// systems (in order, each non-empty, together covering ids [0, n) with no gap
// or overlap), and the saved memory order (a permutation that keeps every
// system in its own id range).  Any failure is XDEM_ERR_ARGUMENT.
struct SnapData {
  SnapHeader h{};
  std::vector<WorldScalars> all;
  std::vector<int32_t> ints[5];
  std::vector<double> dbl[16];
  std::vector<int32_t> mem_id;
  std::vector<double> segv[4];
  std::vector<int32_t> ci, cj;
  std::vector<std::vector<double>> cd;
};

int32_t read_snapshot(const char* path, SnapData& d) {
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) return XDEM_ERR_ARGUMENT;
  if (fseek(fc.f, 0, SEEK_END) != 0) return XDEM_ERR_ARGUMENT;
  const long long fsize = (long long)ftell(fc.f);
  if (fsize < 0 || fseek(fc.f, 0, SEEK_SET) != 0) return XDEM_ERR_ARGUMENT;
  SnapHeader& h = d.h;
  if (!get(fc.f, &h, 1) || std::memcmp(h.magic, kSnapMagic, 8) != 0 || h.version != 1 ||
      h.scalars_bytes != sizeof(WorldScalars) || h.params_bytes != sizeof(xdem_params) ||
      h.n <= 0 || h.nsys == 0 || h.nsys > (uint32_t)h.n || h.ncontacts < 0 ||
      (h.has_seg != 0 && h.has_seg != 1))
    return XDEM_ERR_ARGUMENT;
  const long long n = h.n, nsys = h.nsys, nc = h.ncontacts;
  // the exact length the header implies (checked before anything is sized by it)
  const long long per_particle = 5 * 4 + 16 * 8 + 4 + (h.has_seg ? 4 * 8 : 0);
  if (nc > (fsize / 8)) return XDEM_ERR_ARGUMENT;
  const long long want = (long long)sizeof(SnapHeader) + nsys * (long long)sizeof(WorldScalars) +
                         n * per_particle + nc * (2 * 4 + 19 * 8);
  if (want != fsize) return XDEM_ERR_ARGUMENT;
  d.all.resize(nsys);
  bool ok = get(fc.f, d.all.data(), nsys);
  for (int k = 0; k < 5 && ok; ++k) {
    d.ints[k].resize(n);
    ok = get(fc.f, d.ints[k].data(), n);
  }
  for (int k = 0; k < 16 && ok; ++k) {
    d.dbl[k].resize(n);
    ok = get(fc.f, d.dbl[k].data(), n);
  }
  d.mem_id.resize(n);
  ok = ok && get(fc.f, d.mem_id.data(), n);
  for (int k = 0; k < 4 && ok && h.has_seg; ++k) {
    d.segv[k].resize(n);
    ok = get(fc.f, d.segv[k].data(), n);
  }
  d.ci.resize(nc);
  d.cj.resize(nc);
  d.cd.assign(19, std::vector<double>(nc));
  ok = ok && get(fc.f, d.ci.data(), nc) && get(fc.f, d.cj.data(), nc);
  for (int k = 0; k < 19 && ok; ++k) ok = get(fc.f, d.cd[k].data(), nc);
  if (!ok) return XDEM_ERR_ARGUMENT;
  // systems: consecutive, non-empty, covering [0, n)
  long long next = 0;
  for (long long k = 0; k < nsys; ++k) {
    const WorldScalars& o = d.all[k];
    if (o.first != next || o.count <= 0 || (long long)o.first + o.count > n) return XDEM_ERR_ARGUMENT;
    next = (long long)o.first + o.count;
  }
  if (next != n) return XDEM_ERR_ARGUMENT;
  // memory order: a permutation of each system's id range
  std::vector<char> taken(n, 0);
  for (long long k = 0; k < nsys; ++k) {
    const int lo = d.all[k].first, hi = d.all[k].first + d.all[k].count;
    for (int m = lo; m < hi; ++m) {
      const int id = d.mem_id[m];
      if (id < lo || id >= hi || taken[id]) return XDEM_ERR_ARGUMENT;
      taken[id] = 1;
    }
  }
  // contact ids inside the world (xdem_set_contacts checks the rest)
  for (long long c = 0; c < nc; ++c)
    if (d.ci[c] < 0 || d.ci[c] >= n || d.cj[c] < 0 || d.cj[c] >= n) return XDEM_ERR_ARGUMENT;
  return XDEM_OK;
}

}  // namespace
extern "C" {

int32_t xdem_save_snapshot(xdem_world w, const char* path) {
  if (!w || !path || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n;
  const DevWorld& d = w->dw;
  std::vector<WorldScalars> all(w->nsys);
  CK(w, cudaMemcpyAsync(all.data(), w->ws, sizeof(WorldScalars) * w->nsys, cudaMemcpyDeviceToHost,
                        w->stream));
  CK(w, cudaStreamSynchronize(w->stream));
  std::vector<int32_t> id_of;
  CK(w, fetch_id_of(w, id_of));
  // particles
  std::vector<int32_t> ints[5];
  const int32_t* isrc[5] = {d.shape, d.up, d.setting, d.rattler, d.num_sub};
  for (int k = 0; k < 5; ++k) CK(w, by_id(w, isrc[k], id_of, ints[k]));
  std::vector<double> dbl[16];
  std::vector<double2> v2;
  CK(w, by_id(w, d.pos, id_of, v2));
  dbl[3].resize(n);
  dbl[4].resize(n);
  for (int i = 0; i < n; ++i) {
    dbl[3][i] = v2[i].x;
    dbl[4][i] = v2[i].y;
  }
  CK(w, by_id(w, d.vel, id_of, v2));
  dbl[5].resize(n);
  dbl[6].resize(n);
  for (int i = 0; i < n; ++i) {
    dbl[5][i] = v2[i].x;
    dbl[6][i] = v2[i].y;
  }
  CK(w, by_id(w, d.branch, id_of, v2));
  dbl[14].resize(n);
  dbl[15].resize(n);
  for (int i = 0; i < n; ++i) {
    dbl[14][i] = v2[i].x;
    dbl[15][i] = v2[i].y;
  }
  const double* dsrc[16] = {d.orad, d.rad, d.asp, nullptr, nullptr, nullptr, nullptr, d.rot,
                            d.w,    d.vol, d.mass, d.im,   d.I,     d.iI,    nullptr, nullptr};
  for (int k = 0; k < 16; ++k)
    if (dsrc[k]) CK(w, by_id(w, dsrc[k], id_of, dbl[k]));
  // contacts
  xdem_contacts c{};
  c.capacity = 0;
  int32_t st = xdem_get_contacts(w, &c);
  if (st && st != XDEM_ERR_CAPACITY) return st;
  const int64_t nc = c.count;
  std::vector<int32_t> ci(nc), cj(nc);
  std::vector<std::vector<double>> cd(19, std::vector<double>(nc));
  c.capacity = nc;
  c.id_i = ci.data();
  c.id_j = cj.data();
  double** fields[19] = {&c.normal_x, &c.normal_y, &c.point_x, &c.point_y, &c.branch_x,
                         &c.branch_y, &c.bv1_x,    &c.bv1_y,   &c.bv2_x,   &c.bv2_y,
                         &c.shear_x,  &c.shear_y,  &c.fn_x,    &c.fn_y,    &c.ft_x,
                         &c.ft_y,     &c.torque_i, &c.torque_j, &c.damping};
  for (int k = 0; k < 19; ++k) *fields[k] = cd[k].data();
  if (nc > 0) {
    st = xdem_get_contacts(w, &c);
    if (st) return st;
  }
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) return XDEM_ERR_ARGUMENT;
  SnapHeader h{};
  std::memcpy(h.magic, kSnapMagic, 8);
  h.version = 1;
  h.nsys = (uint32_t)w->nsys;
  h.n = n;
  h.K = d.K;
  h.ncontacts = nc;
  h.scalars_bytes = sizeof(WorldScalars);
  h.params_bytes = sizeof(xdem_params);
  h.since_resort = w->since_resort;
  h.has_seg = d.seg ? 1 : 0;
  h.prm = w->prm;
  std::vector<double> segv[4];
  if (d.seg) {
    std::vector<double4> sv(n);
    CK(w, download(sv.data(), d.seg, n, w->stream));
    CK(w, cudaStreamSynchronize(w->stream));
    for (int k = 0; k < 4; ++k) segv[k].resize(n);
    for (int i = 0; i < n; ++i) {
      segv[0][i] = sv[i].x;
      segv[1][i] = sv[i].y;
      segv[2][i] = sv[i].z;
      segv[3][i] = sv[i].w;
    }
  }
  bool ok = put(fc.f, &h, 1) && put(fc.f, all.data(), all.size());
  for (int k = 0; k < 5 && ok; ++k) ok = put(fc.f, ints[k].data(), n);
  for (int k = 0; k < 16 && ok; ++k) ok = put(fc.f, dbl[k].data(), n);
  ok = ok && put(fc.f, id_of.data(), n);
  for (int k = 0; k < 4 && ok && h.has_seg; ++k) ok = put(fc.f, segv[k].data(), n);
  ok = ok && put(fc.f, ci.data(), nc) && put(fc.f, cj.data(), nc);
  for (int k = 0; k < 19 && ok; ++k) ok = put(fc.f, cd[k].data(), nc);
  return ok ? XDEM_OK : XDEM_ERR_ARGUMENT;
}

int32_t xdem_load_snapshot(xdem_world w, const char* path) {
  if (!w || !path) return XDEM_ERR_ARGUMENT;
  SnapData sd;
  if (int32_t e = read_snapshot(path, sd)) return e;
  SnapHeader& h = sd.h;
  if (h.prm.world_kind != w->prm.world_kind) return XDEM_ERR_ARGUMENT;
  const int n = h.n;
  const int nsys = (int)h.nsys;
  std::vector<WorldScalars>& all = sd.all;
  std::vector<int32_t>* ints = sd.ints;
  std::vector<double>* dbl = sd.dbl;
  std::vector<int32_t>& mem_id = sd.mem_id;
  std::vector<double>* segv = sd.segv;
  const int64_t nc = h.ncontacts;
  std::vector<int32_t>& ci = sd.ci;
  std::vector<int32_t>& cj = sd.cj;
  std::vector<std::vector<double>>& cd = sd.cd;
  // the particles (the snapshot's contact-model and run settings are restored
  // below; its precision, ellipse law and slot count are the world's own)
  w->prm.dt = h.prm.dt;
  xdem_particles P{};
  P.n = n;
  P.shape = ints[0].data();
  P.up_level = ints[1].data();
  P.setting = ints[2].data();
  P.is_rattler = ints[3].data();
  P.num_sub = ints[4].data();
  P.outer_radius = dbl[0].data();
  P.radius = dbl[1].data();
  P.aspect_ratio = dbl[2].data();
  P.x = dbl[3].data();
  P.y = dbl[4].data();
  P.vx = dbl[5].data();
  P.vy = dbl[6].data();
  P.rot = dbl[7].data();
  P.rot_vel = dbl[8].data();
  P.volume = dbl[9].data();
  P.mass = dbl[10].data();
  P.inv_mass = dbl[11].data();
  P.inertia = dbl[12].data();
  P.inv_inertia = dbl[13].data();
  P.branch_x = dbl[14].data();
  P.branch_y = dbl[15].data();
  if (h.has_seg) {
    P.seg_x1 = segv[0].data();
    P.seg_y1 = segv[1].data();
    P.seg_x2 = segv[2].data();
    P.seg_y2 = segv[3].data();
  }
  std::vector<SysDesc> sys(nsys);
  for (int k = 0; k < nsys; ++k) {
    sys[k].first = all[k].first;
    sys[k].count = all[k].count;
    sys[k].box[0] = all[k].xmin;
    sys[k].box[1] = all[k].xmax;
    sys[k].box[2] = all[k].ymin;
    sys[k].box[3] = all[k].ymax;
    sys[k].dt = all[k].dt;
  }
  // the memory order (read_snapshot checked it is a permutation keeping
  // every system in its id range)
  std::vector<int32_t> newpos(n, -1);
  for (int m = 0; m < n; ++m) newpos[mem_id[m]] = m;
  int32_t st = set_particles_impl(w, &P, sys);
  if (st) return st;
  // set_particles leaves memory order = id order: move every particle array
  // to the saved order (the history is uploaded afterwards, into that order)
  CK(w, upload(w->dw.newpos, newpos.data(), n, w->stream));
  k_permute<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, w->perm);
  CK(w, cudaGetLastError());
  k_copy_back<<<blocks_for(n, kBlock), kBlock, 0, w->stream>>>(w->dw, w->perm);
  CK(w, cudaGetLastError());
  w->since_resort = std::max(0, std::min(h.since_resort, kResortDue));
  // the world scalars of every system: box, time step, contact model,
  // Lees-Edwards and box-law state, the last stress
  CK(w, modify_all(w, [&](WorldScalars& s, int k) {
       const WorldScalars& o = all[k];
       s.xmin = o.xmin;
       s.xmax = o.xmax;
       s.ymin = o.ymin;
       s.ymax = o.ymax;
       s.xlen = o.xlen;
       s.ylen = o.ylen;
       s.shift = o.shift;
       s.shift_vel = o.shift_vel;
       s.strain = o.strain;
       s.shift_rate = o.shift_rate;
       s.velX = o.velX;
       s.velY = o.velY;
       s.vmass = o.vmass;
       s.max_strain_rate = o.max_strain_rate;
       for (int c = 0; c < 4; ++c) s.stress[c] = o.stress[c];
       s.scale_x = o.scale_x;
       s.scale_y = o.scale_y;
       s.ke = o.ke;
       s.dt = o.dt;
       s.g = o.g;
       s.kn = o.kn;
       s.kt = o.kt;
       s.mu = o.mu;
       s.factor = o.factor;
     }));
  if (nc > 0) {
    xdem_contacts c{};
    c.count = nc;
    c.capacity = nc;
    c.id_i = ci.data();
    c.id_j = cj.data();
    double** fields[19] = {&c.normal_x, &c.normal_y, &c.point_x, &c.point_y, &c.branch_x,
                           &c.branch_y, &c.bv1_x,    &c.bv1_y,   &c.bv2_x,   &c.bv2_y,
                           &c.shear_x,  &c.shear_y,  &c.fn_x,    &c.fn_y,    &c.ft_x,
                           &c.ft_y,     &c.torque_i, &c.torque_j, &c.damping};
    for (int k = 0; k < 19; ++k) *fields[k] = cd[k].data();
    st = xdem_set_contacts(w, &c);
    if (st) return st;
  }
  return XDEM_OK;
}

int32_t xdem_snapshot_info(const char* path, int64_t out[4]) {
  if (!path || !out) return XDEM_ERR_ARGUMENT;
  SnapData sd;
  if (int32_t e = read_snapshot(path, sd)) return e;
  out[0] = sd.h.n;
  out[1] = sd.h.nsys;
  out[2] = sd.h.ncontacts;
  out[3] = sd.h.prm.world_kind;
  return XDEM_OK;
}

int32_t xdem_snapshot_layout(int64_t out[4]) {
  if (!out) return XDEM_ERR_ARGUMENT;
  out[0] = (int64_t)sizeof(SnapHeader);
  out[1] = (int64_t)sizeof(WorldScalars);
  out[2] = (int64_t)offsetof(WorldScalars, first);
  out[3] = (int64_t)offsetof(WorldScalars, count);
  return XDEM_OK;
}

// ---- rattler-free coordination number and solid fraction --------------------------
namespace {
int32_t core_z_phi(xdem_world_s* w, std::vector<double>& res) {
  const int n = w->dw.n, K = w->dw.K;
  const int nsys = w->nsys;
  int32_t *deg = nullptr, *changed = nullptr;
  uint8_t *active = nullptr, *leave = nullptr, *eact = nullptr;
  double* out = nullptr;
  cudaStream_t s = w->stream;
  cudaError_t e = cudaMalloc(&deg, sizeof(int32_t) * n);
  if (e == cudaSuccess) e = cudaMalloc(&changed, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&active, n);
  if (e == cudaSuccess) e = cudaMalloc(&leave, n);
  if (e == cudaSuccess) e = cudaMalloc(&eact, (size_t)K * n);
  if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double) * 3 * nsys);
  const int nb = blocks_for(n, kBlock);
  if (e == cudaSuccess) e = cudaMemsetAsync(deg, 0, sizeof(int32_t) * n, s);
  if (e == cudaSuccess) {
    k_core_init<<<nb, kBlock, 0, s>>>(w->dw, w->par, deg, eact);
    k_core_active<<<nb, kBlock, 0, s>>>(w->dw, deg, active);
    e = cudaGetLastError();
  }
  // parallel rounds until no particle leaves (at most n rounds)
  for (int round = 0; round <= n && e == cudaSuccess; ++round) {
    int32_t h = 0;
    e = cudaMemsetAsync(changed, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) break;
    k_core_mark<<<nb, kBlock, 0, s>>>(w->dw, deg, active, leave, changed);
    k_core_edges<<<nb, kBlock, 0, s>>>(w->dw, w->par, deg, leave, eact);
    e = cudaMemcpyAsync(&h, changed, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (h == 0) break;
  }
  if (e == cudaSuccess) {
    k_core_sums<<<nsys, 256, 0, s>>>(w->dw, active, eact, out);
    e = cudaGetLastError();
  }
  res.assign(3 * (size_t)nsys, 0.0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(res.data(), out, sizeof(double) * 3 * nsys, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(deg);
  cudaFree(changed);
  cudaFree(active);
  cudaFree(leave);
  cudaFree(eact);
  cudaFree(out);
  return e == cudaSuccess ? XDEM_OK : (int32_t)cuda_check(w, e);
}
}  // namespace

int32_t xdem_quadron_z_phi(xdem_world w, double out[2]) {
  if (!w || !out || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  std::vector<double> r;
  int32_t st = core_z_phi(w, r);
  if (st) return st;
  out[0] = r[0];
  out[1] = r[1];
  return XDEM_OK;
}

int32_t xdem_batch_quadron_z_phi(xdem_world w, double* out) {
  if (!w || !out || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  std::vector<double> r;
  int32_t st = core_z_phi(w, r);
  if (st) return st;
  for (int k = 0; k < w->nsys; ++k) {
    out[2 * k] = r[3 * k];
    out[2 * k + 1] = r[3 * k + 1];
  }
  return XDEM_OK;
}

// ---- launch configuration and autotuning -----------------------------------------
int32_t xdem_set_launch_config(xdem_world w, int32_t pair_blocks_per_sm, double cell_factor) {
  if (!w || pair_blocks_per_sm < 1 || pair_blocks_per_sm > 64 || !(cell_factor >= 1.0) ||
      cell_factor > 4.0)
    return XDEM_ERR_ARGUMENT;
  cudaStreamSynchronize(w->stream);
  w->pair_blocks_per_sm = pair_blocks_per_sm;
  w->cell_factor = cell_factor;
  if (w->dw.n > 0 && !w->base_maxsize.empty()) {
    // a coarser grid must still fit the cell blocks allocated for the base size
    CK(w, modify_all(w, [&](WorldScalars& s, int k) { s.maxsize = w->base_maxsize[k] * cell_factor; }));
  }
  return XDEM_OK;
}

int32_t xdem_set_candidate_lists(xdem_world w, int32_t capacity, double skin_fraction) {
  if (!w || capacity < 0 || capacity > 256 || !(skin_fraction > 0.0) || skin_fraction > 1.0)
    return XDEM_ERR_ARGUMENT;
  if (w->dw.n > 0) return XDEM_ERR_ARGUMENT;  // before xdem_set_particles
  w->vl_capacity = capacity;
  w->skin_fraction = skin_fraction;
  return XDEM_OK;
}

int32_t xdem_set_memory_order_refresh(xdem_world w, int32_t interval) {
  // odd: a captured chunk (one re-sort and `interval` steps) must swap the
  // record sets an even number of times
  if (!w || interval < 0 || (interval > 0 && (interval % 2) == 0) || interval > (1 << 20))
    return XDEM_ERR_ARGUMENT;
  w->resort_every = interval;
  return XDEM_OK;
}

int32_t xdem_get_candidate_list_stats(xdem_world w, int64_t out[4]) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  out[0] = (int64_t)s.vl_builds;
  out[1] = out[2] = 0;
  out[3] = w->dw.V;
  if (w->dw.V > 0 && w->dw.n > 0) {
    std::vector<int32_t> cnt(w->dw.n);
    CK(w, download(cnt.data(), w->dw.vl_cnt, w->dw.n, w->stream));
    CK(w, cudaStreamSynchronize(w->stream));
    int64_t tot = 0, mx = 0;
    for (int32_t c : cnt) {
      tot += c;
      mx = std::max<int64_t>(mx, c);
    }
    out[1] = mx;
    out[2] = tot;
  }
  return XDEM_OK;
}

int32_t xdem_get_launch_config(xdem_world w, int32_t* pair_blocks_per_sm, double* cell_factor) {
  if (!w) return XDEM_ERR_ARGUMENT;
  if (pair_blocks_per_sm) *pair_blocks_per_sm = w->pair_blocks_per_sm;
  if (cell_factor) *cell_factor = w->cell_factor;
  return XDEM_OK;
}

int32_t xdem_autotune(xdem_world w, const xdem_control* ctl, int32_t steps_per_trial,
                      double* trial_ms) {
  if (!w || !ctl || steps_per_trial < 1 || w->dw.n <= 0 || ctl->stop_on_pressure)
    return XDEM_ERR_ARGUMENT;
  static const int kBlocks[4] = {4, 8, 16, 32};
  static const double kFactors[3] = {1.0, 1.2, 1.5};
  double best = 1e300;
  int bb = w->pair_blocks_per_sm;
  double bf = w->cell_factor;
  uint32_t st_all = 0;
  for (int fi = 0; fi < 3; ++fi)
    for (int bi = 0; bi < 4; ++bi) {
      int32_t s = xdem_set_launch_config(w, kBlocks[bi], kFactors[fi]);
      if (s) return s;
      // one untimed step settles the grid, then the timed trial
      int32_t done = 0;
      st_all |= (uint32_t)xdem_run(w, 1, ctl, &done);
      CK(w, xdem_timer_start(w) == XDEM_OK ? cudaSuccess : cudaErrorUnknown);
      st_all |= (uint32_t)xdem_run(w, steps_per_trial, ctl, &done);
      double ms = 0.0;
      CK(w, xdem_timer_stop(w, &ms) == XDEM_OK ? cudaSuccess : cudaErrorUnknown);
      if (trial_ms) trial_ms[fi * 4 + bi] = ms;
      if (ms < best) {
        best = ms;
        bb = kBlocks[bi];
        bf = kFactors[fi];
      }
    }
  int32_t s = xdem_set_launch_config(w, bb, bf);
  return s ? s : (int32_t)st_all;
}

int32_t xdem_harvest_pairs(xdem_world w, xdem_mlp m, int32_t stride, int64_t max_new, int64_t* added) {
  if (!w || !m || stride <= 0 || max_new <= 0 || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  if (added) *added = 0;
  CK(w, cudaStreamSynchronize(m->stream));
  CK(w, mlp_reserve(m, m->size + max_new));
  unsigned long long* dcount = nullptr;
  CK(w, cudaMalloc(&dcount, sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), w->stream);
  if (e == cudaSuccess) {
    k_harvest<<<148 * 8, 128, 0, w->stream>>>(w->dw, m->dev(), stride, m->x, m->target, m->contact,
                                              m->size, m->size + max_new, dcount);
    e = cudaGetLastError();
  }
  unsigned long long got = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&got, dcount, sizeof(got), cudaMemcpyDeviceToHost, w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  cudaFree(dcount);
  CK(w, e);
  const int64_t n = std::min<int64_t>((int64_t)got, max_new);
  m->size += n;
  if (added) *added = n;
  return XDEM_OK;
}

int32_t xdem_get_kinetic_energy(xdem_world w, double* out) {
  if (!w || !out || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  int nb = blocks_for(w->dw.n, kReduceBlock);
  LAUNCH(w, KK_KE, k_ke_partial<<<nb, kReduceBlock, 0, w->stream>>>(w->dw));
  LAUNCH(w, KK_KE, k_ke_final<<<1, 1024, 0, w->stream>>>(w->dw, nb));
  CK(w, cudaGetLastError());
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  *out = s.ke;
  return XDEM_OK;
}

// ---- sub-steps ---------------------------------------------------------------
#define SUBSTEP_BEGIN                                   \
  if (!w || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;     \
  do {                                                  \
  } while (0)
#define SUBSTEP_END                  \
  CK(w, cudaGetLastError());         \
  return (int32_t)fetch_status(w)

int32_t xdem_modify_particle_position(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_modify(w);
  SUBSTEP_END;
}

int32_t xdem_apply_background_velocity(xdem_world w) {
  SUBSTEP_BEGIN;
  LAUNCH(w, KK_BACKGROUND, k_background_velocity<<<blocks_for(w->dw.n, kBlock), kBlock, 0, w->stream>>>(w->dw, 1));
  SUBSTEP_END;
}

int32_t xdem_remove_background_velocity(xdem_world w) {
  SUBSTEP_BEGIN;
  LAUNCH(w, KK_BACKGROUND, k_background_velocity<<<blocks_for(w->dw.n, kBlock), kBlock, 0, w->stream>>>(w->dw, 0));
  SUBSTEP_END;
}

int32_t xdem_find_possible_contacts(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_find(w);
  SUBSTEP_END;
}

int32_t xdem_update_contacts(xdem_world w) {
  SUBSTEP_BEGIN;
  CK(w, cudaMemsetAsync(w->dw.incnt, 0, sizeof(int32_t) * w->dw.n, w->stream));
  launch_update(w, false, 1);
  SUBSTEP_END;
}

int32_t xdem_collect_force_and_torque(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_collect(w);
  SUBSTEP_END;
}

int32_t xdem_take_time_integral(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_integrate(w, false, 0);
  SUBSTEP_END;
}

int32_t xdem_reset_velocity_of_rattlers(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_rattlers(w, 1, 0.0);
  SUBSTEP_END;
}

int32_t xdem_scale_velocity_of_rattlers(xdem_world w, double scale) {
  SUBSTEP_BEGIN;
  launch_rattlers(w, 0, scale);
  SUBSTEP_END;
}

int32_t xdem_update_total_stress(xdem_world w, double stress[4]) {
  SUBSTEP_BEGIN;
  launch_stress(w);
  CK(w, cudaGetLastError());
  int32_t st = (int32_t)fetch_status(w);
  if (stress) {
    int32_t e = xdem_get_stress(w, stress);
    if (e) return st | e;
  }
  return st;
}

int32_t xdem_update_boundary(xdem_world w, int32_t law, double p0, double p1) {
  SUBSTEP_BEGIN;
  if (law < 0 || law > 4) return XDEM_ERR_ARGUMENT;
  launch_end_of_step(w, law, p0, p1, 0, 0, 0.0, 0);
  SUBSTEP_END;
}

int32_t xdem_update_lees_edwards_boundary(xdem_world w) {
  SUBSTEP_BEGIN;
  launch_end_of_step(w, BOX_NONE, 0.0, 0.0, 1, 0, 0.0, 0);
  SUBSTEP_END;
}

int32_t xdem_scale_boundary_to_solid_fraction(xdem_world w, double phi) {
  // scaleBoundarySizeToGivenSolidFraction (PeriodicBoundaryWorld.cpp:276-284)
  SUBSTEP_BEGIN;
  if (!(phi > 0.0) || w->nsys > 1) return XDEM_ERR_ARGUMENT;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  double cur = w->total_volume / (s.xlen * s.ylen);
  double scale = std::sqrt(cur / phi);
  s.vl_valid = 0;
  s.scale_x = scale;
  s.scale_y = scale;
  s.xmin *= scale;
  s.xmax *= scale;
  s.ymin *= scale;
  s.ymax *= scale;
  s.xlen = s.xmax - s.xmin;
  s.ylen = s.ymax - s.ymin;
  CK(w, write_scalars(w, &s));
  LAUNCH(w, KK_SCALE, k_scale_positions<<<blocks_for(w->dw.n, kBlock), kBlock, 0, w->stream>>>(w->dw));
  SUBSTEP_END;
}

// ---- whole steps -------------------------------------------------------------
int32_t xdem_take_time_step(xdem_world w) {
  SUBSTEP_BEGIN;
  xdem_control ctl{};
  ctl.sequence = XDEM_SEQ_TAKE_TIME_STEP;
  policy_step(w, &ctl, 1);
  SUBSTEP_END;
}

int32_t xdem_run(xdem_world w, int32_t nsteps, const xdem_control* ctl, int32_t* steps_done) {
  SUBSTEP_BEGIN;
  if (!ctl || nsteps < 0 || ctl->sequence < 0 || ctl->sequence > 1 || ctl->box_law < 0 ||
      ctl->box_law > 4)
    return XDEM_ERR_ARGUMENT;
  // a batch steps all its systems together (one slot-set parity)
  if (w->nsys > 1 && ctl->stop_on_pressure) return XDEM_ERR_ARGUMENT;
  if (steps_done) *steps_done = 0;
  if (nsteps == 0) return XDEM_OK;
  WorldScalars s;
  CK(w, read_scalars(w, &s));
  s.stop = 0;
  s.steps_done = 0;
  s.flips = 0;
  CK(w, write_scalars(w, &s));
  const int start_par = w->par;
  // every step but the last skips the recorded contact fields unless the run
  // may stop early
  const int rec_all = ctl->stop_on_pressure ? 1 : 0;
  int body = nsteps - 1;
  // direct steps until a re-sort is due, then whole chunks (one re-sort and
  // resort_every steps, or 32 steps without re-sorts) captured once in a
  // CUDA graph and replayed
  const int chunk = w->resort_every > 0 ? w->resort_every : 32;
  while (w->resort_every > 0 && body > 0 && w->since_resort < w->resort_every) {
    policy_step(w, ctl, rec_all);
    --body;
  }
  if (body >= chunk && !w->prof_on) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const int par0 = w->par;
    const int64_t launches_before = w->launches;
    CK(w, cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) policy_step(w, ctl, rec_all);
    cudaError_t e = cudaStreamEndCapture(w->stream, &graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return (int32_t)(cuda_check(w, e) | fetch_status(w));
    }
    // a chunk swaps the record sets an even number of times: parity unchanged
    w->par = par0;
    const int reps = body / chunk;
    const int64_t per_chunk = w->launches - launches_before;
    w->launches += per_chunk * (reps - 1);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = cudaGraphLaunch(exec, w->stream);
    body -= reps * chunk;
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    CK(w, e);
  }
  for (; body > 0; --body) policy_step(w, ctl, rec_all);
  policy_step(w, ctl, 1);
  CK(w, cudaGetLastError());
  uint32_t st = fetch_status(w);
  CK(w, read_scalars(w, &s));
  if (steps_done) *steps_done = s.steps_done;
  // slot-set swaps that actually ran (none after a stop)
  w->par = start_par ^ (s.flips & 1);
  return (int32_t)st;
}

int32_t xdem_synchronize(xdem_world w) {
  if (!w) return XDEM_ERR_ARGUMENT;
  return (int32_t)fetch_status(w);
}

int32_t xdem_upload_state(xdem_world w, const double* x, const double* y, const double* vx,
                          const double* vy, const double* rot, const double* rot_vel) {
  if (!w || w->dw.n <= 0 || !x || !y || !vx || !vy || !rot || !rot_vel) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n;
  cudaStream_t s = w->stream;
  double* st = w->dw.stage;
  const double* src[6] = {x, y, vx, vy, rot, rot_vel};
  for (int k = 0; k < 6; ++k) CK(w, upload(st + (size_t)k * n, src[k], n, s));
  LAUNCH(w, KK_STAGE, k_stage<<<blocks_for(n, kBlock), kBlock, 0, s>>>(w->dw, 1));
  CK(w, cudaGetLastError());
  return XDEM_OK;
}

int32_t xdem_download_state(xdem_world w, double* x, double* y, double* vx, double* vy,
                            double* rot, double* rot_vel) {
  if (!w || w->dw.n <= 0) return XDEM_ERR_ARGUMENT;
  const int n = w->dw.n;
  cudaStream_t s = w->stream;
  LAUNCH(w, KK_STAGE, k_stage<<<blocks_for(n, kBlock), kBlock, 0, s>>>(w->dw, 0));
  const double* st = w->dw.stage;
  double* dst[6] = {x, y, vx, vy, rot, rot_vel};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) CK(w, download(dst[k], st + (size_t)k * n, n, s));
  CK(w, cudaStreamSynchronize(s));
  return XDEM_OK;
}

int32_t xdem_set_profiling(xdem_world w, int32_t enable) {
  if (!w) return XDEM_ERR_ARGUMENT;
  CK(w, cudaStreamSynchronize(w->stream));
  w->prof_on = enable != 0;
  w->prof_used = 0;
  return XDEM_OK;
}

int32_t xdem_profile_kinds(void) { return KK_COUNT; }

const char* xdem_profile_name(int32_t kind) {
  return (kind >= 0 && kind < KK_COUNT) ? kKindNames[kind] : "unknown";
}

int32_t xdem_get_profile(xdem_world w, int32_t nkinds, int64_t* launches, double* total_ms) {
  if (!w || nkinds < 0 || !launches || !total_ms) return XDEM_ERR_ARGUMENT;
  CK(w, cudaStreamSynchronize(w->stream));
  for (int k = 0; k < nkinds; ++k) {
    launches[k] = 0;
    total_ms[k] = 0.0;
  }
  for (size_t i = 0; i < w->prof_used; ++i) {
    float ms = 0.f;
    CK(w, cudaEventElapsedTime(&ms, w->prof_events[2 * i], w->prof_events[2 * i + 1]));
    int k = w->prof_kind[i];
    if (k < nkinds) {
      launches[k] += 1;
      total_ms[k] += ms;
    }
  }
  return XDEM_OK;
}

int32_t xdem_launch_count(xdem_world w, int64_t* out) {
  if (!w || !out) return XDEM_ERR_ARGUMENT;
  *out = w->launches;
  return XDEM_OK;
}

int32_t xdem_timer_start(xdem_world w) {
  if (!w) return XDEM_ERR_ARGUMENT;
  if (!w->timer[0]) {
    CK(w, cudaEventCreate(&w->timer[0]));
    CK(w, cudaEventCreate(&w->timer[1]));
  }
  CK(w, cudaEventRecord(w->timer[0], w->stream));
  return XDEM_OK;
}

int32_t xdem_timer_stop(xdem_world w, double* ms) {
  if (!w || !ms || !w->timer[0]) return XDEM_ERR_ARGUMENT;
  CK(w, cudaEventRecord(w->timer[1], w->stream));
  CK(w, cudaEventSynchronize(w->timer[1]));
  float f = 0.f;
  CK(w, cudaEventElapsedTime(&f, w->timer[0], w->timer[1]));
  *ms = f;
  return XDEM_OK;
}

void* xdem_host_alloc(int64_t bytes) {
  void* p = nullptr;
  if (bytes <= 0 || cudaHostAlloc(&p, (size_t)bytes, cudaHostAllocDefault) != cudaSuccess)
    return nullptr;
  return p;
}

void xdem_host_free(void* p) {
  if (p) cudaFreeHost(p);
}


// ---- single-pair geometry ------------------------------------------------------
int32_t xdem_pair_geometry(int32_t npairs, int32_t method, int32_t precision, const double* pi,
                           const double* pj, const double* off, double* out) {
  if (npairs <= 0 || !pi || !pj || !off || !out || precision < 0 || precision > 1)
    return XDEM_ERR_ARGUMENT;
  double *dpi = nullptr, *dpj = nullptr, *doff = nullptr, *dout = nullptr;
  uint32_t* dst = nullptr;
  uint32_t st = 0;
  cudaError_t e = cudaMalloc(&dpi, sizeof(double) * 9 * npairs);
  if (e == cudaSuccess) e = cudaMalloc(&dpj, sizeof(double) * 9 * npairs);
  if (e == cudaSuccess) e = cudaMalloc(&doff, sizeof(double) * 4 * npairs);
  if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 17 * npairs);
  if (e == cudaSuccess) e = cudaMalloc(&dst, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(dst, 0, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemcpy(dpi, pi, sizeof(double) * 9 * npairs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dpj, pj, sizeof(double) * 9 * npairs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(doff, off, sizeof(double) * 4 * npairs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (precision == XDEM_PRECISION_MIXED)
      k_pair_geometry_m<<<blocks_for(npairs, 128), 128>>>(npairs, method, dpi, dpj, doff, dout, dst);
    else
      k_pair_geometry<<<blocks_for(npairs, 128), 128>>>(npairs, method, dpi, dpj, doff, dout, dst);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 17 * npairs, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&st, dst, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(dpi);
  cudaFree(dpj);
  cudaFree(doff);
  cudaFree(dout);
  cudaFree(dst);
  if (e != cudaSuccess) st |= XDEM_ERR_CUDA;
  return (int32_t)st;
}

}  // extern "C"
