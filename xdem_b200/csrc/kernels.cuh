// kernels.cuh — the per-timestep kernels (FP64 path).
//
// Step of a PeriodicBoundaryWorld (PeriodicBoundaryWorld.cpp:119-127):
//   k_modify_position           wrap into the box                     (a2)
//   k_bin / k_scan_* / k_scatter  counting sort of particles by cell   (a3, a4)
//   k_update_contacts           3x3 cell scan, geometry, force, history (a5-a15)
//   k_collect                   deterministic per-particle sums         (a16)
//   k_integrate                 semi-implicit Euler, clumps, rattlers (a17-a19)
// plus k_stress_* (a21), k_end_of_step / k_scale_positions (a20, a22).
// Every thread works on memory position m (world.cuh); ids come from id_of.
#pragma once
#include "geometry.cuh"
#include "world.cuh"

namespace xdem {

enum : int { WORLD_PERIODIC = 0, WORLD_CONTROL = 1, WORLD_LE = 2 };
enum : int { SKIP_TIME_INTEGRAL = 1, SKIP_CONTACT_DETECTION = 2, SKIP_MACRO_SUM = 4 };
enum : int { CAND_REGULAR = 0, CAND_TOP = 1, CAND_BOTTOM = 2 };

constexpr int kCandidateCap = 200;  // MAXIMUM_POSSIBLE_CONTACT_LIST_SIZE (BaseWorld.h:11)

struct Grid {
  int nx, ny, ncell;
  int base;  // first cell of the system in the cell arrays
  double lx, ly;
};

// system of the particle at memory position m
__device__ __forceinline__ int sys_at(const DevWorld& w, int m) {
  return w.nsys > 1 ? w.sys_of[m] : 0;
}

// run-level stop flag (set by a stop condition; ends the kernels of a run)
__device__ __forceinline__ bool stopped(const DevWorld& w) { return w.ws->stop != 0; }

// Programmatic dependent launch of a step's kernels: a kernel launched with
// it may become resident while the kernel before it in the stream runs;
// pdl_begin first waits until that kernel has completed and its writes are
// visible (a no-op for an ordinary launch), then lets the next kernel launch
// (it becomes resident once every block of this one has started, and waits
// in its own pdl_begin).  Every kernel that a step launches this way calls
// pdl_begin before touching memory.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Grid of PeriodicBoundaryWorld::findPossibleContacts (PeriodicBoundaryWorld.cpp:17-22):
// nx = floor(xlen / (2.01 r_max)); clamped to the allocated capacity, which
// only makes cells larger and leaves the contact set unchanged.  Regular cell
// (ix, iy) is base + iy*nx + ix; the Lees-Edwards ghost rows follow at
// base + ncell.
__device__ __forceinline__ Grid grid_of(const WorldScalars& ws) {
  Grid g;
  double xlen = ws.xmax - ws.xmin, ylen = ws.ymax - ws.ymin;
  g.nx = (int)floor(xlen / ws.maxsize);
  g.ny = (int)floor(ylen / ws.maxsize);
  if (g.nx > ws.nx_cap) g.nx = ws.nx_cap;
  if (g.ny > ws.ny_cap) g.ny = ws.ny_cap;
  g.ncell = g.nx * g.ny;
  g.base = ws.cell_base;
  g.lx = xlen / g.nx;
  g.ly = ylen / g.ny;
  return g;
}

// system owning cell c (binary search over the systems' first cells)
__device__ __forceinline__ int sys_of_cell(const DevWorld& w, int c) {
  if (w.nsys <= 1) return 0;
  int lo = 0, hi = w.nsys - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (w.sys_cell_base[mid] <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// cell of a coordinate; the reference's floor() can reach numGrid at the upper
// edge (an out-of-range bin there), clamped here
__device__ __forceinline__ int cell_of(double v, double vmin, double len, int ng) {
  int c = (int)floor((v - vmin) / len);
  return c < 0 ? 0 : (c > ng - 1 ? ng - 1 : c);
}

__device__ __forceinline__ void raise(uint32_t* status, uint32_t bits) {
  if (bits) atomicOr(status, bits);
}

// A thread's status bits and closest-approach Newton counts, combined over
// its warp and added by one lane: the counters are single addresses shared by
// the whole grid, where one atomic per thread would serialise.  Every lane of
// the warp must call it.
__device__ __forceinline__ void flush_warp(const DevWorld& w, uint32_t st, uint32_t solves,
                                           uint32_t iters, uint32_t capped) {
  const unsigned full = 0xffffffffu;
  st = __reduce_or_sync(full, st);
  solves = __reduce_add_sync(full, solves);
  iters = __reduce_add_sync(full, iters);
  capped = __reduce_add_sync(full, capped);
  if ((threadIdx.x & 31) == 0) {
    if (st) atomicOr(w.status, st);
    if (solves) {
      WorldScalars* wsm = w.ws;
      atomicAdd(&wsm->newton_solves, (unsigned long long)solves);
      atomicAdd(&wsm->newton_iters, (unsigned long long)iters);
      if (capped) atomicAdd(&wsm->newton_capped, (unsigned long long)capped);
    }
  }
}

// Whether this block is the last of its launch to get here (the same answer in
// every thread of the block): every thread fences its writes, then the block
// counts itself in `counter`; the last block sees what the others wrote.  The
// caller resets the counter.  Nothing waits.
__device__ __forceinline__ bool last_block(uint32_t* counter, bool& sh_last) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) sh_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  const bool last = sh_last;
  if (last) __threadfence();
  return last;
}

// ---------------------------------------------------------------------------
// a2: modifyParticlePosition (PeriodicBoundaryWorld.cpp:129-142,
//     LeesEdwardsBoundaryWorld.cpp:304-333)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 modify_position_at(const DevWorld& w, const WorldScalars& ws,
                                                      int i) {
  double2 p = w.pos[i];
  if (w.kind == WORLD_LE) {
    if (p.y < ws.ymin) {
      p.y += ws.ylen;
      p.x += ws.shift;
      if (w.V) w.ws->vl_valid = 0;  // its image kinds change: rebuild the candidate lists
    } else if (p.y > ws.ymax) {
      p.y += -ws.ylen;
      p.x += -ws.shift;
      if (w.V) w.ws->vl_valid = 0;
    }
    if (p.x < ws.xmin) p.x += ws.xlen;
    else if (p.x > ws.xmax) p.x += -ws.xlen;
  } else {
    if (p.x < ws.xmin) p.x += ws.xlen;
    else if (p.x > ws.xmax) p.x += -ws.xlen;
    if (p.y < ws.ymin) p.y += ws.ylen;
    else if (p.y > ws.ymax) p.y += -ws.ylen;
  }
  w.pos[i] = p;
  return p;
}

__global__ void k_modify_position(DevWorld w) {
  if (stopped(w)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  modify_position_at(w, w.ws[sys_at(w, i)], i);
}

// scaleAllParticlePosition(scale_x, scale_y) (BaseWorld.cpp:119-124); after a
// run's stop the scales are 1 and the pass leaves positions unchanged
__global__ void k_scale_positions(DevWorld w) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  const WorldScalars& ws = w.ws[sys_at(w, i)];
  double2 p = w.pos[i];
  const double2 old = p;
  p.x *= ws.scale_x;
  p.y *= ws.scale_y;
  w.pos[i] = p;
  // the lists' travel budget covers relative moves between bodies; a wall
  // segment's reach also changes with its own move (screen_radius)
  if (w.V && w.seg && w.shape[i] == SHAPE_SEGMENT) {
    const double ex = p.x - old.x, ey = p.y - old.y;
    w.vl_disp[i] += 2.0 * sqrt(ex * ex + ey * ey);
  }
}

// a6: LeesEdwardsBoundaryWorld::apply/removeBackgroudVelocity (:508-530)
__global__ void k_background_velocity(DevWorld w, int apply) {
  if (stopped(w)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  const WorldScalars& ws = w.ws[sys_at(w, i)];
  double2 v = w.vel[i];
  double y = w.pos[i].y;
  if (apply) v.x = v.x + ws.shift_rate * y;
  else v.x = v.x - ws.shift_rate * y;
  w.vel[i] = v;
}

// the record of the body at m for this step's pair kernels; cs = (cos, sin)
// of its orientation for an ellipse
__device__ __forceinline__ void write_body(const DevWorld& w, int m, double2 cs) {
  BodyRec b;
  b.pos = w.pos[m];
  b.vel = w.vel[m];
  b.rot = w.rot[m];
  b.w = w.w[m];
  b.r = w.rad[m];
  b.asp = w.asp[m];
  b.cs = cs;
  b.shape = w.shape[m];
  b.id = w.id_of[m];
  b.setting = w.setting[m];
  b.pad = 0;
  w.body[m] = b;
}

// ---------------------------------------------------------------------------
// a3/a4: cell binning.  Counting sort: per-cell counts by atomics, an
// exclusive scan, and a scatter.  Ghost rows after the regular cells hold the
// Lees-Edwards images: row ncell+[0,nx) takes bottom-row particles shifted by
// +shift (boxLE_top, LeesEdwardsBoundaryWorld.cpp:75-81), row
// ncell+nx+[0,nx) top-row particles shifted by -shift (boxLE_bottom, :82-88).
// The order inside a cell is not fixed; nothing downstream depends on it.
// ---------------------------------------------------------------------------
// The binning of the body at i.
// MODIFY: k_modify_position's wrap first, in the same thread (a step's
// position move followed by the binning)
template <bool MODIFY>
__device__ __forceinline__ void bin_at(const DevWorld& w, int i) {
  const WorldScalars& ws = w.ws[sys_at(w, i)];
  const double2 p = MODIFY ? modify_position_at(w, ws, i) : w.pos[i];
  if (MODIFY) {
    // this step's body record for the pair kernels (the candidate kernel
    // writes it instead after a re-sort, or when the step runs as sub-steps)
    double2 cs = make_double2(0.0, 0.0);
    if (w.shape[i] == SHAPE_ELLIPSE) {
      const double r = w.rot[i];
      cs = make_double2(cos(r), sin(r));
    }
    write_body(w, i, cs);
  }
  if (w.axis && w.shape[i] == SHAPE_ELLIPSE) {
    // the centre-line screen's record (pairs.cuh, axis_shape): the
    // orientation reduced to [-pi, pi] in FP64 before the FP32 sine and cosine
    double r = w.rot[i];
    r -= 6.283185307179586 * rint(r * 0.15915494309189535);
    float sn, cs;
    __sincosf((float)r, &sn, &cs);
    const float a = (float)w.rad[i];
    w.axis[i] = make_float4(cs, sn, a, __fdividef(a, (float)w.asp[i]));
  }
  Grid G = grid_of(ws);
  w.incnt[i] = 0;  // incoming-contact counters of this step's update
  if (G.nx < 3 || G.ny < 3) {
    if (i == ws.first) raise(w.status, ST_GRID);
    return;
  }
  int ix = cell_of(p.x, ws.xmin, G.lx, G.nx);
  int iy = cell_of(p.y, ws.ymin, G.ly, G.ny);
  int c = G.base + iy * G.nx + ix;
  w.pcell[i] = c;
  w.prank[i] = atomicAdd(&w.cell_count[c], 1);
  int gc = -1;
  if (w.kind == WORLD_LE) {
    if (iy == 0) {
      double t = p.x + ws.shift;
      if (t < ws.xmin) t += ws.xlen;
      else if (t > ws.xmax) t -= ws.xlen;
      gc = G.base + G.ncell + cell_of(t, ws.xmin, G.lx, G.nx);
    } else if (iy == G.ny - 1) {
      double t = p.x - ws.shift;
      if (t < ws.xmin) t += ws.xlen;
      else if (t > ws.xmax) t -= ws.xlen;
      gc = G.base + G.ncell + G.nx + cell_of(t, ws.xmin, G.lx, G.nx);
    }
  }
  w.gcell[i] = gc;
  if (gc >= 0) w.grank[i] = atomicAdd(&w.cell_count[gc], 1);
}

// Whether this step rebuilds the candidate lists (system 0's vl_build), from
// mx, the largest path length since the last build, and every system's travel
// budget (the block's threads read the systems' budgets side by side); every
// thread of the block calls
__device__ __forceinline__ void list_rebuild_decision(const DevWorld& w, double mx) {
  WorldScalars* ws = w.ws;
  int need = threadIdx.x == 0 && ws[0].vl_valid == 0;
  for (int s = threadIdx.x; s < w.nsys; s += blockDim.x)
    if (2.0 * mx + ws[s].vl_travel >= w.skin) need = 1;
  const bool rebuild = __syncthreads_or(need) != 0;
  if (rebuild)
    for (int s = threadIdx.x; s < w.nsys; s += blockDim.x) ws[s].vl_travel = 0.0;
  if (threadIdx.x == 0) {
    ws[0].vl_build = rebuild ? 1 : 0;
    if (rebuild) {
      ws[0].vl_valid = 1;
      ws[0].vl_overflow = 0;
      ws[0].vl_builds += 1;
    }
  }
}

// Whether this step's scan reads the cell records: a list rebuild, a list
// that overflowed at the last build (scanned in full every step), or nine
// cells that may hold the 200-candidate cap's count (counted from the
// records); known once the rebuild decision is taken
__device__ __forceinline__ bool cells_needed(const DevWorld& w) {
  return w.ws->vl_build || w.ws->vl_overflow || 9 * *w.cell_max + 1 >= kCandidateCap;
}

// a3: the binning of every body
template <bool MODIFY = false>
__global__ void k_bin(DevWorld w) {
  pdl_begin();
  if (stopped(w)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *w.cell_max = 0;  // k_scan_tiles takes the maximum
  if (i < w.n) bin_at<MODIFY>(w, i);
}

// Exclusive scan of cell_count[0 .. ncell + 2nx) into cell_start, in three
// passes over tiles of kScanTile cells: tile sums, a scan of the tile sums
// (one block), and the per-tile exclusive prefixes.
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

// block-wide inclusive scan of one value per thread (kScanThreads threads)
__device__ __forceinline__ int32_t block_inclusive_scan(int32_t v, int32_t* sh_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) sh_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int32_t s = (lane < kScanThreads / 32) ? sh_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t u = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += u;
    }
    if (lane < kScanThreads / 32) sh_warp[lane] = s;
  }
  __syncthreads();
  if (warp > 0) v += sh_warp[warp - 1];
  return v;
}

// exclusive scan of the tile sums (one block); cell_start[total] = total
// count.  The tile sums come from other blocks of the same launch: read past
// the L1.
__device__ __forceinline__ void scan_tile_sums(const DevWorld& w, int32_t* sh_warp) {
  const int total = w.ncell_total;
  int ntiles = (total + kScanTile - 1) / kScanTile;
  int32_t carry = 0;
  for (int base = 0; base < ntiles; base += kScanThreads) {
    int t = base + threadIdx.x;
    int32_t v = t < ntiles ? __ldcg(w.tile_sum + t) : 0;
    int32_t inc = block_inclusive_scan(v, sh_warp);
    if (t < ntiles) w.tile_sum[t] = carry + inc - v;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) sh_warp[0] = inc;
    __syncthreads();
    carry += sh_warp[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) w.cell_start[total] = carry;
}

// tile sums, and the largest cell count; the last block to finish scans the
// tile sums (a fence before the count of finished blocks makes every tile
// sum visible to it; nothing waits)
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(DevWorld w) {
  pdl_begin();
  if (stopped(w)) return;
  const int total = w.ncell_total;
  int ntiles = (total + kScanTile - 1) / kScanTile;
  __shared__ int32_t sh_warp[kScanThreads / 32];
  __shared__ bool last;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int base = tile * kScanTile + threadIdx.x * kScanPer;
    int32_t s = 0, mx = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
      if (base + k < total) {
        const int32_t c = w.cell_count[base + k];
        s += c;
        mx = max(mx, c);
      }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if ((threadIdx.x & 31) == 0 && mx > 0) atomicMax(w.cell_max, mx);
    int32_t inc = block_inclusive_scan(s, sh_warp);
    if (threadIdx.x == kScanThreads - 1) w.tile_sum[tile] = inc;
    __syncthreads();
  }
  if (last_block(&w.done[1], last)) {
    scan_tile_sums(w, sh_warp);
    if (threadIdx.x == 0) w.done[1] = 0;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(DevWorld w) {
  pdl_begin();
  if (stopped(w)) return;
  const int total = w.ncell_total;
  int ntiles = (total + kScanTile - 1) / kScanTile;
  __shared__ int32_t sh_warp[kScanThreads / 32];
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int base = tile * kScanTile + threadIdx.x * kScanPer;
    int32_t c[kScanPer];
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
      c[k] = (base + k < total) ? w.cell_count[base + k] : 0;
      s += c[k];
    }
    int32_t run = block_inclusive_scan(s, sh_warp) - s + w.tile_sum[tile];
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
      if (base + k < total) w.cell_start[base + k] = run;
      run += c[k];
    }
    __syncthreads();
  }
}

// Radius of the coarse FP32 screen of the body at m: its screening radius, or
// for a wall segment the farthest point it can touch from its position (its
// half length, or more once a box law has moved its midpoint but not its
// vertices), with a relative margin of 1e-6.  The candidate lists count a
// segment's moves twice (its reach grows with them), see seg_path_factor.
__device__ __forceinline__ float screen_radius(const DevWorld& w, int m) {
  if (w.seg && w.shape[m] == SHAPE_SEGMENT) {
    const double4 v = w.seg[w.id_of[m]];
    const double2 p = w.pos[m];
    const double a = sqrt((v.x - p.x) * (v.x - p.x) + (v.y - p.y) * (v.y - p.y));
    const double b = sqrt((v.z - p.x) * (v.z - p.x) + (v.w - p.y) * (v.w - p.y));
    return (float)(fmax(w.rad[m], fmax(a, b)) * (1.0 + 1e-6));
  }
  return (float)w.screen_r[m];
}

// path-length weight of the body at m for the candidate lists: 2 for a wall
// segment (its position and its reach both move), 1 otherwise
__device__ __forceinline__ double seg_path_factor(const DevWorld& w, int m) {
  return (w.seg && w.shape[m] == SHAPE_SEGMENT) ? 2.0 : 1.0;
}

// The cell-ordered records of the 3x3 scan; also clears cell_count (already
// consumed by the scan) for the next binning.  when_needed: this step's
// rebuild decision is taken, and the records are written only where a scan
// reads them (cells_needed).
__global__ void k_scatter(DevWorld w, int when_needed) {
  pdl_begin();
  if (stopped(w)) return;
  const int total = w.ncell_total;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x)
    w.cell_count[c] = 0;
  if (when_needed && !cells_needed(w)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  const Grid G = grid_of(w.ws[sys_at(w, i)]);
  if (G.nx < 3 || G.ny < 3) return;
  const WorldScalars& ws = w.ws[sys_at(w, i)];
  const double2 p = w.pos[i];
  const int pc = w.pcell[i], local = pc - G.base;
  const int ix = local % G.nx, iy = local / G.nx;
  // position relative to the cell's corner; y is the same in a ghost row
  const float ry = (float)(p.y - (ws.ymin + iy * G.ly));
  const float sr = screen_radius(w, i);
  const float idb = __int_as_float((w.setting[i] & SKIP_CONTACT_DETECTION) ? -1 : w.id_of[i]);
  const int up = w.up[i];
  int q = w.cell_start[pc] + w.prank[i];
  w.cell_mem[q] = i;
  w.cell_pos[q] = p;
  w.cell_scr[q] = make_float4((float)(p.x - (ws.xmin + ix * G.lx)), ry, sr, idb);
  w.cell_up[q] = up;
  int gc = w.gcell[i];
  if (gc >= 0) {
    // the image's x as k_bin placed it: shifted by +shift (bottom row, into
    // the ghost row above the top) or -shift (top row), wrapped into the box
    double t = iy == 0 ? p.x + ws.shift : p.x - ws.shift;
    if (t < ws.xmin) t += ws.xlen;
    else if (t > ws.xmax) t -= ws.xlen;
    const int gx = gc - G.base - G.ncell - (iy == 0 ? 0 : G.nx);
    q = w.cell_start[gc] + w.grank[i];
    w.cell_mem[q] = i;
    w.cell_pos[q] = p;
    w.cell_scr[q] = make_float4((float)(t - (ws.xmin + gx * G.lx)), ry, sr, idb);
    w.cell_up[q] = up;
  }
}

// ---------------------------------------------------------------------------
// a5-a15: updateContacts.  One thread per owner (memory position m) scans the
// 3x3 neighbourhood (PeriodicBoundaryWorld.cpp:47-84,
// LeesEdwardsBoundaryWorld.cpp:128-204), evaluates every candidate with a
// larger id at its image offset (PeriodicBoundaryWorld.cpp:97-101,
// LeesEdwardsBoundaryWorld.cpp:233-279), and writes the contacts into its
// records of the new record set:
//   - new contact: initial shear overlap and damping constant (BaseParticle.cpp:38-65)
//   - old contact: shear overlap rotated with the normal (BaseParticle.cpp:67-82)
//   - candidate not in contact: dropped (BaseParticle.cpp:95)
//   - history of a pair that is no longer a candidate: carried over unchanged,
//     as the reference's map entry is.
// FOLD_BG adds the Lees-Edwards background velocity on the fly, bit for bit the
// value applyBackgroudVelocity would have stored.
// ---------------------------------------------------------------------------

template <bool FOLD_BG>
__device__ __forceinline__ PState load_state(const DevWorld& w, const WorldScalars& ws, int m) {
  PState p;
  p.shape = w.shape[m];
  p.r = w.rad[m];
  p.asp = w.asp[m];
  double2 q = w.pos[m];
  double2 v = w.vel[m];
  p.x = q.x;
  p.y = q.y;
  p.vx = FOLD_BG ? v.x + ws.shift_rate * q.y : v.x;
  p.vy = v.y;
  p.rot = w.rot[m];
  p.w = w.w[m];
  return p;
}

// the state load_state gives, from a body record
template <bool FOLD_BG>
__device__ __forceinline__ PState body_state(const BodyRec& b, const WorldScalars& ws) {
  PState p;
  p.shape = b.shape;
  p.r = b.r;
  p.asp = b.asp;
  p.x = b.pos.x;
  p.y = b.pos.y;
  p.vx = FOLD_BG ? b.vel.x + ws.shift_rate * b.pos.y : b.vel.x;
  p.vy = b.vel.y;
  p.rot = b.rot;
  p.w = b.w;
  return p;
}

// vertices of a wall segment from its record (zero for other shapes)
__device__ __forceinline__ double4 seg_of(const DevWorld& w, const BodyRec& b) {
  return b.shape == SHAPE_SEGMENT ? w.seg[b.id] : double4{};
}

// damping constant of a new contact (the records carry the settings)
__device__ __forceinline__ double damping_of(const DevWorld& w, double factor, const BodyRec& bi,
                                             const BodyRec& bj, int mi, int mj) {
  // calculateDampingConstact (ContactModel_LinearDissipativeFrictional.cpp:73-82)
  // selected by SKIP_TIME_INTEGRAL (BaseParticle.cpp:53-64)
  const int si = bi.setting & SKIP_TIME_INTEGRAL, sj = bj.setting & SKIP_TIME_INTEGRAL;
  const double a = w.mass[mi], b = w.mass[mj];
  if (!si && sj) return sqrt(a) * factor;
  if (si && !sj) return sqrt(b) * factor;
  return sqrt((a * b) / (a + b)) * factor;
}

// small insertion sorts of keys held in local arrays
template <class T>
__device__ __forceinline__ void isort(T* key, int cnt) {
  for (int a = 1; a < cnt; ++a) {
    T x = key[a];
    int b = a - 1;
    while (b >= 0 && key[b] > x) {
      key[b + 1] = key[b];
      --b;
    }
    key[b + 1] = x;
  }
}

// ---------------------------------------------------------------------------
// a16: collectForceAndTorque (BaseWorld.cpp:17-57).  Each particle sums, in a
// fixed order, the contacts owned by lower ids (ascending owner id; -F and
// torqueOnP2) and then its own contacts (ascending partner id; F and
// torqueOnP1), starting from zero as the reference's per-thread arrays do.
// Particles with no contact are rattlers (BaseWorld.cpp:25,44-45).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void cmp_swap(T& a, T& b) {
  const T lo = a < b ? a : b, hi = a < b ? b : a;
  a = lo;
  b = hi;
}

// ascending sort of eight keys held in registers (a 19-comparator network)
template <class T>
__device__ __forceinline__ void sort8(T* k) {
  cmp_swap(k[0], k[1]); cmp_swap(k[2], k[3]); cmp_swap(k[4], k[5]); cmp_swap(k[6], k[7]);
  cmp_swap(k[0], k[2]); cmp_swap(k[1], k[3]); cmp_swap(k[4], k[6]); cmp_swap(k[5], k[7]);
  cmp_swap(k[1], k[2]); cmp_swap(k[5], k[6]); cmp_swap(k[0], k[4]); cmp_swap(k[3], k[7]);
  cmp_swap(k[1], k[5]); cmp_swap(k[2], k[6]); cmp_swap(k[1], k[4]); cmp_swap(k[3], k[6]);
  cmp_swap(k[2], k[4]); cmp_swap(k[3], k[5]); cmp_swap(k[3], k[4]);
}

// the force sum of the particle at p: written to force, torque, ncp and
// rattler, and returned in (Fo, To, rat)
__device__ __forceinline__ void collect_at(const DevWorld& w, int par, int p, double2& Fo,
                                           double& To, int& rat) {
  const int n = w.n, K = w.K;
  const Slots& cur = w.slots[par];
  int nown = min(cur.count[p], K);
  const int base = nown > 0 ? cur.base[p] : 0;
  int ninc = min(w.incnt[p], K);
  double fx = 0.0, fy = 0.0, t = 0.0;
  if (ninc <= 8 && nown <= 8) {
    // the usual case: both key sets sorted in registers, every load of a set
    // in flight at once; the same order and operations as below
    uint64_t ki[8];
    uint32_t ko[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      ki[a] = a < ninc ? w.inref[(size_t)a * n + p] : ~0ull;
      const int partner = a < nown ? cur.partner[base + a] : -1;
      ko[a] = partner >= 0 ? (((uint32_t)partner << 5) | (uint32_t)a) : 0xffffffffu;
    }
    sort8(ki);
    sort8(ko);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (a < ninc) {
        const size_t ci = (uint32_t)ki[a];
        const double2 F = cur.f[ci];
        fx += -F.x;
        fy += -F.y;
        t += cur.t2[ci];
      }
    }
    int nk = 0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      if (ko[a] != 0xffffffffu) {
        const size_t ci = (size_t)base + (ko[a] & 31u);
        const double2 F = cur.f[ci];
        fx += F.x;
        fy += F.y;
        t += cur.t1[ci];
        ++nk;
      }
    }
    Fo = make_double2(fx, fy);
    To = t;
    rat = (nk + ninc) == 0 ? 1 : 0;
    w.force[p] = Fo;
    w.torque[p] = t;
    w.ncp[p] = nk + ninc;
    w.rattler[p] = rat;
    return;
  }
  {
    uint64_t key[kMaxSlots];  // owner id << 32 | reference
    for (int a = 0; a < ninc; ++a) key[a] = w.inref[(size_t)a * n + p];
    isort(key, ninc);
    for (int a = 0; a < ninc; ++a) {
      size_t ci = (uint32_t)key[a];
      double2 F = cur.f[ci];
      fx += -F.x;
      fy += -F.y;
      t += cur.t2[ci];
    }
  }
  {
    uint32_t key[kMaxSlots];  // partner id << 5 | slot; empty slots skipped
    int nk = 0;
    for (int a = 0; a < nown; ++a) {
      int partner = cur.partner[base + a];
      if (partner >= 0) key[nk++] = ((uint32_t)partner << 5) | a;
    }
    nown = nk;
    isort(key, nown);
    for (int a = 0; a < nown; ++a) {
      size_t ci = (size_t)base + (key[a] & 31u);
      double2 F = cur.f[ci];
      fx += F.x;
      fy += F.y;
      t += cur.t1[ci];
    }
  }
  Fo = make_double2(fx, fy);
  To = t;
  rat = (nown + ninc) == 0 ? 1 : 0;
  w.force[p] = Fo;
  w.torque[p] = t;
  w.ncp[p] = nown + ninc;
  w.rattler[p] = rat;
}

__global__ void __launch_bounds__(128) k_collect(DevWorld w, int par) {
  if (stopped(w)) return;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= w.n) return;
  double2 F;
  double T;
  int rat;
  collect_at(w, par, p, F, T, rat);
}

// GluedParticle::isRattlerParticle (GluedParticle.cpp:141-147)
__device__ __forceinline__ bool is_rattler(const DevWorld& w, int m) {
  if (w.shape[m] == SHAPE_CLUMP) {
    int ns = w.num_sub[m], id = w.id_of[m];
    for (int k = 1; k <= ns; ++k)
      if (!w.rattler[w.mpos[id + k]]) return false;
    return true;
  }
  return w.rattler[m] != 0;
}

// ---------------------------------------------------------------------------
// a17/a18/a19: takeTimeIntegral (BaseWorld.cpp:59-77; BaseParticle.cpp:107-118;
// GluedParticle.cpp:91-125), then optionally resetVelocityOfRattlers
// (BaseWorld.cpp:79-92).  FOLD_BG first removes the Lees-Edwards background
// velocity exactly as removeBackgroudVelocity would after applyBackgroudVelocity.
// ---------------------------------------------------------------------------
// SUMS: the particle's force, torque and rattler flag come from the caller
// (k_collect_integrate, a world without clumps) instead of memory
template <bool FOLD_BG, bool SUMS>
__device__ __forceinline__ void integrate_at(const DevWorld& w, int i, int reset_rattlers,
                                             double2 Fs, double Ts, int rat) {
  const WorldScalars& ws = w.ws[sys_at(w, i)];
  const double dt = ws.dt, g = ws.g;
  const int set = w.setting[i];
  const int id = w.id_of[i];
  double2 v = w.vel[i];
  if (FOLD_BG) {
    double y = w.pos[i].y;
    v.x = (v.x + ws.shift_rate * y) - ws.shift_rate * y;
  }
  if (set & SKIP_TIME_INTEGRAL) {
    // a sub-particle's velocity is rewritten by its clump below
    if (FOLD_BG && w.up[i] == id) w.vel[i] = v;
    if (reset_rattlers && !(set & SKIP_MACRO_SUM) && w.up[i] == id && is_rattler(w, i)) {
      w.vel[i] = make_double2(0.0, 0.0);
      w.w[i] = 0.0;
    }
    return;
  }
  double2 p = w.pos[i];
  double om = w.w[i];
  // (SUMS: a world without clumps; the branch is left out of that kernel)
  if (!SUMS && w.shape[i] == SHAPE_CLUMP) {
    vec2<double> F = V(0.0, 0.0);
    double T = 0.0;
    const int ns = w.num_sub[i];
    for (int k = 1; k <= ns; ++k) {
      int sk = w.mpos[id + k];
      double2 fk = w.force[sk];
      double2 bk = w.branch[sk];
      F = F + V(fk.x, fk.y);
      T += w.torque[sk];
      T += cross(V(bk.x, bk.y), V(fk.x, fk.y));
    }
    vec2<double> vv = (V(v.x, v.y) * (1.0 - g * dt) + (F * w.im[i]) * dt) / (1.0 + g * dt);
    p.x += vv.x * dt;
    p.y += vv.y * dt;
    om = (om * (1.0 - g * dt) + T * w.iI[i] * dt) / (1.0 + g * dt);
    double rot = w.rot[i] + om * dt;
    double angle = om * dt;
    double ca = cos(angle), sa = sin(angle);
    mat2<double> R = M(ca, -sa, sa, ca);
    for (int k = 1; k <= ns; ++k) {
      int sk = w.mpos[id + k];
      double2 bk = w.branch[sk];
      vec2<double> b = R * V(bk.x, bk.y);
      w.branch[sk] = make_double2(b.x, b.y);
      vec2<double> sv = vv + crossw(b, om);
      w.vel[sk] = make_double2(sv.x, sv.y);
      if (w.V) {  // path length for the candidate lists
        // the sub-particle's move from its stored position, which a box law
        // may have scaled apart from the clump's centre plus its branch; the
        // periodic wrap moves each body on its own, so a wrap of the
        // sub-particle alone shows here as a jump of one box image, which is
        // no move and is taken out (a wrap across the sheared edge already
        // rebuilds the lists)
        const double2 op = w.pos[sk];
        double ex = (p.x + b.x) - op.x, ey = (p.y + b.y) - op.y;
        if (w.kind == WORLD_LE) {
          if (ey > 0.5 * ws.ylen) {
            ey -= ws.ylen;
            ex -= ws.shift;
          } else if (ey < -0.5 * ws.ylen) {
            ey += ws.ylen;
            ex += ws.shift;
          }
        } else {
          ey -= ws.ylen * rint(ey / ws.ylen);
        }
        ex -= ws.xlen * rint(ex / ws.xlen);
        w.vl_disp[sk] += sqrt(ex * ex + ey * ey);
      }
      w.pos[sk] = make_double2(p.x + b.x, p.y + b.y);
      w.w[sk] = om;
      w.rot[sk] += angle;
    }
    if (w.V) w.vl_disp[i] += sqrt(vv.x * vv.x + vv.y * vv.y) * dt;
    if (!(isfinite(p.x) && isfinite(p.y) && isfinite(vv.x) && isfinite(vv.y) && isfinite(om)))
      raise(w.status, ST_NONFINITE);
    w.pos[i] = p;
    w.rot[i] = rot;
    if (reset_rattlers && !(set & SKIP_MACRO_SUM) && is_rattler(w, i)) {
      w.vel[i] = make_double2(0.0, 0.0);
      w.w[i] = 0.0;
    } else {
      w.vel[i] = make_double2(vv.x, vv.y);
      w.w[i] = om;
    }
    return;
  }
  double2 F = SUMS ? Fs : w.force[i];
  double im = w.im[i];
  vec2<double> vv = (V(v.x, v.y) * (1.0 - g * dt) + (V(F.x, F.y) * im) * dt) / (1.0 + g * dt);
  p.x += vv.x * dt;
  p.y += vv.y * dt;
  om = (om * (1.0 - g * dt) + (SUMS ? Ts : w.torque[i]) * w.iI[i] * dt) / (1.0 + g * dt);
  if (w.V) w.vl_disp[i] += sqrt(vv.x * vv.x + vv.y * vv.y) * dt * seg_path_factor(w, i);  // candidate lists
  // a non-finite state raises XDEM_ERR_NONFINITE (the reference carries NaN
  // on without a word)
  if (!(isfinite(p.x) && isfinite(p.y) && isfinite(vv.x) && isfinite(vv.y) && isfinite(om)))
    raise(w.status, ST_NONFINITE);
  w.pos[i] = p;
  w.rot[i] = w.rot[i] + om * dt;
  if (reset_rattlers && !(set & SKIP_MACRO_SUM) && (SUMS ? rat : w.rattler[i])) {
    w.vel[i] = make_double2(0.0, 0.0);
    w.w[i] = 0.0;
  } else {
    w.vel[i] = make_double2(vv.x, vv.y);
    w.w[i] = om;
  }
}

template <bool FOLD_BG>
__global__ void k_integrate(DevWorld w, int reset_rattlers) {
  if (stopped(w)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  integrate_at<FOLD_BG, false>(w, i, reset_rattlers, make_double2(0.0, 0.0), 0.0, 0);
}


// BaseWorld::resetVelocityOfRattlers / scaleVelocityOfRattlers (BaseWorld.cpp:79-106)
__global__ void k_rattlers(DevWorld w, int reset, double scale) {
  if (stopped(w)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w.n) return;
  if (w.setting[i] & SKIP_MACRO_SUM) return;
  if (!is_rattler(w, i)) return;
  if (reset) {
    w.vel[i] = make_double2(0.0, 0.0);
    w.w[i] = 0.0;
  } else {
    double2 v = w.vel[i];
    w.vel[i] = make_double2(v.x * scale, v.y * scale);
    w.w[i] = w.w[i] * scale;
  }
}

// ---------------------------------------------------------------------------
// a21: updateTotalStress (BaseWorld.cpp:158-176) with getStressFromContactList
// of BaseParticle (BaseParticle.cpp:143-151) and GluedParticle
// (GluedParticle.cpp:127-139).  Per-particle sums in ascending partner order,
// then a fixed tree over the memory order, which is a deterministic function
// of the state: deterministic run to run.
// ---------------------------------------------------------------------------
constexpr int kReduceBlock = 256;

__device__ __forceinline__ void own_stress(const DevWorld& w, const Slots& cur, int p, bool sub,
                                           double2 bvo, mat2<double>& s) {
  const int K = w.K;
  int c0 = min(cur.count[p], K), cnt = 0;
  if (c0 <= 0) return;
  const int base = cur.base[p];
  uint32_t key[kMaxSlots];
  for (int a = 0; a < c0; ++a) {
    int partner = cur.partner[base + a];
    if (partner >= 0) key[cnt++] = ((uint32_t)partner << 5) | a;
  }
  isort(key, cnt);
  for (int a = 0; a < cnt; ++a) {
    size_t ci = (size_t)base + (key[a] & 31u);
    double2 F = cur.f[ci], b = cur.b[ci];
    vec2<double> bb = V(b.x, b.y);
    if (sub) bb = bb + V(bvo.x, bvo.y);
    s = s + dyad(V(F.x, F.y), bb);
  }
}

// the stress contribution of the body at memory position p
__device__ __forceinline__ mat2<double> body_stress(const DevWorld& w, const Slots& cur, int p) {
  mat2<double> s = M(0.0, 0.0, 0.0, 0.0);
  if (w.setting[p] & SKIP_MACRO_SUM) return s;
  if (w.shape[p] == SHAPE_CLUMP) {
    // one running sum over all sub-particles (GluedParticle.cpp:128-137)
    int id = w.id_of[p];
    for (int k = 1; k <= w.num_sub[p]; ++k) {
      int sk = w.mpos[id + k];
      own_stress(w, cur, sk, true, w.branch[sk], s);
    }
  } else {
    own_stress(w, cur, p, false, make_double2(0.0, 0.0), s);
  }
  return s;
}

// batched worlds: one block per system sums the system's bodies (its memory
// range) in a fixed tree and divides by its box area
__global__ void __launch_bounds__(kReduceBlock) k_stress_systems(DevWorld w, int par) {
  if (stopped(w)) return;
  __shared__ double sh[4][kReduceBlock];
  WorldScalars& ws = w.ws[blockIdx.x];
  const Slots& cur = w.slots[par];
  const int t = threadIdx.x;
  mat2<double> s = M(0.0, 0.0, 0.0, 0.0);
  for (int p = ws.first + t; p < ws.first + ws.count; p += kReduceBlock) s = s + body_stress(w, cur, p);
  sh[0][t] = s.xx;
  sh[1][t] = s.xy;
  sh[2][t] = s.yx;
  sh[3][t] = s.yy;
  __syncthreads();
  for (int off = kReduceBlock / 2; off > 0; off >>= 1) {
    if (t < off)
      for (int c = 0; c < 4; ++c) sh[c][t] += sh[c][t + off];
    __syncthreads();
  }
  if (t == 0) {
    double area = ws.xlen * ws.ylen;
    for (int c = 0; c < 4; ++c) ws.stress[c] = sh[c][0] / area;
  }
}

__global__ void __launch_bounds__(kReduceBlock) k_stress_partial(DevWorld w, int par) {
  if (stopped(w)) return;
  __shared__ double sh[4][kReduceBlock];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  mat2<double> s = M(0.0, 0.0, 0.0, 0.0);
  if (p < w.n) s = body_stress(w, w.slots[par], p);
  int t = threadIdx.x;
  sh[0][t] = s.xx;
  sh[1][t] = s.xy;
  sh[2][t] = s.yx;
  sh[3][t] = s.yy;
  __syncthreads();
  for (int off = kReduceBlock / 2; off > 0; off >>= 1) {
    if (t < off)
      for (int c = 0; c < 4; ++c) sh[c][t] += sh[c][t + off];
    __syncthreads();
  }
  if (t == 0)
    for (int c = 0; c < 4; ++c) w.partials[(size_t)c * gridDim.x + blockIdx.x] = sh[c][0];
}

// sums nblocks partials in a fixed tree; divides by the box area
__global__ void k_stress_final(DevWorld w, int nblocks) {
  WorldScalars& ws = *w.ws;
  if (ws.stop) return;  // single-system worlds only
  __shared__ double sh[4][1024];
  int t = threadIdx.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = t; b < nblocks; b += blockDim.x)
    for (int c = 0; c < 4; ++c) acc[c] += w.partials[(size_t)c * nblocks + b];
  for (int c = 0; c < 4; ++c) sh[c][t] = acc[c];
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (t < off)
      for (int c = 0; c < 4; ++c) sh[c][t] += sh[c][t + off];
    __syncthreads();
  }
  if (t == 0) {
    double area = ws.xlen * ws.ylen;
    for (int c = 0; c < 4; ++c) ws.stress[c] = sh[c][0] / area;
  }
}

// ---------------------------------------------------------------------------
// a20: PeriodicControlWorld box laws (PeriodicControlWorld.cpp:124-237).  One
// thread updates the box and leaves the affine scale for k_scale_positions.
// ---------------------------------------------------------------------------
enum : int { BOX_NONE = 0, BOX_STRAIN = 1, BOX_STRESS_XY = 2, BOX_STRESS_UNIFORM = 3,
             BOX_STRESS_UNIFORM_LIMIT = 4 };

__device__ __forceinline__ void box_law(WorldScalars& ws, int law, double p0, double p1) {
  const double dt = ws.dt;
  const double kMaxScaleRate = 100000000.0;
  ws.scale_x = 1.0;
  ws.scale_y = 1.0;
  if (law == BOX_STRAIN) {
    double sx = 1.0 + p0 * ws.xlen * dt;
    double sy = 1.0 + p1 * ws.ylen * dt;
    ws.xmin *= sx;
    ws.xmax *= sx;
    ws.ymin *= sy;
    ws.ymax *= sy;
    ws.xlen = ws.xmax - ws.xmin;
    ws.ylen = ws.ymax - ws.ymin;
    ws.scale_x = sx;
    ws.scale_y = sy;
  } else if (law == BOX_STRESS_UNIFORM) {
    double hydro = (ws.stress[0] + ws.stress[3]) / 2.0;
    double dv = (p0 - hydro) * ws.xlen * dt;
    ws.velX += dv;
    ws.velY = ws.velX;
    double scale = (ws.xmin + dv * dt) / ws.xmin;
    ws.xmin += dv * dt;
    ws.xmax = -ws.xmin;
    ws.xlen = ws.xmax - ws.xmin;
    ws.ymin += dv * dt;
    ws.ymax = -ws.ymin;
    ws.ylen = ws.ymax - ws.ymin;
    ws.scale_x = scale;
    ws.scale_y = scale;
  } else if (law == BOX_STRESS_XY) {
    // stressControlX then stressControlY; the two scales compose into one
    // pass because each multiplies a different coordinate
    double pre = ws.xmin;
    double sxx = ws.stress[0];
    if (fabs(sxx) < p0) ws.velX *= (1.0 - dt * 1.0);
    double dv = (p0 - sxx) * ws.xlen / ws.vmass * dt;
    ws.velX = dv;
    if (fabs(ws.velX) / ws.xlen > kMaxScaleRate * dt) ws.velX = kMaxScaleRate * dt * ws.xlen;
    ws.xmin += ws.velX * dt;
    ws.xmax = -ws.xmin;
    ws.xlen = ws.xmax - ws.xmin;
    ws.scale_x = ws.xmin / pre;
    pre = ws.ymin;
    double syy = ws.stress[3];
    if (fabs(syy) < p0) ws.velY *= (1.0 - dt * 1.0);
    dv = (p0 - syy) * ws.ylen / ws.vmass * dt;
    ws.velY = dv;
    if (fabs(ws.velY) / ws.ylen > kMaxScaleRate * dt) ws.velY = kMaxScaleRate * dt * ws.ylen;
    ws.ymin += ws.velY * dt;
    ws.ymax = -ws.ymin;
    ws.ylen = ws.ymax - ws.ymin;
    ws.scale_y = ws.ymin / pre;
  } else if (law == BOX_STRESS_UNIFORM_LIMIT) {
    double prex = ws.xmin;
    double hydro = (ws.stress[0] + ws.stress[3]) / 2.0;
    double dv = (p0 - hydro) * ws.xlen * dt;
    ws.velX += dv;
    if ((fabs(ws.velX) / (ws.xlen / 2.0)) > ws.max_strain_rate)
      ws.velX = fabs(ws.velX) / ws.velX * (ws.xlen / 2.0) * ws.max_strain_rate;
    ws.velY = ws.velX;
    ws.xmin += ws.velX * dt;
    ws.xmax = -ws.xmin;
    ws.xlen = ws.xmax - ws.xmin;
    ws.ymin += ws.velY * dt;
    ws.ymax = -ws.ymin;
    ws.ylen = ws.ymax - ws.ymin;
    double scale = ws.xmin / prex;
    ws.scale_x = scale;
    ws.scale_y = scale;
  }
}

// End-of-step scalar work: Lees-Edwards update (LeesEdwardsBoundaryWorld.cpp:
// 285-296, part of its takeTimeStep), then the driver's box law, the step
// count and the stop test.  After a stop the scales are 1.
// One thread per system; the run-level counters and the stop test (single
// systems only) belong to system 0.
// the end of a step for system sys (k_end_of_step)
__device__ __forceinline__ void end_of_step_at(const DevWorld& w, int sys, int law, double p0,
                                               double p1, int le_update, int stop_on_pressure,
                                               double stop_pressure, int count_step) {
  WorldScalars& ws = w.ws[sys];
  if (stopped(w)) {
    ws.scale_x = 1.0;
    ws.scale_y = 1.0;
    return;
  }
  if (le_update) {
    ws.shift_vel = ws.shift_rate * ws.ylen;
    ws.strain += ws.shift_rate * ws.dt;
    ws.shift += ws.shift_vel * ws.dt;
    if (ws.shift > ws.xmax) ws.shift -= ws.xlen;
    else if (ws.shift < ws.xmin) ws.shift += ws.xlen;
    // pairs across the sheared edge move apart by the shift travelled
    ws.vl_travel += fabs(ws.shift_vel * ws.dt);
  }
  if (law != BOX_NONE) {
    box_law(ws, law, p0, p1);
    // an affine scale s moves a pair at distance d by |s - 1| d
    ws.vl_travel += fmax(fabs(ws.scale_x - 1.0), fabs(ws.scale_y - 1.0)) * (ws.maxsize + w.skin);
  }
  if (sys != 0) return;
  if (count_step) {
    ws.steps_done += 1;
    ws.flips += 1;
  }
  if (stop_on_pressure && (ws.stress[0] + ws.stress[3]) / 2.0 >= stop_pressure) ws.stop = 1;
}

__global__ void k_end_of_step(DevWorld w, int law, double p0, double p1, int le_update,
                              int stop_on_pressure, double stop_pressure, int count_step) {
  const int sys = blockIdx.x * blockDim.x + threadIdx.x;
  if (sys >= w.nsys) return;
  end_of_step_at(w, sys, law, p0, p1, le_update, stop_on_pressure, stop_pressure, count_step);
}

// k_collect then k_integrate, one thread per particle, for a world without
// clumps (a body's time integral then reads only its own sums): the force,
// torque and rattler flag go from the sum to the integral in registers.  (The
// step's end taken by the last block to finish, with a fence in every thread
// before the count of finished blocks, measured slower than its own launch:
// 0.081 + 0.007 ms against 0.089 ms at 1M.)
template <bool FOLD_BG>
__global__ void __launch_bounds__(128) k_collect_integrate(DevWorld w, int par, int reset_rattlers) {
  pdl_begin();
  if (stopped(w)) return;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < w.n) {
    double2 F;
    double T;
    int rat;
    collect_at(w, par, p, F, T, rat);
    integrate_at<FOLD_BG, true>(w, p, reset_rattlers, F, T, rat);
  }
}

// kinetic energy (BaseWorld.cpp:302-310), fixed-tree sum
__global__ void __launch_bounds__(kReduceBlock) k_ke_partial(DevWorld w) {
  __shared__ double sh[kReduceBlock];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (p < w.n) {
    double2 v = w.vel[p];
    double om = w.w[p];
    e = 0.5 * (w.mass[p] * (v.x * v.x + v.y * v.y) + w.I[p] * om * om);
  }
  int t = threadIdx.x;
  sh[t] = e;
  __syncthreads();
  for (int off = kReduceBlock / 2; off > 0; off >>= 1) {
    if (t < off) sh[t] += sh[t + off];
    __syncthreads();
  }
  if (t == 0) w.partials[blockIdx.x] = sh[0];
}

__global__ void k_ke_final(DevWorld w, int nblocks) {
  __shared__ double sh[1024];
  int t = threadIdx.x;
  double acc = 0.0;
  for (int b = t; b < nblocks; b += blockDim.x) acc += w.partials[b];
  sh[t] = acc;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (t < off) sh[t] += sh[t + off];
    __syncthreads();
  }
  if (t == 0) w.ws->ke = sh[0];
}

// id-ordered staging of the dynamic state (x, y, vx, vy, rot, rot_vel blocks
// of n doubles each) <-> memory order
__global__ void k_stage(DevWorld w, int to_world) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= w.n) return;
  const int n = w.n;
  const int m = w.mpos[id];
  double* s = w.stage;
  if (to_world) {
    if (w.V) {  // the host's move counts toward the candidate lists' skin
      const double2 op = w.pos[m];
      const double ex = s[id] - op.x, ey = s[n + id] - op.y;
      w.vl_disp[m] += sqrt(ex * ex + ey * ey) * seg_path_factor(w, m);
    }
    w.pos[m] = make_double2(s[id], s[n + id]);
    w.vel[m] = make_double2(s[2 * n + id], s[3 * n + id]);
    w.rot[m] = s[4 * n + id];
    w.w[m] = s[5 * n + id];
  } else {
    double2 p = w.pos[m], v = w.vel[m];
    s[id] = p.x;
    s[n + id] = p.y;
    s[2 * n + id] = v.x;
    s[3 * n + id] = v.y;
    s[4 * n + id] = w.rot[m];
    s[5 * n + id] = w.w[m];
  }
}

// single-pair geometry for known-answer tests (xdem_pair_geometry)
__global__ void k_pair_geometry(int npairs, int method, const double* pi, const double* pj,
                                const double* off, double* out, uint32_t* status) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const double* a = pi + 9 * k;
  const double* b = pj + 9 * k;
  PState A{(int)a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]};
  PState B{(int)b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8]};
  double2 csa = make_double2(cos(A.rot), sin(A.rot));
  double2 csb = make_double2(cos(B.rot), sin(B.rot));
  Geom g;
  uint32_t st = 0;
  bool c = contact_geometry(method, A, B, a[1], b[1], V(off[4 * k], off[4 * k + 1]),
                            V(off[4 * k + 2], off[4 * k + 3]), csa, csb, g, st);
  double* o = out + 17 * k;
  o[0] = c ? 1.0 : 0.0;
  o[1] = g.n.x;
  o[2] = g.n.y;
  o[3] = g.cp.x;
  o[4] = g.cp.y;
  o[5] = g.bv1.x;
  o[6] = g.bv1.y;
  o[7] = g.bv2.x;
  o[8] = g.bv2.y;
  o[9] = g.overlap;
  o[10] = g.rv.x;
  o[11] = g.rv.y;
  o[12] = g.nrv.x;
  o[13] = g.nrv.y;
  o[14] = g.srv.x;
  o[15] = g.srv.y;
  o[16] = (double)g.iters;
  if (st) atomicOr(status, st);
}

}  // namespace xdem
