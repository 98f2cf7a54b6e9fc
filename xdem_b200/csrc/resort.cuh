// resort.cuh — refreshes the memory order of a world (world.cuh).
//
// Runs after a step's binning: particles are ordered by regular cell, ties by
// id (k_sort_cells, deterministic), every particle array is moved to its new
// position through a scratch slab and copied back (array addresses stay fixed,
// so captured graphs stay valid), each owner's record count and first record
// move with it into the other record set (the records keep their indices; the
// next update overwrites them anyway), and the cell lists are renumbered.  Nothing the reference computes depends on the memory order.
#pragma once
#include "kernels.cuh"

namespace xdem {

constexpr int kMaxPermArrays = 28;

struct PermList {
  void* base[kMaxPermArrays];
  size_t offset[kMaxPermArrays];  // byte offset of the array's slab in scratch
  int esize[kMaxPermArrays];      // 4, 8 or 16 bytes
  int count;
};

// members of each regular cell in ascending id, their screening copies moved
// along; newpos = the sorted index
__global__ void k_sort_cells(DevWorld w) {
  if (stopped(w)) return;
  // memory positions move: the candidate lists hold them
  if (blockIdx.x == 0 && threadIdx.x == 0) w.ws->vl_valid = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w.ncell_total;
       c += gridDim.x * blockDim.x) {
    const Grid G = grid_of(w.ws[sys_of_cell(w, c)]);
    // regular cells of a valid grid only (ghost rows hold images)
    if (G.nx < 3 || G.ny < 3 || c - G.base >= G.ncell) continue;
    int q0 = w.cell_start[c], q1 = w.cell_start[c + 1];
    for (int a = q0 + 1; a < q1; ++a) {
      const int x = w.cell_mem[a];
      const double2 px = w.cell_pos[a];
      const float4 rx = w.cell_scr[a];
      const int ux = w.cell_up[a];
      const int kx = w.id_of[x];
      int b = a - 1;
      while (b >= q0 && w.id_of[w.cell_mem[b]] > kx) {
        w.cell_mem[b + 1] = w.cell_mem[b];
        w.cell_pos[b + 1] = w.cell_pos[b];
        w.cell_scr[b + 1] = w.cell_scr[b];
        w.cell_up[b + 1] = w.cell_up[b];
        --b;
      }
      w.cell_mem[b + 1] = x;
      w.cell_pos[b + 1] = px;
      w.cell_scr[b + 1] = rx;
      w.cell_up[b + 1] = ux;
    }
    for (int q = q0; q < q1; ++q) w.newpos[w.cell_mem[q]] = q;
  }
}

template <int E>
struct Elem;
template <>
struct Elem<4> {
  using T = int32_t;
};
template <>
struct Elem<8> {
  using T = double;
};
template <>
struct Elem<16> {
  using T = double2;
};

template <int E>
__device__ __forceinline__ void move_elem(void* src, int si, void* dst, int di) {
  using T = typename Elem<E>::T;
  static_cast<T*>(dst)[di] = static_cast<const T*>(src)[si];
}

// every array element m -> scratch slab at newpos[m]; mpos follows
__global__ void k_permute(DevWorld w, PermList L) {
  if (stopped(w)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  const Grid G = grid_of(w.ws[sys_at(w, m)]);
  if (G.nx < 3 || G.ny < 3) return;
  int t = w.newpos[m];
  w.mpos[w.id_of[m]] = t;
  for (int a = 0; a < L.count; ++a) {
    void* dst = w.scratch + L.offset[a];
    switch (L.esize[a]) {
      case 4: move_elem<4>(L.base[a], m, dst, t); break;
      case 8: move_elem<8>(L.base[a], m, dst, t); break;
      default: move_elem<16>(L.base[a], m, dst, t); break;
    }
  }
}

__global__ void k_copy_back(DevWorld w, PermList L) {
  if (stopped(w)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  // a system keeps its memory range, so the slab entry at m was written by a
  // particle of the same system
  const Grid G = grid_of(w.ws[sys_at(w, m)]);
  if (G.nx < 3 || G.ny < 3) return;
  for (int a = 0; a < L.count; ++a) {
    void* src = w.scratch + L.offset[a];
    switch (L.esize[a]) {
      case 4: move_elem<4>(src, m, L.base[a], m); break;
      case 8: move_elem<8>(src, m, L.base[a], m); break;
      default: move_elem<16>(src, m, L.base[a], m); break;
    }
  }
}

// history of the owner at m -> record set par^1: its count and first record
// go to newpos[m], its records keep their indices; counts one swap.  With an
// invalid grid the particles did not move and the history is copied in
// place, so that the record-set parity stays what the host expects.
__global__ void k_permute_history(DevWorld w, int par) {
  if (stopped(w)) return;
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) w.ws->flips += 1;
  if (m >= w.n) return;
  const Grid G = grid_of(w.ws[sys_at(w, m)]);
  const bool moved = G.nx >= 3 && G.ny >= 3;
  const int K = w.K;
  const Slots& src = w.slots[par];
  const Slots& dst = w.slots[par ^ 1];
  int t = moved ? w.newpos[m] : m;
  int c = min(src.count[m], K);
  const int base = c > 0 ? src.base[m] : 0;
  dst.count[t] = c;
  dst.base[t] = base;
  for (int s = 0; s < c; ++s) {
    const size_t a = (size_t)base + s;
    dst.partner[a] = src.partner[a];
    dst.n[a] = src.n[a];
    dst.s[a] = src.s[a];
    dst.damp[a] = src.damp[a];
    dst.f[a] = src.f[a];
    dst.t1[a] = src.t1[a];
    dst.t2[a] = src.t2[a];
    dst.b[a] = src.b[a];
    dst.cp[a] = src.cp[a];
    dst.bv1[a] = src.bv1[a];
    dst.bv2[a] = src.bv2[a];
    dst.fn[a] = src.fn[a];
    dst.ft[a] = src.ft[a];
  }
}

// cell lists hold positions: renumber them
__global__ void k_remap_cells(DevWorld w) {
  if (stopped(w)) return;
  int total = w.cell_start[w.ncell_total];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x)
    w.cell_mem[q] = w.newpos[w.cell_mem[q]];
}

}  // namespace xdem
