// verlet.cuh — candidate lists kept across steps (Verlet lists with a skin).
//
// The reference rescans the 3x3 cells of every particle each step
// (PeriodicBoundaryWorld.cpp:47-84).  A pair passes its coarse test only
// within the screening distance R = r_i + r_j (bounding circles for ellipses).
// Here each owner keeps the partners that were within R + skin at the last
// full scan, with the image kind the scan saw; each step only those are
// tested, with the reference's image offset and coarse test, so the listed
// pairs are exactly the full scan's as long as no pair has come closer by
// more than the skin since the build.  The lists are rebuilt (one full scan)
// when that budget — twice the largest path length of a particle since the
// build, plus the Lees-Edwards shift travelled and the affine box scaling of
// a pair at the cut-off distance — reaches the skin, after every re-sort
// (memory positions move), after the host changes positions or the box, and
// when a particle crosses the y edge of a Lees-Edwards world (its image kinds
// change).  What else the full scan decides is still decided every step from
// the cell grid: the `seen` mask of old partners and the 200-candidate cap
// (an exact count runs only where the nine cells hold that many records).
#pragma once
#include "pairs.cuh"

namespace xdem {

constexpr int kVlBlock = 256;
constexpr int kVlGroup = 2;  // list entries whose loads k_candidates_vl issues together

// block maxima of the path lengths since the last build
__global__ void __launch_bounds__(kVlBlock) k_vl_maxdisp(DevWorld w) {
  if (stopped(w)) return;
  __shared__ double sh[kVlBlock / 32];
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  double v = m < w.n ? w.vl_disp[m] : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int k = 0; k < kVlBlock / 32; ++k) mx = fmax(mx, sh[k]);
    w.vl_part[blockIdx.x] = mx;
  }
}

// whether this step rebuilds the lists (system 0's vl_build)
__global__ void __launch_bounds__(1024) k_vl_check(DevWorld w, int nblocks) {
  if (stopped(w)) return;
  __shared__ double sh[32];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmax(v, w.vl_part[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mx = fmax(mx, sh[k]);
    WorldScalars* ws = w.ws;
    bool rebuild = ws[0].vl_valid == 0;
    for (int s = 0; s < w.nsys && !rebuild; ++s)
      if (2.0 * mx + ws[s].vl_travel >= w.skin) rebuild = true;
    ws[0].vl_build = rebuild ? 1 : 0;
    if (rebuild) {
      for (int s = 0; s < w.nsys; ++s) ws[s].vl_travel = 0.0;
      ws[0].vl_valid = 1;
      ws[0].vl_builds += 1;
    }
  }
}

// One thread per owner: the full 3x3 scan with the reference's filters, the
// partners within R + skin (an FP32 test with a margin that only widens the
// list) kept as (memory position, image kind); the path lengths restart.  An
// owner with more partners than the list holds is marked (count -1) and
// scanned in full every step until the next build.
template <int LAW>
__global__ void __launch_bounds__(128) k_vl_build(DevWorld w) {
  if (stopped(w) || !w.ws->vl_build) return;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= w.n) return;
  w.vl_disp[m] = 0.0;
  const WorldScalars& ws = w.ws[sys_at(w, m)];
  const int n = w.n;
  int cnt = 0;
  const Grid G = grid_of(ws);
  if (G.nx >= 3 && G.ny >= 3 && !(w.setting[m] & SKIP_CONTACT_DETECTION)) {
    const double2 pi = w.pos[m];
    const int id_i = w.id_of[m], up_i = w.up[m];
    // the owner's cell from this step's binning (k_bin, the same cell_of)
    const int cell_local = w.pcell[m] - G.base;
    const int ix = cell_local % G.nx, iy = cell_local / G.nx;
    const float rxi = (float)(pi.x - (ws.xmin + ix * G.lx));
    const float ryi = (float)(pi.y - (ws.ymin + iy * G.ly));
    const float flx = (float)G.lx, fly = (float)G.ly;
    const float sr_i = screen_radius(w, m) + (float)w.skin;
#pragma unroll 1
    for (int k = 0; k < 9; ++k) {
      const int dx = k / 3 - 1, dy = k % 3 - 1;
      int kind;
      const int c = neighbour_cell(G, w.kind, ix, iy, dx, dy, kind);
      const int q0 = w.cell_start[c], q1 = w.cell_start[c + 1];
      const float ox = dx * flx - rxi, oy = dy * fly - ryi;
      for (int q = q0; q < q1; ++q) {
        const float4 rj = w.cell_scr[q];
        if (__float_as_int(rj.w) <= id_i) continue;
        if (w.cell_up[q] == up_i) continue;
        const float ddx = ox + rj.x, ddy = oy + rj.y;
        const float R = sr_i + rj.z;
        if (ddx * ddx + ddy * ddy > R * R * (1.0f + 1e-4f) + 1e-4f) continue;
        if (cnt >= w.V) {
          cnt = -1;
          break;
        }
        w.vl[(size_t)cnt * n + m] = (w.cell_mem[q] << 2) | kind;
        ++cnt;
      }
      if (cnt < 0) break;
    }
  }
  w.vl_cnt[m] = cnt;
}

// k_candidates with the lists: same outputs (body records, slot counts,
// carried-over history, the compact pair list), the same filters and
// tests.  Seven blocks per SM (72 registers): the kernel is latency-bound on
// its partner gathers, and six blocks with more registers measured slower.
template <int LAW>
__global__ void __launch_bounds__(128, 7) k_candidates_vl(DevWorld w, int par) {
  if (stopped(w)) return;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = m < w.n;
  const WorldScalars& ws = w.ws[valid ? sys_at(w, m) : 0];
  const int n = w.n, K = w.K;
  const Slots& old = w.slots[par];
  const Slots& cur = w.slots[par ^ 1];
  uint32_t st = 0;
  int nlist = 0;
  int32_t list_mj[kMaxSlots];
  int32_t list_code[kMaxSlots];
  if (valid) {
    write_owner_body<LAW>(w, m);
    const AxisShape shape_ax = owner_axis_shape<LAW>(w, m);
    const Grid G = grid_of(ws);
    const int id_i = w.id_of[m];
    const int nold = min(old.count[m], K);
    uint32_t seen = 0;
    if (G.nx >= 3 && G.ny >= 3 && !(w.setting[m] & SKIP_CONTACT_DETECTION)) {
      const double2 pi = w.pos[m];
      const int up_i = w.up[m];
      const int shape_i = (LAW == LAW_ANY) ? w.shape[m] : 0;
      const double r_i = w.rad[m], orad_i = w.orad[m];
      // the owner's cell from this step's binning (k_bin, the same cell_of)
      const int cell_local = w.pcell[m] - G.base;
      const int ix = cell_local % G.nx, iy = cell_local / G.nx;
      const int cnt = w.vl_cnt[m];
      // old slots of listed pairs known to be candidates now (see below)
      uint32_t matched = 0;
      if (cnt < 0) {  // the list overflowed at its build: the full scan
        scan_cells<LAW>(w, ws, G, m, ix, iy, pi, id_i, up_i, shape_i, r_i, orad_i, old, nold,
                        nlist, list_mj, list_code, st, matched, shape_ax);
      } else {
        // the 200-candidate cap (PeriodicBoundaryWorld.cpp:75-78): the nine
        // cells' record counts bound each kind's candidates; where a bound
        // reaches the cap, the candidates are counted as the full scan does
        // (skipped when no nine cells can hold that many records)
        int tot0 = 0, tot1 = 0, tot2 = 0;
        const bool cap_reachable = 9 * *w.cell_max + 1 >= kCandidateCap;
#pragma unroll
        for (int k = 0; k < 9 && cap_reachable; ++k) {
          int kind;
          const int c = neighbour_cell(G, w.kind, ix, iy, k / 3 - 1, k % 3 - 1, kind);
          const int cc = w.cell_start[c + 1] - w.cell_start[c];
          tot0 += kind == CAND_REGULAR ? cc : 0;
          tot1 += kind == CAND_TOP ? cc : 0;
          tot2 += kind == CAND_BOTTOM ? cc : 0;
        }
        if (tot0 + 1 >= kCandidateCap || tot1 + 1 >= kCandidateCap || tot2 + 1 >= kCandidateCap) {
          int c0 = 0, c1 = 0, c2 = 0;
          for (int k = 0; k < 9; ++k) {
            int kind;
            const int c = neighbour_cell(G, w.kind, ix, iy, k / 3 - 1, k % 3 - 1, kind);
            for (int q = w.cell_start[c]; q < w.cell_start[c + 1]; ++q) {
              if (__float_as_int(w.cell_scr[q].w) <= id_i || w.cell_up[q] == up_i) continue;
              int& nc = kind == CAND_REGULAR ? c0 : (kind == CAND_TOP ? c1 : c2);
              if (nc + 1 >= kCandidateCap) st |= ST_CAPACITY;
              else nc++;
            }
          }
        }
        // the first four old partners in registers (the usual case); the
        // others are read where they are
        int op[4];
#pragma unroll
        for (int z = 0; z < 4; ++z) op[z] = z < nold ? old.partner[(size_t)z * n + m] : -1;
        // the list in groups of kVlGroup entries: the group's entries,
        // positions and screening radii are loaded together (all in flight at
        // once), then tested one by one as before
        for (int v0 = 0; v0 < cnt; v0 += kVlGroup) {
          int eg[kVlGroup];
          double2 pg[kVlGroup];
          double sg[kVlGroup];
#pragma unroll
          for (int u = 0; u < kVlGroup; ++u)
            eg[u] = v0 + u < cnt ? w.vl[(size_t)(v0 + u) * n + m] : 0;
#pragma unroll
          for (int u = 0; u < kVlGroup; ++u) {
            const bool in = v0 + u < cnt;
            pg[u] = in ? w.pos[eg[u] >> 2] : make_double2(0.0, 0.0);
            sg[u] = (in && LAW != LAW_ANY) ? w.screen_r[eg[u] >> 2] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kVlGroup; ++u) {
          if (v0 + u >= cnt) break;
          const int e = eg[u];
          const int mj = e >> 2, kind = e & 3;
          const double2 pj = pg[u];
          vec2<double> off, ovel;
          image_offset(ws, kind, pi, pj, off, ovel);
          bool pass;
          if (LAW == LAW_ANY)
            pass = coarse_pass<LAW>(shape_i, w.shape[mj], r_i, w.rad[mj], orad_i, w.orad[mj], pi,
                                    pj, off);
          else
            pass = coarse_pass<LAW>(0, 0, r_i, sg[u], orad_i, sg[u], pi, pj, off);
          if (!pass) continue;
          int cls = CL_REGULAR;
          if (centre_line_screen<LAW>(w)) {
            cls = centre_line_class((float)((pj.x + off.x) - pi.x), (float)((pj.y + off.y) - pi.y),
                                    shape_ax, axis_shape(w, mj));
            if (cls == CL_SEPARATED) continue;
          }
          if (nlist >= K) {
            st |= ST_CAPACITY;
            continue;
          }
          const int id_j = w.id_of[mj];
          int oslot = kNoOldSlot;
#pragma unroll
          for (int z = 0; z < 4; ++z)
            if (op[z] == id_j) oslot = z;
          for (int z = 4; z < nold; ++z)
            if (old.partner[(size_t)z * n + m] == id_j) oslot = z;
          // a pair that passed a distance test lies within one cell size,
          // so it is a candidate of the 3x3 scan (LAW_ANY's other pairs pass
          // without one and take the cell test below)
          const bool near = LAW != LAW_ANY ||
                            (shape_i == w.shape[mj] &&
                             (shape_i == SHAPE_CIRCLE || shape_i == SHAPE_ELLIPSE));
          if (oslot != kNoOldSlot && near) matched |= 1u << oslot;
          list_mj[nlist] = mj;
          list_code[nlist] = kind | (nlist << 8) | (oslot << 16) |
                             (LAW == LAW_CLOSEST && cls == CL_DEEP ? kDeepFlag : 0);
          ++nlist;
          }
        }
      }
      // old partners among the candidates
      seen = matched;
      for (int z = 0; z < nold; ++z) {
        if (matched & (1u << z)) continue;
        const int p = old.partner[(size_t)z * n + m];
        if (p < 0) continue;
        const int mj = w.mpos[p];
        if (w.setting[mj] & SKIP_CONTACT_DETECTION) continue;
        if (w.up[mj] == up_i) continue;
        const int cr = w.pcell[mj], cg = w.gcell[mj];
        bool hit = false;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          int kind;
          const int c = neighbour_cell(G, w.kind, ix, iy, k / 3 - 1, k % 3 - 1, kind);
          hit |= c == cr || c == cg;
        }
        if (hit) seen |= 1u << z;
      }
    }
    cur.count[m] = carry_over(w, old, cur, m, nold, seen, nlist, st);
  }
  write_pairs(w, m, nlist, list_mj, list_code);
  raise(w.status, st);
}

}  // namespace xdem
