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
constexpr int kVlRounds = 1;  // rounds of 32 list entries whose loads k_candidates_vl issues together (two spill at 72 registers and measured slower)

// the step's list-rebuild decision from the block maxima of the path lengths
// (nblocks of them; written by other blocks of the launch, so read past the
// L1); every thread of the block calls
__device__ __forceinline__ void vl_decide(const DevWorld& w, int nblocks, double* sh) {
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmax(v, __ldcg(w.vl_part + b));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double mx = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mx = fmax(mx, sh[k]);
  list_rebuild_decision(w, mx);
}

// block maxima of the path lengths since the last build; the last block to
// finish takes the rebuild decision (a fence before the count of finished
// blocks makes every maximum visible to it; nothing waits)
__global__ void __launch_bounds__(kVlBlock) k_vl_maxdisp(DevWorld w) {
  pdl_begin();
  if (stopped(w)) return;
  __shared__ double sh[kVlBlock / 32];
  __shared__ bool last;
  double v = 0.0;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < w.n; m += gridDim.x * blockDim.x)
    v = fmax(v, w.vl_disp[m]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int k = 0; k < kVlBlock / 32; ++k) mx = fmax(mx, sh[k]);
    w.vl_part[blockIdx.x] = mx;
  }
  if (last_block(&w.done[0], last)) {
    vl_decide(w, gridDim.x, sh);
    if (threadIdx.x == 0) w.done[0] = 0;
  }
}

// One thread per owner: the full 3x3 scan with the reference's filters, the
// partners within R + skin (an FP32 test with a margin that only widens the
// list) kept as (memory position, image kind); the path lengths restart.  An
// owner with more partners than the list holds is marked (count -1) and
// scanned in full every step until the next build.
template <int LAW>
__global__ void __launch_bounds__(128) k_vl_build(DevWorld w) {
  pdl_begin();
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
      // two cell entries at a time, their loads issued together
      for (int q = q0; q < q1; q += 2) {
        const bool two = q + 1 < q1;
        const float4 ra = w.cell_scr[q];
        const float4 rb = two ? w.cell_scr[q + 1] : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        const int ua = w.cell_up[q], ub = two ? w.cell_up[q + 1] : up_i;
        const int ma = w.cell_mem[q], mb = two ? w.cell_mem[q + 1] : 0;
        const bool ka = __float_as_int(ra.w) > id_i && ua != up_i &&
                        !((ox + ra.x) * (ox + ra.x) + (oy + ra.y) * (oy + ra.y) >
                          (sr_i + ra.z) * (sr_i + ra.z) * (1.0f + 1e-4f) + 1e-4f);
        const bool kb = __float_as_int(rb.w) > id_i && ub != up_i &&
                        !((ox + rb.x) * (ox + rb.x) + (oy + rb.y) * (oy + rb.y) >
                          (sr_i + rb.z) * (sr_i + rb.z) * (1.0f + 1e-4f) + 1e-4f);
        if (ka) {
          if (cnt >= w.V) {
            cnt = -1;
            break;
          }
          w.vl[(size_t)cnt * n + m] = (ma << 2) | kind;
          ++cnt;
        }
        if (kb) {
          if (cnt >= w.V) {
            cnt = -1;
            break;
          }
          w.vl[(size_t)cnt * n + m] = (mb << 2) | kind;
          ++cnt;
        }
      }
      if (cnt < 0) break;
    }
  }
  w.vl_cnt[m] = cnt;
  if (cnt < 0) w.ws->vl_overflow = 1;  // k_scatter then writes the cell records every step
}

// k_candidates with the lists: same outputs (body records, slot counts,
// carried-over history, the compact pair list), the same filters and tests,
// evaluated by the warp together.  One lane per owner loads the owner and its
// old partners; the warp's list entries are then taken 32 at a time across
// all lanes (entry e of the warp belongs to the owner lane whose prefix range
// of list lengths holds e), so that owners with long and short lists keep
// every lane busy, and each lane fetches what it needs of its entry's owner
// with warp shuffles.  The entries an owner keeps are ranked in list order
// (a ballot per round), so the owner's list and its slot numbering are the
// ones a thread walking its own list produces; they are staged in shared
// memory, slot-major (entry s of the thread at tid at s * 128 + tid), and the
// warp writes its pairs to the pair list together, coalesced, in owner order.
// Dynamic shared memory: 2 * K * 128 int32.
template <int LAW>
// body: write the owners' body records here (after a re-sort, or when the
// step runs as sub-steps; otherwise the binning kernel has written them)
__global__ void __launch_bounds__(128, 7) k_candidates_vl(DevWorld w, int par, int body) {
  pdl_begin();
  if (stopped(w)) return;
  extern __shared__ int32_t s_list[];
  __shared__ uint32_t s_matched[128];
  const unsigned full = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, wbase = tid & ~31;
  const int m = blockIdx.x * blockDim.x + tid;
  const bool valid = m < w.n;
  const int n = w.n, K = w.K;
  int32_t* s_mj = s_list;
  int32_t* s_code = s_list + K * 128;
  const Slots& old = w.slots[par];
  const Slots& cur = w.slots[par ^ 1];
  uint32_t st = 0;
  int nlist = 0, cnt = 0, nold = 0, ob = 0, up_i = 0, shape_i = 0, ix = 0, iy = 0;
  bool scan = false;
  double2 pi = make_double2(0.0, 0.0);
  double r_i = 0.0, orad_i = 0.0;
  AxisShape shape_ax{0.0f, 0.0f, 0.0f, 0.0f};
  Grid G{};
  // the memory positions of the first four old partners (the usual case);
  // the others are read where they are
  int op0 = -1, op1 = -1, op2 = -1, op3 = -1;
  s_matched[tid] = 0u;
  if (valid) {
    const WorldScalars& ws = w.ws[sys_at(w, m)];
    if (body) write_owner_body<LAW>(w, m);
    shape_ax = owner_axis_shape<LAW>(w, m);
    G = grid_of(ws);
    nold = min(old.count[m], K);
    ob = nold > 0 ? old.base[m] : 0;  // the owner's first old record
    scan = G.nx >= 3 && G.ny >= 3 && !(w.setting[m] & SKIP_CONTACT_DETECTION);
    if (scan) {
      pi = w.pos[m];
      up_i = w.up[m];
      shape_i = (LAW == LAW_ANY) ? w.shape[m] : 0;
      r_i = w.rad[m];
      orad_i = w.orad[m];
      // the owner's cell from this step's binning (k_bin, the same cell_of)
      const int cell_local = w.pcell[m] - G.base;
      ix = cell_local % G.nx;
      iy = cell_local / G.nx;
      cnt = w.vl_cnt[m];
      if (cnt < 0) {  // the list overflowed at its build: the full scan
        uint32_t matched = 0;
        scan_cells<LAW>(w, ws, G, m, ix, iy, pi, w.id_of[m], up_i, shape_i, r_i, orad_i, old,
                        nold, nlist, s_mj + tid, s_code + tid, 128, st, matched, shape_ax);
        s_matched[tid] = matched;
        cnt = 0;
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
          const int id_i = w.id_of[m];
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
        // the first four old partners' memory positions (list entries are
        // memory positions; ids and positions are one to one)
        const int p0 = nold > 0 ? old.partner[ob] : -1;
        const int p1 = nold > 1 ? old.partner[ob + 1] : -1;
        const int p2 = nold > 2 ? old.partner[ob + 2] : -1;
        const int p3 = nold > 3 ? old.partner[ob + 3] : -1;
        op0 = p0 >= 0 ? w.mpos[p0] : -1;
        op1 = p1 >= 0 ? w.mpos[p1] : -1;
        op2 = p2 >= 0 ? w.mpos[p2] : -1;
        op3 = p3 >= 0 ? w.mpos[p3] : -1;
      }
    }
  }
  __syncwarp();
  // the warp's list entries, flattened: lane o owns entries [excl, incl)
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += v;
  }
  const int excl = incl - cnt;
  const int total = __shfl_sync(full, incl, 31);
  // kVlRounds rounds of 32 entries at a time: the owners and list entries of
  // all of them are located and their loads issued before any is tested
  for (int r0 = 0; r0 < total; r0 += 32 * kVlRounds) {
    int oh[kVlRounds], oex[kVlRounds], moh[kVlRounds], ent[kVlRounds];
    double2 pjh[kVlRounds];
    double sjh[kVlRounds];
    AxisShape axh[kVlRounds];
#pragma unroll
    for (int h = 0; h < kVlRounds; ++h) {
      const int e = r0 + 32 * h + lane;
      // the owner lane: the number of lanes whose range ends at or before e
      int o = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1)
        if (__shfl_sync(full, incl, o + step - 1) <= e) o += step;
      oh[h] = o;
      oex[h] = __shfl_sync(full, excl, o);
      moh[h] = __shfl_sync(full, m, o);
      ent[h] = e < total ? w.vl[(size_t)(e - oex[h]) * n + moh[h]] : 0;
    }
#pragma unroll
    for (int h = 0; h < kVlRounds; ++h) {
      const bool act = r0 + 32 * h + lane < total;
      const int mj = ent[h] >> 2;
      pjh[h] = act ? w.pos[mj] : make_double2(0.0, 0.0);
      sjh[h] = act && LAW != LAW_ANY ? w.screen_r[mj] : 0.0;
      axh[h] = act && centre_line_screen<LAW>(w) && LAW != LAW_ANY ? axis_shape(w, mj)
                                                                 : AxisShape{0.0f, 0.0f, 0.0f, 0.0f};
    }
#pragma unroll
    for (int h = 0; h < kVlRounds; ++h) {
      const int rb = r0 + 32 * h;
      const int e = rb + lane;
      const bool act = e < total;
      const int o = oh[h], o_excl = oex[h], mo = moh[h];
      const double pix = __shfl_sync(full, pi.x, o), piy = __shfl_sync(full, pi.y, o);
      const double ro = __shfl_sync(full, r_i, o), orado = __shfl_sync(full, orad_i, o);
      const int shape_o = (LAW == LAW_ANY) ? __shfl_sync(full, shape_i, o) : 0;
      AxisShape ax_o{0.0f, 0.0f, 0.0f, 0.0f};
      if (centre_line_screen<LAW>(w)) {
        ax_o.c = __shfl_sync(full, shape_ax.c, o);
        ax_o.s = __shfl_sync(full, shape_ax.s, o);
        ax_o.a = __shfl_sync(full, shape_ax.a, o);
        ax_o.b = __shfl_sync(full, shape_ax.b, o);
      }
      const int q0 = __shfl_sync(full, op0, o), q1 = __shfl_sync(full, op1, o);
      const int q2 = __shfl_sync(full, op2, o), q3 = __shfl_sync(full, op3, o);
      const int nold_o = __shfl_sync(full, nold, o), ob_o = __shfl_sync(full, ob, o);
      const int nl = __shfl_sync(full, nlist, o);
      bool keep = false;
      int mj = 0, code = 0, oslot = kNoOldSlot;
      bool near = true;
      if (act) {
        const WorldScalars& wo = w.ws[sys_at(w, mo)];
        mj = ent[h] >> 2;
        const int kind = ent[h] & 3;
        const double2 pio = make_double2(pix, piy);
        const double2 pj = pjh[h];
        vec2<double> off, ovel;
        image_offset(wo, kind, pio, pj, off, ovel);
        bool pass;
        if (LAW == LAW_ANY)
          pass = coarse_pass<LAW>(shape_o, w.shape[mj], ro, w.rad[mj], orado, w.orad[mj], pio, pj, off);
        else
          pass = coarse_pass<LAW>(0, 0, ro, sjh[h], orado, sjh[h], pio, pj, off);
        int cls = CL_REGULAR;
        if (pass && screens_pair<LAW>(w, shape_o, LAW == LAW_ANY ? w.shape[mj] : 0)) {
          // (a world of several shapes reads the partner's axis record here,
          // for the pairs of two ellipses only)
          const AxisShape ax_j = LAW == LAW_ANY ? axis_shape(w, mj) : axh[h];
          cls = centre_line_class((float)((pj.x + off.x) - pio.x), (float)((pj.y + off.y) - pio.y),
                                  ax_o, ax_j);
          pass = cls != CL_SEPARATED;
        }
        if (pass) {
          keep = true;
          if (q0 == mj) oslot = 0;
          if (q1 == mj) oslot = 1;
          if (q2 == mj) oslot = 2;
          if (q3 == mj) oslot = 3;
          if (nold_o > 4) {
            const int id_j = w.id_of[mj];
            for (int z = 4; z < nold_o; ++z)
              if (old.partner[ob_o + z] == id_j) oslot = z;
          }
          // a pair that passed a distance test lies within one cell size, so
          // it is a candidate of the 3x3 scan (LAW_ANY's other pairs pass
          // without one and take the cell test of carry_mask)
          if (LAW == LAW_ANY) {
            const int shape_j = w.shape[mj];
            near = shape_o == shape_j && (shape_o == SHAPE_CIRCLE || shape_o == SHAPE_ELLIPSE);
          }
          code = kind | (oslot << 16) | (lists_deep<LAW>(w) && cls == CL_DEEP ? kDeepFlag : 0);
        }
      }
      // rank among the owner's kept entries of this round, in list order
      const unsigned kmask = __ballot_sync(full, keep);
      if (keep) {
        const int first = max(o_excl - rb, 0);
        const unsigned before = ((1u << lane) - 1u) & ~((1u << first) - 1u);
        const int idx = nl + __popc(kmask & before);
        if (idx < K) {
          s_mj[idx * 128 + wbase + o] = mj;
          s_code[idx * 128 + wbase + o] = code | (idx << 8);
          if (oslot != kNoOldSlot && near) atomicOr(&s_matched[wbase + o], 1u << oslot);
        } else {
          st |= ST_CAPACITY;
        }
      }
      // this lane as owner: its entries of this round are lanes [lo, hi)
      const int lo = max(excl - rb, 0), hi = min(incl - rb, 32);
      if (hi > lo) {
        const unsigned mine = (hi == 32 ? full : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
        nlist = min(nlist + __popc(kmask & mine), K);
      }
    }
  }
  __syncwarp();
  int ndeep = 0;
  uint32_t carry = 0;
  if (valid) {
    if (scan) {
      // the owner's grid, cell and up-level again (reloaded rather than kept
      // in registers through the entry loop)
      const Grid G2 = grid_of(w.ws[sys_at(w, m)]);
      const int cl = w.pcell[m] - G2.base;
      carry = carry_mask(w, old, G2, m, cl % G2.nx, cl / G2.nx, w.up[m], nold, s_matched[tid],
                         K - nlist, st);
    } else {
      carry = carry_all(w, old, m, nold, st);
    }
    for (int s = 0; s < nlist; ++s) ndeep += (s_code[s * 128 + tid] & kDeepFlag) ? 1 : 0;
  }
  const int nrec = nlist + __popc(carry);  // the owner's records: listed pairs, then carried
  int at, dk;
  reserve_pairs(w, nrec, ndeep, at, dk);
  if (valid) {
    cur.base[m] = at;
    cur.count[m] = nrec;
  }
  // the warp's records take consecutive entries of the pair list from its
  // lane 0's, in owner order, and its deep pairs consecutive deep-list
  // entries
  int pincl = nrec;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(full, pincl, o);
    if (lane >= o) pincl += v;
  }
  const int pexcl = pincl - nrec;
  const int ptotal = __shfl_sync(full, pincl, 31);
  const int wat = __shfl_sync(full, at, 0), wdk = __shfl_sync(full, dk, 0);
  int dcount = 0;
  for (int r0 = 0; r0 < ptotal; r0 += 32) {
    const int i = r0 + lane;
    const bool act = i < ptotal;
    int o = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
      if (__shfl_sync(full, pincl, o + step - 1) <= i) o += step;
    const int s = i - __shfl_sync(full, pexcl, o);
    const int mo = __shfl_sync(full, m, o);
    const int nl_o = __shfl_sync(full, nlist, o), ob_o = __shfl_sync(full, ob, o);
    const uint32_t carry_o = __shfl_sync(full, carry, o);
    int c = 0;
    if (act && s < nl_o) c = s_code[s * 128 + wbase + o];
    const bool deep = act && (c & kDeepFlag);
    const unsigned dmask = __ballot_sync(full, deep);
    if (act && s < nl_o) {
      const int oslot = (c >> 16) & 0xff;
      w.pairs[wat + i] = PairEntry{mo, s_mj[s * 128 + wbase + o], c,
                                   oslot != kNoOldSlot ? ob_o + oslot : -1};
      if (deep) w.deep[wdk + dcount + __popc(dmask & ((1u << lane) - 1u))] = wat + i;
    } else if (act) {
      // the (s - nl_o)-th carried old slot
      uint32_t cm = carry_o;
      for (int q = nl_o; q < s; ++q) cm &= cm - 1;
      const int z = __ffs(cm) - 1, ro = ob_o + z;
      w.pairs[wat + i] = PairEntry{mo, w.mpos[old.partner[ro]], kCarryFlag | (s << 8) | (z << 16), ro};
      carry_record(w, old, cur, w.id_of[mo], ro, wat + i, st);
    }
    dcount += __popc(dmask);
  }
  raise(w.status, st);
}

}  // namespace xdem
