// pairs.cuh — updateContacts in three phases (rows a3-a15).
//
//   k_candidates    one thread per owner: the reference's 3x3 candidate scan
//                   (PeriodicBoundaryWorld.cpp:47-84, LeesEdwardsBoundaryWorld.cpp:
//                   128-204) with its filters and 200-candidate cap, a cheap
//                   coarse test, and a compact list of the pairs that pass;
//                   it also carries over the history of old contacts whose
//                   pair was not a candidate this step, as the reference's map
//                   entries survive;
//   k_pair_forces   one thread per listed pair: image offset, contact geometry,
//                   history, contact force and torques (BaseParticle.cpp:27-98),
//                   written to the pair's record (its pair-list index);
// both register every contact they write with its partner (an atomic entry in
// the partner's incoming list) for the partner's force sum.
// Splitting the light scan from the heavy geometry keeps warps full on the
// FP64 ellipse solvers.  A candidate rejected by the coarse test is still a
// candidate: its history is dropped, as the reference erases it
// (BaseParticle.cpp:95).  A listed pair that turns out not to touch leaves an
// empty record (partner -1) that every reader skips.
#pragma once
#include "kernels.cuh"

namespace xdem {

// image offset of candidate j (PeriodicBoundaryWorld.cpp:97-101,
// LeesEdwardsBoundaryWorld.cpp:233-279)
__device__ __forceinline__ void image_offset(const WorldScalars& ws, int kind, double2 pi,
                                             double2 pj, vec2<double>& off, vec2<double>& ovel) {
  ovel = V(0.0, 0.0);
  if (kind == CAND_REGULAR) {
    double ox = 0.0, oy = 0.0;
    if (pj.x - pi.x > ws.xlen / 2.0) ox = -ws.xlen;
    else if (pj.x - pi.x < -ws.xlen / 2.0) ox = ws.xlen;
    if (pj.y - pi.y > ws.ylen / 2.0) oy = -ws.ylen;
    else if (pj.y - pi.y < -ws.ylen / 2.0) oy = ws.ylen;
    off = V(ox, oy);
    return;
  }
  off = (kind == CAND_TOP) ? V(ws.shift, ws.ylen) : V(-ws.shift, -ws.ylen);
  double t = off.x + pj.x;
  if (t < ws.xmin) {
    off.x += ws.xlen;
    t += ws.xlen;
  } else if (t > ws.xmax) {
    off.x += -ws.xlen;
    t -= ws.xlen;
  }
  if (t - pi.x > ws.xlen / 2.0) off.x += -ws.xlen;
  else if (t - pi.x < -ws.xlen / 2.0) off.x += ws.xlen;
  ovel = V((kind == CAND_TOP) ? ws.shift_vel : -ws.shift_vel, 0.0);
}

// Cheap test that every contact passes: the full overlap test for two circles
// (CircularParticle.cpp:73-77, same operations), the bounding-circle test for
// two ellipses (takeCoarseDetection, BaseParticle.h:131-132).  Other pairs
// (mixed shapes, clumps) go on to the dispatcher, which rejects or flags them.
template <int LAW>
__device__ __forceinline__ bool coarse_pass(int shape_i, int shape_j, double r_i, double r_j,
                                            double orad_i, double orad_j, double2 pi, double2 pj,
                                            vec2<double> off) {
  vec2<double> pa = V(pi.x, pi.y);
  vec2<double> pb = V(pj.x, pj.y) + off;
  // a world-wide law decides; only a mixed world looks at the two shapes
  const bool circles =
      LAW == LAW_CIRCLE || (LAW == LAW_ANY && shape_i == SHAPE_CIRCLE && shape_j == SHAPE_CIRCLE);
  const bool ellipses = LAW == LAW_CLOSEST || LAW == LAW_INTERSECTION ||
                        (LAW == LAW_ANY && shape_i == SHAPE_ELLIPSE && shape_j == SHAPE_ELLIPSE);
  // the squared distance decides unless it lies within 1e-14 (relative) of
  // the squared radius sum, where the reference's expression (with its
  // correctly rounded sqrt) is evaluated as written
  if (circles) {
    const vec2<double> dv = pb - pa;
    const double R = r_i + r_j, d2 = len2(dv), R2 = R * R;
    if (d2 < R2 * (1.0 - 1e-14)) return true;
    if (d2 > R2 * (1.0 + 1e-14)) return false;
    double distance = len(dv);
    return !(R - distance < 0.0);
  }
  if (ellipses) {
    const double R = orad_i + orad_j, d2 = len2(pa - pb), R2 = R * R;
    if (d2 < R2 * (1.0 - 1e-14)) return true;
    if (d2 > R2 * (1.0 + 1e-14)) return false;
    return R > sqrt(len2(pa - pb));
  }
  return true;
}

// Shape of a body for the centre-line screen of two ellipses: (cos, sin) of
// its major axis and its semi-axes, FP32.
struct AxisShape {
  float c, s, a, b;
};

// the screen's record of the ellipse at m (k_scatter wrote it this step)
__device__ __forceinline__ AxisShape axis_shape(const DevWorld& w, int m) {
  const float4 r = w.axis[m];
  return AxisShape{r.x, r.y, r.z, r.w};
}

// Class of a pair of ellipses on the line of their centres, from the centre
// distance |d| and the sum S of their half-widths along d̂:
//   CL_SEPARATED  |d| > 1.001 S: the projections on that line are disjoint.
//                 The exact distance of closest approach along d̂ is at most
//                 S, and two disjoint ellipses do not intersect, so neither
//                 law has a contact there and the pair's history is erased
//                 (BaseParticle.cpp:95), as it is for a candidate that is not
//                 listed: the pair is dropped.
//   CL_DEEP       |d| < 0.7 S: a deep overlap.  The closest-approach Newton
//                 iterations that run to their cap come from such pairs; they
//                 are listed apart and evaluated beside the other pairs, so
//                 that their long serial solve starts first.
//   CL_REGULAR    otherwise.
// The screen serves the mixed-precision path only: the reference's own
// construction can report a contact for a separated pair when its Newton
// result is not finite (it then takes d' = 1 + a2', EllipticParticle.cpp:
// 168-170), and the FP64 path reproduces the reference pair for pair.  With
// H = half-width * |d| = sqrt(a²(d·k)² + b²(d×k)²) the tests compare |d|²
// with (H_i + H_j); the 1e-3 relative margin is far above the FP32 rounding
// of d, the angles and the axes (below 1e-5 relative).
enum { CL_SEPARATED = 0, CL_REGULAR = 1, CL_DEEP = 2 };

__device__ __forceinline__ int centre_line_class(float dx, float dy, const AxisShape& i,
                                                 const AxisShape& j) {
  const float pi = dx * i.c + dy * i.s, qi = dx * i.s - dy * i.c;
  const float pj = dx * j.c + dy * j.s, qj = dx * j.s - dy * j.c;
  const float hi = sqrtf(i.a * i.a * pi * pi + i.b * i.b * qi * qi);
  const float hj = sqrtf(j.a * j.a * pj * pj + j.b * j.b * qj * qj);
  const float d2 = dx * dx + dy * dy, S = hi + hj;
  return d2 > S * 1.001f ? CL_SEPARATED : (d2 < S * 0.7f ? CL_DEEP : CL_REGULAR);
}


// the centre-line screen applies to pairs of ellipses in mixed-precision
// worlds: under one law every pair, in a world of several shapes (LAW_ANY)
// the pairs of two ellipses
template <int LAW>
__device__ __forceinline__ bool centre_line_screen(const DevWorld& w) {
  return (LAW == LAW_CLOSEST || LAW == LAW_INTERSECTION || LAW == LAW_ANY) &&
         w.precision == XDEM_PRECISION_MIXED;
}
template <int LAW>
__device__ __forceinline__ bool screens_pair(const DevWorld& w, int shape_i, int shape_j) {
  return centre_line_screen<LAW>(w) &&
         (LAW != LAW_ANY || (shape_i == SHAPE_ELLIPSE && shape_j == SHAPE_ELLIPSE));
}

// the deep pairs of the screen are listed apart where the closest-approach
// law applies
template <int LAW>
__device__ __forceinline__ bool lists_deep(const DevWorld& w) {
  return LAW == LAW_CLOSEST || (LAW == LAW_ANY && w.method == ELLIPSE_CLOSEST);
}

// the owner's record for the screen (an ellipse's; zeros for other shapes)
template <int LAW>
__device__ __forceinline__ AxisShape owner_axis_shape(const DevWorld& w, int m) {
  AxisShape e{0.0f, 0.0f, 0.0f, 0.0f};
  if (centre_line_screen<LAW>(w) && (LAW != LAW_ANY || w.shape[m] == SHAPE_ELLIPSE))
    e = axis_shape(w, m);
  return e;
}

// this step's record of the owner's body for the pair kernels; an ellipse's
// (cos, sin) is computed once per body instead of once per pair
template <int LAW>
__device__ __forceinline__ void write_owner_body(const DevWorld& w, int m) {
  double2 cs = make_double2(0.0, 0.0);
  if (LAW == LAW_CLOSEST || LAW == LAW_INTERSECTION ||
      (LAW == LAW_ANY && w.shape[m] == SHAPE_ELLIPSE)) {
    const double r = w.rot[m];
    cs = make_double2(cos(r), sin(r));
  }
  write_body(w, m, cs);
}

// ---- phase A --------------------------------------------------------------------
// Cell (ix+dx, iy+dy) of the reference's 3x3 scan with its image kind
// (PeriodicBoundaryWorld.cpp:47-84; LeesEdwardsBoundaryWorld.cpp:128-204 for
// the ghost rows beyond the top and bottom edges).  The scan order does not
// matter: the pair list, slots and force sums are order independent.
__device__ __forceinline__ int neighbour_cell(const Grid& G, int world_kind, int ix, int iy, int dx,
                                              int dy, int& kind) {
  int jx = ix + dx;
  if (jx == -1) jx = G.nx - 1;
  else if (jx == G.nx) jx = 0;
  int jy = iy + dy;
  if (world_kind == WORLD_LE && (jy == -1 || jy == G.ny)) {
    kind = jy == -1 ? CAND_BOTTOM : CAND_TOP;
    return jy == -1 ? G.base + G.ncell + G.nx + jx : G.base + G.ncell + jx;
  }
  if (jy == -1) jy = G.ny - 1;
  else if (jy == G.ny) jy = 0;
  kind = CAND_REGULAR;
  return G.base + jy * G.nx + jx;
}

// The reference's 3x3 scan for the owner at m (cell ix, iy): every candidate
// j with a larger id and another upLevel, counted per image kind against the
// 200-candidate cap, and the ones passing the coarse test appended to
// (list_mj, list_code), entry s at index s * stride; `matched` receives the
// old slots of the listed pairs (all of them candidates, so their old slots
// count as seen).  The distance
// screen runs in FP32 on positions relative to the cell corners; only
// candidates within its rounding margin of the threshold take the
// reference's FP64 test.
template <int LAW>
__device__ __forceinline__ void scan_cells(const DevWorld& w, const WorldScalars& ws, const Grid& G,
                                           int m, int ix, int iy, double2 pi, int id_i, int up_i,
                                           int shape_i, double r_i, double orad_i,
                                           const Slots& old, int nold, int& nlist,
                                           int32_t* list_mj, int32_t* list_code, int stride,
                                           uint32_t& st, uint32_t& matched,
                                           const AxisShape& shape_ax) {
  const int K = w.K;
  const int ob = nold > 0 ? old.base[m] : 0;  // the owner's first old record
  // the owner relative to its cell's corner, in FP32 (see k_scatter)
  const float rxi = (float)(pi.x - (ws.xmin + ix * G.lx));
  const float ryi = (float)(pi.y - (ws.ymin + iy * G.ly));
  const float flx = (float)G.lx, fly = (float)G.ly;
  const float sr_i = screen_radius(w, m);
  int ncand0 = 0, ncand1 = 0, ncand2 = 0;
#pragma unroll 1
  for (int k = 0; k < 9; ++k) {
    const int dx = k / 3 - 1, dy = k % 3 - 1;
    int kind;
    const int c = neighbour_cell(G, w.kind, ix, iy, dx, dy, kind);
    const int q0 = w.cell_start[c], q1 = w.cell_start[c + 1];
    // the neighbour cell's corner relative to the owner's
    const float ox = dx * flx - rxi, oy = dy * fly - ryi;
    for (int q = q0; q < q1; ++q) {
      const float4 rj = w.cell_scr[q];
      const int id_j = __float_as_int(rj.w);
      if (id_j <= id_i) continue;  // also drops SKIP_CONTACT_DETECTION
      if (w.cell_up[q] == up_i) continue;
      int& nc = kind == CAND_REGULAR ? ncand0 : (kind == CAND_TOP ? ncand1 : ncand2);
      if (nc + 1 >= kCandidateCap) {
        st |= ST_CAPACITY;
        continue;
      }
      nc++;
      // FP32 screen with a margin well above its rounding error; the band
      // around the threshold takes the reference's FP64 test
      const float ddx = ox + rj.x, ddy = oy + rj.y;
      const float d2 = ddx * ddx + ddy * ddy;
      const float R = sr_i + rj.z, R2 = R * R;
      if (d2 > R2 * (1.0f + 1e-4f) + 1e-4f) continue;
      if (LAW == LAW_ANY || !(d2 < R2 * (1.0f - 1e-4f) - 1e-4f)) {
        const double2 pj = w.cell_pos[q];
        vec2<double> off, ovel;
        image_offset(ws, kind, pi, pj, off, ovel);
        const int mj = w.cell_mem[q];
        bool pass;
        if (LAW == LAW_ANY)
          pass = coarse_pass<LAW>(shape_i, w.shape[mj], r_i, w.rad[mj], orad_i, w.orad[mj], pi,
                                  pj, off);
        else
          pass = coarse_pass<LAW>(0, 0, r_i, w.screen_r[mj], orad_i, w.screen_r[mj], pi, pj, off);
        if (!pass) continue;
      }
      int cls = CL_REGULAR;
      if (screens_pair<LAW>(w, shape_i, LAW == LAW_ANY ? w.shape[w.cell_mem[q]] : 0)) {
        // the same FP64 image offset as the candidate lists' test (verlet.cuh)
        const double2 pj = w.cell_pos[q];
        vec2<double> off, ovel;
        image_offset(ws, kind, pi, pj, off, ovel);
        cls = centre_line_class((float)((pj.x + off.x) - pi.x), (float)((pj.y + off.y) - pi.y),
                                shape_ax, axis_shape(w, w.cell_mem[q]));
        if (cls == CL_SEPARATED) continue;
      }
      if (nlist >= K) {
        st |= ST_CAPACITY;
        continue;
      }
      int oslot = kNoOldSlot;
      for (int z = 0; z < nold; ++z)
        if (old.partner[ob + z] == id_j) oslot = z;
      if (oslot != kNoOldSlot) matched |= 1u << oslot;
      list_mj[nlist * stride] = w.cell_mem[q];
      list_code[nlist * stride] =
          kind | (nlist << 8) | (oslot << 16) | (lists_deep<LAW>(w) && cls == CL_DEEP ? kDeepFlag : 0);
      ++nlist;
    }
  }
}

// Old slots of the owner at m (cell ix, iy) to carry over: a valid old
// contact whose partner is not a candidate of the 3x3 scan this step.  A
// candidate's history is replaced by the pair kernel or dropped: the listed
// pairs (`matched`) are candidates, and so is a partner that sits in one of
// the nine cells and passes the candidate filters.  The history of the other
// old contacts survives unchanged, as the reference's map entries do.  At
// most `room` slots are kept (the first ones); more raise ST_CAPACITY.
__device__ __forceinline__ uint32_t carry_mask(const DevWorld& w, const Slots& old, const Grid& G,
                                               int m, int ix, int iy, int up_i, int nold,
                                               uint32_t matched, int room, uint32_t& st) {
  uint32_t carry = 0;
  if (nold <= 0) return 0;
  const int ob = old.base[m];
  int kept = 0;
  for (int z = 0; z < nold; ++z) {
    if (matched & (1u << z)) continue;
    const int p = old.partner[ob + z];
    if (p < 0) continue;
    const int mj = w.mpos[p];
    if (!(w.setting[mj] & SKIP_CONTACT_DETECTION) && w.up[mj] != up_i) {
      const int cr = w.pcell[mj], cg = w.gcell[mj];
      bool hit = false;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        int kind;
        const int c = neighbour_cell(G, w.kind, ix, iy, k / 3 - 1, k % 3 - 1, kind);
        hit |= c == cr || c == cg;
      }
      if (hit) continue;
    }
    if (kept >= room) {
      st |= ST_CAPACITY;
      break;
    }
    carry |= 1u << z;
    ++kept;
  }
  return carry;
}

// Old slots to carry over of an owner that takes no part in this step's
// contact detection (an invalid grid, SKIP_CONTACT_DETECTION): all valid
// ones, up to K.
__device__ __forceinline__ uint32_t carry_all(const DevWorld& w, const Slots& old, int m, int nold,
                                              uint32_t& st) {
  uint32_t carry = 0;
  if (nold <= 0) return 0;
  const int ob = old.base[m];
  int kept = 0;
  for (int z = 0; z < nold; ++z) {
    if (old.partner[ob + z] < 0) continue;
    if (kept >= w.K) {
      st |= ST_CAPACITY;
      break;
    }
    carry |= 1u << z;
    ++kept;
  }
  return carry;
}

// Registers the contact of record r (owner id owner_id) with its partner at
// memory position mj, for the partner's force sum.  The arrival order is
// free: k_collect orders the references by owner id.
__device__ __forceinline__ void register_contact(const DevWorld& w, int mj, int owner_id, int r,
                                                 uint32_t& st) {
  const int pos = atomicAdd(&w.incnt[mj], 1);
  if (pos < w.K)
    w.inref[(size_t)pos * w.n + mj] = ((uint64_t)(uint32_t)owner_id << 32) | (uint32_t)r;
  else st |= ST_CAPACITY;
}

// A carried-over contact: old record ro copied to record r of this step and
// registered with its partner.
__device__ __forceinline__ void carry_record(const DevWorld& w, const Slots& old, const Slots& cur,
                                             int owner_id, int ro, int r, uint32_t& st) {
  const int partner = old.partner[ro];
  cur.partner[r] = partner;
  cur.n[r] = old.n[ro];
  cur.s[r] = old.s[ro];
  cur.damp[r] = old.damp[ro];
  cur.f[r] = old.f[ro];
  cur.t1[r] = old.t1[ro];
  cur.t2[r] = old.t2[ro];
  cur.b[r] = old.b[ro];
  cur.cp[r] = old.cp[ro];
  cur.bv1[r] = old.bv1[ro];
  cur.bv2[r] = old.bv2[ro];
  cur.fn[r] = old.fn[ro];
  cur.ft[r] = old.ft[ro];
  register_contact(w, w.mpos[partner], owner_id, r, st);
}

// Reserves room for a block's listed pairs (nlist per thread) and deep-pair
// indices (ndeep per thread) with one atomic on the packed counter of the two
// lists (pairs in the low 32 bits, deep pairs in the high 32 bits); returns
// each thread's first index in both.  A block's pairs stay together in the
// list, in owner order, which keeps the pair kernel's gathers local.  Every
// thread of the block (of 128) calls.
__device__ __forceinline__ void reserve_pairs(const DevWorld& w, int nlist, int ndeep, int& at,
                                              int& deep_at) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int a = nlist, b = ndeep;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int va = __shfl_up_sync(full, a, o), vb = __shfl_up_sync(full, b, o);
    if (lane >= o) {
      a += va;
      b += vb;
    }
  }
  __shared__ int warp_a[4], warp_b[4];
  __shared__ unsigned long long block_base;
  if (lane == 31) {
    warp_a[warp] = a;
    warp_b[warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ta = warp_a[0] + warp_a[1] + warp_a[2] + warp_a[3];
    const unsigned tb = warp_b[0] + warp_b[1] + warp_b[2] + warp_b[3];
    block_base = (ta | tb) ? atomicAdd(w.pair_counts, ((unsigned long long)tb << 32) | ta) : 0ull;
  }
  __syncthreads();
  int ba = (int)(uint32_t)block_base, bb = (int)(uint32_t)(block_base >> 32);
  for (int k = 0; k < warp; ++k) {
    ba += warp_a[k];
    bb += warp_b[k];
  }
  at = ba + a - nlist;
  deep_at = bb + b - ndeep;
}

// Writes the owner's records to the pair list, after reserving their room
// (reserve_pairs): its listed pairs, with last step's record of each (old
// base + old slot, -1 for a new pair), then the old contacts it carries over
// (`carry`, a mask of old slots), whose records it copies here.  A pair
// classed deep (kDeepFlag) also goes to the deep-pair list.  Records the
// owner's first record and count.  Every thread of the block calls.
__device__ __forceinline__ void write_pairs(const DevWorld& w, const Slots& old, const Slots& cur,
                                            int m, bool valid, int nlist, const int32_t* list_mj,
                                            const int32_t* list_code, uint32_t carry,
                                            uint32_t& st) {
  int ndeep = 0;
  for (int s = 0; s < nlist; ++s) ndeep += (list_code[s] & kDeepFlag) ? 1 : 0;
  const int ncarry = __popc(carry);
  int at, k;
  reserve_pairs(w, nlist + ncarry, ndeep, at, k);
  if (!valid) return;
  cur.base[m] = at;
  cur.count[m] = nlist + ncarry;
  const int ob = old.base[m];  // used only where the owner has old records
  for (int s = 0; s < nlist; ++s) {
    const int c = list_code[s], oslot = (c >> 16) & 0xff;
    w.pairs[at + s] = PairEntry{m, list_mj[s], c, oslot != kNoOldSlot ? ob + oslot : -1};
    if (c & kDeepFlag) w.deep[k++] = at + s;
  }
  int s = nlist;
  for (uint32_t cm = carry; cm; cm &= cm - 1, ++s) {
    const int z = __ffs(cm) - 1, ro = ob + z;
    w.pairs[at + s] = PairEntry{m, w.mpos[old.partner[ro]], kCarryFlag | (s << 8) | (z << 16), ro};
    carry_record(w, old, cur, w.id_of[m], ro, at + s, st);
  }
}

// One thread per owner m.  Cell entries are read from the cell-ordered
// screening records (cell_scr, cell_up), so a neighbour cell is one
// contiguous run of 20-byte records; the distance screen runs in FP32 on
// positions relative to the cell corners, and only candidates within its
// rounding margin of the threshold take the reference's FP64 test.  Old
// slots whose partner sits in one of the nine cells (and passes the same
// filters) belong to candidates, so their history is replaced or dropped;
// the others are carried over (carry_mask).
template <int LAW>
__global__ void __launch_bounds__(128) k_candidates(DevWorld w, int par) {
  if (stopped(w)) return;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = m < w.n;
  const WorldScalars& ws = w.ws[valid ? sys_at(w, m) : 0];
  const int K = w.K;
  const Slots& old = w.slots[par];
  const Slots& cur = w.slots[par ^ 1];
  uint32_t st = 0;
  int nlist = 0;
  uint32_t carry = 0;
  int32_t list_mj[kMaxSlots];
  int32_t list_code[kMaxSlots];
  if (valid) {
    write_owner_body<LAW>(w, m);
    const AxisShape shape_ax = owner_axis_shape<LAW>(w, m);
    Grid G = grid_of(ws);
    const int id_i = w.id_of[m];
    const int nold = min(old.count[m], K);
    if (G.nx >= 3 && G.ny >= 3 && !(w.setting[m] & SKIP_CONTACT_DETECTION)) {
      const double2 pi = w.pos[m];
      const int up_i = w.up[m];
      const int shape_i = (LAW == LAW_ANY) ? w.shape[m] : 0;
      const double r_i = w.rad[m], orad_i = w.orad[m];
      // the owner's cell from this step's binning (k_bin, the same cell_of)
      const int cell_local = w.pcell[m] - G.base;
      const int ix = cell_local % G.nx, iy = cell_local / G.nx;
      uint32_t matched = 0;
      scan_cells<LAW>(w, ws, G, m, ix, iy, pi, id_i, up_i, shape_i, r_i, orad_i, old, nold, nlist,
                      list_mj, list_code, 1, st, matched, shape_ax);
      carry = carry_mask(w, old, G, m, ix, iy, up_i, nold, matched, K - nlist, st);
    } else {
      carry = carry_all(w, old, m, nold, st);
    }
  }
  write_pairs(w, old, cur, m, valid, nlist, list_mj, list_code, carry, st);
  raise(w.status, st);
}

// ---- phase B --------------------------------------------------------------------
// learned warm-start counters of a thread, combined over its warp (every lane
// must call)
__device__ __forceinline__ void flush_warm(const DevWorld& w, uint32_t offered, uint32_t used,
                                           uint32_t rejected, uint32_t restarted, uint32_t right) {
  const unsigned full = 0xffffffffu;
  offered = __reduce_add_sync(full, offered);
  used = __reduce_add_sync(full, used);
  rejected = __reduce_add_sync(full, rejected);
  restarted = __reduce_add_sync(full, restarted);
  right = __reduce_add_sync(full, right);
  if ((threadIdx.x & 31) == 0 && offered) {
    WorldScalars* wsm = w.ws;
    atomicAdd(&wsm->warm_offered, (unsigned long long)offered);
    atomicAdd(&wsm->warm_used, (unsigned long long)used);
    atomicAdd(&wsm->warm_rejected, (unsigned long long)rejected);
    atomicAdd(&wsm->warm_restarted, (unsigned long long)restarted);
    atomicAdd(&wsm->logit_right, (unsigned long long)right);
  }
}

// Counters of one thread of a pair kernel, flushed per warp at its end.
struct PairCounters {
  uint32_t st = 0;
  uint32_t n_solves = 0, n_iters = 0, n_capped = 0;
  uint32_t w_off = 0, w_used = 0, w_rej = 0, w_rest = 0, w_right = 0;
};

// One listed pair t: image offset, contact geometry, history and force,
// written to record t.  WARM: a closest-approach pair starts Newton from the
// learned warm start of its list entry (w.warm, k_mlp_warm).
template <bool FOLD_BG, int LAW, bool WARM>
__device__ __forceinline__ void pair_forces_fp64(const DevWorld& w, int par, int record, int t,
                                                 PairCounters& pc) {
  const Slots& old = w.slots[par];
  const Slots& cur = w.slots[par ^ 1];
  uint32_t& st = pc.st;
  {
    const PairEntry e = w.pairs[t];
    if (e.code & kCarryFlag) return;  // a carried-over record, copied by the candidate kernel
    const int m = e.m, mj = e.mj;
    const WorldScalars& ws = w.ws[sys_at(w, m)];
    const double dt = ws.dt, kn = ws.kn, kt = ws.kt, mu = ws.mu, factor = ws.factor;
    float2 wp = make_float2(0.0f, 0.0f);
    if (WARM && LAW == LAW_CLOSEST) wp = w.warm[t];
    const int kind = e.code & 0xff;
    const size_t ci = (size_t)t;
    const BodyRec ba = w.body[m], bb = w.body[mj];
    PState a = body_state<FOLD_BG>(ba, ws);
    PState b = body_state<FOLD_BG>(bb, ws);
    vec2<double> off, ovel;
    image_offset(ws, kind, make_double2(a.x, a.y), make_double2(b.x, b.y), off, ovel);
    Geom g;
    bool touching;
    if (LAW == LAW_ANY) {
      double2 csa = make_double2(0.0, 0.0), csb = make_double2(0.0, 0.0);
      if (a.shape == SHAPE_ELLIPSE && b.shape == SHAPE_ELLIPSE) {
        csa = ba.cs;
        csb = bb.cs;
      }
      touching = contact_geometry(w.method, a, b, w.orad[m], w.orad[mj], off, ovel, csa, csb, g, st,
                                  seg_of(w, ba), seg_of(w, bb));
    } else {
      // the scan has applied the coarse test of this pair
      double2 csa = make_double2(0.0, 0.0), csb = make_double2(0.0, 0.0);
      if (LAW != LAW_CIRCLE) {
        csa = ba.cs;
        csb = bb.cs;
      }
      touching = contact_geometry_law<LAW, true, WARM && LAW == LAW_CLOSEST>(
          a, b, 0.0, 0.0, off, ovel, csa, csb, g, st, wp.x);
    }
    if (WARM && LAW == LAW_CLOSEST && g.warm) {
      pc.w_off++;
      pc.w_used += g.warm == 1 || g.warm == 3;
      pc.w_rej += g.warm == 2;
      pc.w_rest += g.warm == 3;
      pc.w_right += (wp.y > 0.0f) == touching;
    }
    if (LAW != LAW_CIRCLE && g.iters > 0) {
      pc.n_solves++;
      pc.n_iters += g.iters;
      pc.n_capped += g.stuck ? 1u : 0u;
    }
    if (!touching) {
      cur.partner[ci] = -1;
      return;
    }
    const int id_j = bb.id;
    // BaseParticle::calculateContactForceAndTorque (BaseParticle.cpp:27-98)
    vec2<double> sh, nn = g.n;
    double damp;
    if (e.old < 0) {
      double rvn = dot(g.rv, g.n);
      if (!is_normal(rvn)) sh = g.srv * dt;
      else sh = g.srv * std_min(dt, g.overlap / rvn);
      damp = damping_of(w, factor, ba, bb, m, mj);
    } else {
      size_t oi = (size_t)e.old;
      double2 on = old.n[oi], os = old.s[oi];
      damp = old.damp[oi];
      vec2<double> no = V(on.x, on.y);
      double dd = dot(no, nn);
      double de = cross(no, nn);
      double angle = atan2(de, dd);
      double ca = cos(angle), sa = sin(angle);
      mat2<double> R = M(ca, -sa, sa, ca);
      sh = R * V(os.x, os.y);
      sh = sh + g.srv * dt;
    }
    vec2<double> br = V(a.x, a.y) - (V(b.x, b.y) + off);
    // ContactModel_LinearDissipativeFrictioanl (…Frictional.cpp:3-46)
    vec2<double> fn = ((-nn) * kn) * g.overlap + (-g.nrv) * damp;
    double maxFs = len(fn) * mu;
    vec2<double> el = (-sh) * kt;
    vec2<double> di = (-g.srv) * damp;
    vec2<double> fs = el + di;
    if (len(fs) > maxFs) {
      fs = unit(fs) * maxFs;
      if (len(el) > maxFs) sh = (-fs) / kt;
      else sh = (-el) / kt;
    }
    // ContactInformation::calculateTotalForceAndTorque (ContactInformation.h:62-68)
    vec2<double> F = fn + fs;
    cur.partner[ci] = id_j;
    cur.n[ci] = make_double2(nn.x, nn.y);
    cur.s[ci] = make_double2(sh.x, sh.y);
    cur.damp[ci] = damp;
    cur.f[ci] = make_double2(F.x, F.y);
    cur.t1[ci] = cross(g.bv1, F);
    cur.t2[ci] = cross(g.bv2, -F);
    cur.b[ci] = make_double2(br.x, br.y);
    if (record) {
      cur.cp[ci] = make_double2(g.cp.x, g.cp.y);
      cur.bv1[ci] = make_double2(g.bv1.x, g.bv1.y);
      cur.bv2[ci] = make_double2(g.bv2.x, g.bv2.y);
      cur.fn[ci] = make_double2(fn.x, fn.y);
      cur.ft[ci] = make_double2(fs.x, fs.y);
    }
    register_contact(w, mj, ba.id, t, st);
  }
}

// ---- end of the update ----------------------------------------------------------
// The pair kernels have consumed this step's lists: the counters start again
// from zero for the next update, and the count of listed pairs is kept for
// the host.  Done by the last block to finish the launch that ends the pair
// phase (`finish`): a fence before the count of finished blocks orders every
// block's reads of the counters before the reset; nothing waits.  Every
// thread of the block calls.
__device__ __forceinline__ void finish_pairs(const DevWorld& w) {
  __shared__ bool last;
  if (last_block(&w.done[2], last) && threadIdx.x == 0) {
    w.ws->last_pairs = *w.npairs;
    *w.npairs = 0;
    *w.nfallback = 0;
    *w.ndeep = 0;
    w.done[2] = 0;
  }
}

// one thread per listed pair (grid-stride loop)
template <bool FOLD_BG, int LAW, bool WARM = false>
__global__ void __launch_bounds__(128, 4) k_pair_forces(DevWorld w, int par, int record,
                                                        int finish) {
  if (stopped(w)) return;
  const int npairs = *w.npairs;
  PairCounters pc;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += gridDim.x * blockDim.x)
    pair_forces_fp64<FOLD_BG, LAW, WARM>(w, par, record, t, pc);
  flush_warp(w, pc.st, pc.n_solves, pc.n_iters, pc.n_capped);
  if (WARM) flush_warm(w, pc.w_off, pc.w_used, pc.w_rej, pc.w_rest, pc.w_right);
  if (finish) finish_pairs(w);
}

}  // namespace xdem
