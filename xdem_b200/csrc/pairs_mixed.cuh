// pairs_mixed.cuh — phase B of updateContacts for the mixed-precision path
// (XDEM_PRECISION_MIXED).  Same candidate list, records and history carry-over
// as the FP64 path (pairs.cuh); per listed pair:
//   geometry   geometry_mixed.cuh (FP32 with the FP64 overlap);
//   history    the tangential spring stays FP64: its rotation with the normal
//              (BaseParticle.cpp:67-82) takes cos/sin of the turn angle as
//              (n_old·n, n_old×n)/|…| instead of atan2 followed by cos and sin
//              (the same numbers, without the transcendental calls), and the
//              increment v_t dt is added in FP64;
//   force      ContactModel_LinearDissipativeFrictioanl (…Frictional.cpp:3-46)
//              in FP32, written to the FP64 history records.
// Closest-approach pairs that need the reference's FP64 construction (see
// geometry_mixed.cuh) are appended to a fallback list and evaluated by
// k_pair_fallback_m after the main pass, so that both passes run converged
// warps.
#pragma once
#include "geometry_mixed.cuh"
#include "pairs.cuh"

namespace xdem {

__device__ __forceinline__ bool is_normal_f(float x) {
  const float a = fabsf(x);
  return a >= 1.17549435e-38f && a <= 3.40282347e38f;
}

// history, force and torques of one touching pair, written to its record t
// (its pair-list index) and registered with the partner
__device__ __forceinline__ void write_contact_m(const DevWorld& w, const WorldScalars& ws,
                                                const PairEntry& e, int t, const BodyRec& ba,
                                                const BodyRec& bb, const PState& a,
                                                const PState& b, vec2<double> off,
                                                const GeomM& g, int par, int record,
                                                uint32_t& st) {
  const Slots& old = w.slots[par];
  const Slots& cur = w.slots[par ^ 1];
  const int m = e.m, mj = e.mj;
  const size_t ci = (size_t)t;
  const double dt = ws.dt;
  double sx, sy, damp;
  if (e.old < 0) {
    // new contact (BaseParticle.cpp:38-65)
    const float rvn = g.rv.x * g.n.x + g.rv.y * g.n.y;
    double tt = dt;
    if (is_normal_f(rvn)) tt = std_min(dt, g.overlap / (double)rvn);
    sx = (double)g.srv.x * tt;
    sy = (double)g.srv.y * tt;
    damp = damping_of(w, ws.factor, ba, bb, m, mj);
  } else {
    const size_t oi = (size_t)e.old;
    const double2 on = old.n[oi], os = old.s[oi];
    damp = old.damp[oi];
    const float nox = (float)on.x, noy = (float)on.y;
    const float dd = nox * g.n.x + noy * g.n.y;
    const float de = nox * g.n.y - noy * g.n.x;
    const float r2 = dd * dd + de * de;
    float ca = 1.0f, sa = 0.0f;
    if (r2 > 0.0f) {
      const float ir = rsqrtf(r2);
      ca = dd * ir;
      sa = de * ir;
    }
    sx = (double)ca * os.x - (double)sa * os.y + (double)g.srv.x * dt;
    sy = (double)sa * os.x + (double)ca * os.y + (double)g.srv.y * dt;
  }
  const float kt = (float)ws.kt, mu = (float)ws.mu, fd = (float)damp;
  const float kov = (float)(ws.kn * g.overlap);
  float fnx = -g.n.x * kov - g.nrv.x * fd;
  float fny = -g.n.y * kov - g.nrv.y * fd;
  const float maxFs = sqrtf(fnx * fnx + fny * fny) * mu;
  const float elx = (float)(-sx) * kt, ely = (float)(-sy) * kt;
  float fsx = elx - g.srv.x * fd, fsy = ely - g.srv.y * fd;
  const float fsl = sqrtf(fsx * fsx + fsy * fsy);
  if (fsl > maxFs) {
    const float sc = maxFs / fsl;
    fsx *= sc;
    fsy *= sc;
    if (sqrtf(elx * elx + ely * ely) > maxFs) {
      sx = (double)(-fsx) / ws.kt;
      sy = (double)(-fsy) / ws.kt;
    }
  }
  const float Fx = fnx + fsx, Fy = fny + fsy;
  const int id_j = bb.id;
  cur.partner[ci] = id_j;
  cur.n[ci] = make_double2((double)g.n.x, (double)g.n.y);
  cur.s[ci] = make_double2(sx, sy);
  cur.damp[ci] = damp;
  cur.f[ci] = make_double2((double)Fx, (double)Fy);
  cur.t1[ci] = (double)(g.bv1.x * Fy - g.bv1.y * Fx);
  cur.t2[ci] = (double)(-(g.bv2.x * Fy - g.bv2.y * Fx));
  cur.b[ci] = make_double2(a.x - (b.x + off.x), a.y - (b.y + off.y));
  if (record) {
    cur.cp[ci] = make_double2(a.x + (double)g.cpo.x, a.y + (double)g.cpo.y);
    cur.bv1[ci] = make_double2((double)g.bv1.x, (double)g.bv1.y);
    cur.bv2[ci] = make_double2((double)g.bv2.x, (double)g.bv2.y);
    cur.fn[ci] = make_double2((double)fnx, (double)fny);
    cur.ft[ci] = make_double2((double)fsx, (double)fsy);
  }
  register_contact(w, mj, ba.id, t, st);
}

__device__ __forceinline__ void count_solve(uint32_t it, uint32_t& n_solves, uint32_t& n_iters) {
  if (it > 0) {
    n_solves++;
    n_iters += it;
  }
}


// Which listed pairs a launch of k_pair_forces_m evaluates:
//   PASS_ALL      every listed pair; closest-approach pairs that need the FP64
//                 construction are deferred to k_pair_fallback_m;
//   PASS_REGULAR  every listed pair but the deep ones (PairEntry::pad), with
//                 the same deferral;
//   PASS_DEEP     the deep pairs (the deep-pair list), in k_pair_deep_m,
//                 which runs beside PASS_REGULAR; the FP64 construction runs
//                 in place, so
//                 that the closest-approach Newton iterations that run to their
//                 cap (deep overlaps) start with the step's other pairs
//                 instead of after them.
// Every pair is evaluated by the same operations whichever pass takes it.
enum { PASS_ALL = 0, PASS_REGULAR = 1, PASS_DEEP = 2 };

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Asks the L2 for what the pair at index t will read: its two body records
// (96 bytes each, two lines) and last step's history record.  Issued while
// the thread's current pair is computed, so that the next pair's gathers find
// their data on chip.
__device__ __forceinline__ void prefetch_pair(const DevWorld& w, int par, int t) {
  const PairEntry e = w.pairs[t];
  const char* ba = reinterpret_cast<const char*>(w.body + e.m);
  const char* bb = reinterpret_cast<const char*>(w.body + e.mj);
  prefetch_l2(ba);
  prefetch_l2(ba + sizeof(BodyRec) - 1);
  prefetch_l2(bb);
  prefetch_l2(bb + sizeof(BodyRec) - 1);
  if (e.old >= 0) {
    const Slots& old = w.slots[par];
    prefetch_l2(old.n + e.old);
    prefetch_l2(old.s + e.old);
    prefetch_l2(old.damp + e.old);
  }
}

// tn: the index of the thread's next pair (prefetched), or -1
template <bool FOLD_BG, int LAW, int PASS>
__device__ __forceinline__ void pair_forces_m(const DevWorld& w, int par, int record, int t,
                                              uint32_t& st, uint32_t& n_solves, uint32_t& n_iters,
                                              uint32_t& n_capped, int tn = -1) {
  const Slots& cur = w.slots[par ^ 1];
  const PairEntry e = w.pairs[t];
  // carried-over records are copied by the candidate kernel; the regular
  // pass leaves the deep pairs to k_pair_deep_m
  if (e.code & kCarryFlag) return;
  if (PASS == PASS_REGULAR && (e.code & kDeepFlag)) return;
  const int m = e.m, mj = e.mj;
  const WorldScalars& ws = w.ws[sys_at(w, m)];
  const int kind = e.code & 0xff;
  const size_t ci = (size_t)t;
  const BodyRec ba = w.body[m], bb = w.body[mj];
  if (tn >= 0) prefetch_pair(w, par, tn);
  const PState a = body_state<FOLD_BG>(ba, ws);
  const PState b = body_state<FOLD_BG>(bb, ws);
  vec2<double> off, ovel;
  image_offset(ws, kind, make_double2(a.x, a.y), make_double2(b.x, b.y), off, ovel);
  GeomM g;
  int res = PW_NONE;
  const bool circles = LAW == LAW_CIRCLE ||
                       (LAW == LAW_ANY && a.shape == SHAPE_CIRCLE && b.shape == SHAPE_CIRCLE);
  const bool closest = LAW == LAW_CLOSEST ||
                       (LAW == LAW_ANY && w.method == ELLIPSE_CLOSEST &&
                        a.shape == SHAPE_ELLIPSE && b.shape == SHAPE_ELLIPSE);
  if (circles) {
    res = circle_circle_m(a, b, off, ovel, g) ? PW_CONTACT : PW_NONE;
  } else if (closest) {
    res = ellipse_closest_m(a, b, off, ovel, ba.cs, bb.cs, g);
    if (PASS == PASS_DEEP) {
      if (res == PW_FALLBACK) {
        // the reference's FP64 construction in place (as k_pair_fallback_m)
        Geom gd = Geom{};
        const bool touching =
            ellipse_closest<false>(a, b, off, ovel, ba.cs.x, ba.cs.y, bb.cs.x, bb.cs.y, gd, st, 0.0f);
        if (gd.iters > 0) {
          n_solves++;
          n_iters += gd.iters;
          n_capped += gd.stuck ? 1u : 0u;
        }
        res = PW_NONE;
        if (touching) {
          geom_to_m(gd, a, g);
          res = PW_CONTACT;
        }
      } else {
        count_solve(g.iters, n_solves, n_iters);
      }
    } else {
      // deferred pairs take consecutive list entries, one atomic per warp
      const unsigned act = __activemask();
      const unsigned defer = __ballot_sync(act, res == PW_FALLBACK);
      if (res == PW_FALLBACK) {
        const int lane = threadIdx.x & 31, leader = __ffs(defer) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(w.nfallback, __popc(defer));
        base = __shfl_sync(defer, base, leader);
        w.fallback[base + __popc(defer & ((1u << lane) - 1u))] = t;
        return;
      }
      count_solve(g.iters, n_solves, n_iters);
    }
  } else {
    // intersection law (kept FP64: near tangency its quartic has a near
    // double root), clumps and unsupported pairs: the FP64 dispatcher
    double2 csa = make_double2(0.0, 0.0), csb = make_double2(0.0, 0.0);
    if (LAW == LAW_INTERSECTION || (a.shape == SHAPE_ELLIPSE && b.shape == SHAPE_ELLIPSE)) {
      csa = ba.cs;
      csb = bb.cs;
    }
    Geom gd;
    bool touching;
    if (LAW == LAW_INTERSECTION)
      touching = contact_geometry_law<LAW_INTERSECTION, true>(a, b, 0.0, 0.0, off, ovel, csa, csb, gd, st);
    else
      touching = contact_geometry(w.method, a, b, w.orad[m], w.orad[mj], off, ovel, csa, csb, gd, st,
                                  seg_of(w, ba), seg_of(w, bb));
    if (touching) geom_to_m(gd, a, g);
    res = touching ? PW_CONTACT : PW_NONE;
  }
  if (res != PW_CONTACT) {
    cur.partner[ci] = -1;
    return;
  }
  write_contact_m(w, ws, e, t, ba, bb, a, b, off, g, par, record, st);
}

template <bool FOLD_BG, int LAW, int PASS = PASS_ALL>
__global__ void __launch_bounds__(128, 4) k_pair_forces_m(DevWorld w, int par, int record,
                                                          int finish) {
  if (stopped(w)) return;
  uint32_t st = 0, n_solves = 0, n_iters = 0, n_capped = 0;
  const int npairs = *w.npairs;
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += stride)
    pair_forces_m<FOLD_BG, LAW, PASS>(w, par, record, t, st, n_solves, n_iters, n_capped,
                                      t + stride < npairs ? t + stride : -1);
  flush_warp(w, st, n_solves, n_iters, n_capped);
  if (finish) finish_pairs(w);
}

// PASS_DEEP: a few blocks, registers as the FP64 construction needs them;
// launched ahead of the regular pass, which it lets start at once
template <bool FOLD_BG, int LAW>
__global__ void __launch_bounds__(128) k_pair_deep_m(DevWorld w, int par, int record) {
  // the candidate kernel before it has completed; the regular pair pass,
  // launched after this kernel as a programmatic dependent launch, may start
  // now (it reads nothing this kernel writes)
  pdl_begin();
  if (stopped(w)) return;
  uint32_t st = 0, n_solves = 0, n_iters = 0, n_capped = 0;
  const int ndeep = *w.ndeep;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ndeep; t += gridDim.x * blockDim.x)
    pair_forces_m<FOLD_BG, LAW, PASS_DEEP>(w, par, record, w.deep[t], st, n_solves, n_iters,
                                           n_capped);
  flush_warp(w, st, n_solves, n_iters, n_capped);
}

// the closest-approach pairs deferred by k_pair_forces_m: the reference's FP64
// construction (EllipticParticle.cpp:34-285), then the mixed force
template <bool FOLD_BG, int LAW, bool WARM = false>
__global__ void __launch_bounds__(128) k_pair_fallback_m(DevWorld w, int par, int record,
                                                         int finish) {
  if (stopped(w)) return;
  const Slots& cur = w.slots[par ^ 1];
  const int nfb = *w.nfallback;
  uint32_t st = 0, n_solves = 0, n_iters = 0, n_capped = 0;
  uint32_t w_off = 0, w_used = 0, w_rej = 0, w_rest = 0, w_right = 0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nfb; f += gridDim.x * blockDim.x) {
    const int t = w.fallback[f];
    const PairEntry e = w.pairs[t];
    const int m = e.m, mj = e.mj;
    const WorldScalars& ws = w.ws[sys_at(w, m)];
    const int kind = e.code & 0xff;
    const size_t ci = (size_t)t;
    const BodyRec ba = w.body[m], bb = w.body[mj];
    const PState a = body_state<FOLD_BG>(ba, ws);
    const PState b = body_state<FOLD_BG>(bb, ws);
    vec2<double> off, ovel;
    image_offset(ws, kind, make_double2(a.x, a.y), make_double2(b.x, b.y), off, ovel);
    const double2 csa = ba.cs, csb = bb.cs;
    Geom gd = Geom{};
    const float2 wp = WARM ? w.warm[f] : make_float2(0.0f, 0.0f);
    const bool touching =
        ellipse_closest<WARM>(a, b, off, ovel, csa.x, csa.y, csb.x, csb.y, gd, st, wp.x);
    if (WARM && gd.warm) {
      w_off++;
      w_used += gd.warm == 1 || gd.warm == 3;
      w_rej += gd.warm == 2;
      w_rest += gd.warm == 3;
      w_right += (wp.y > 0.0f) == touching;
    }
    if (gd.iters > 0) {
      n_solves++;
      n_iters += gd.iters;
      n_capped += gd.stuck ? 1u : 0u;
    }
    if (!touching) {
      cur.partner[ci] = -1;
      continue;
    }
    GeomM g;
    geom_to_m(gd, a, g);
    write_contact_m(w, ws, e, t, ba, bb, a, b, off, g, par, record, st);
  }
  flush_warp(w, st, n_solves, n_iters, n_capped);
  if (WARM) flush_warm(w, w_off, w_used, w_rej, w_rest, w_right);
  if (finish) finish_pairs(w);
}

// single pairs through the mixed geometry (xdem_pair_geometry with
// XDEM_PRECISION_MIXED); same output layout as k_pair_geometry
__global__ void k_pair_geometry_m(int npairs, int method, const double* pi, const double* pj,
                                  const double* off, double* out, uint32_t* status) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const double* a = pi + 9 * k;
  const double* b = pj + 9 * k;
  PState A{(int)a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]};
  PState B{(int)b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8]};
  const double2 csa = make_double2(cos(A.rot), sin(A.rot));
  const double2 csb = make_double2(cos(B.rot), sin(B.rot));
  const vec2<double> of = V(off[4 * k], off[4 * k + 1]), ov = V(off[4 * k + 2], off[4 * k + 3]);
  uint32_t st = 0;
  GeomM g{};
  int res = PW_NONE;
  if (A.shape == SHAPE_CIRCLE && B.shape == SHAPE_CIRCLE) {
    res = circle_circle_m(A, B, of, ov, g) ? PW_CONTACT : PW_NONE;
  } else if (method == ELLIPSE_CLOSEST && A.shape == SHAPE_ELLIPSE && B.shape == SHAPE_ELLIPSE) {
    vec2<double> dd = V(A.x, A.y) - (V(B.x, B.y) + of);
    if ((a[1] + b[1]) > sqrt(len2(dd))) {
      res = ellipse_closest_m(A, B, of, ov, csa, csb, g);
      if (res == PW_FALLBACK) {
        Geom gd = Geom{};
        res = ellipse_closest(A, B, of, ov, csa.x, csa.y, csb.x, csb.y, gd, st) ? PW_CONTACT : PW_NONE;
        if (res == PW_CONTACT) geom_to_m(gd, A, g);
      }
    }
  } else {
    Geom gd = Geom{};
    res = contact_geometry(method, A, B, a[1], b[1], of, ov, csa, csb, gd, st) ? PW_CONTACT : PW_NONE;
    if (res == PW_CONTACT) geom_to_m(gd, A, g);
  }
  double* o = out + 17 * k;
  for (int z = 0; z < 17; ++z) o[z] = 0.0;
  o[0] = res == PW_CONTACT ? 1.0 : 0.0;
  if (res == PW_CONTACT) {
    o[1] = g.n.x;
    o[2] = g.n.y;
    o[3] = A.x + (double)g.cpo.x;
    o[4] = A.y + (double)g.cpo.y;
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
  }
  if (st) atomicOr(status, st);
}

}  // namespace xdem
