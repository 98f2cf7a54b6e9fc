// geometry.cuh — pairwise contact geometry on the device, FP64.
//
// Each routine restates one reference routine and keeps its operation order,
// so that, built with -fmad=false, its results differ from the reference only
// where CUDA's cos/sin/atan2/pow round differently from glibc's.
#pragma once
#include "dem_math.cuh"

namespace xdem {

// The reference loop (EllipticParticle.cpp:621) has no cap and never ends on
// some deeply overlapping pairs (δ < 0, the iterate wanders among negative
// values where the quartic has no root); some converging pairs of dense
// packings need several hundred iterations from the analytic start.  The
// iteration here stops when it repeats an earlier iterate exactly (it would
// then cycle forever) or at this cap.
constexpr int kNewtonCap = 1000;

enum : uint32_t {
  ST_CAPACITY = 1u << 0,
  ST_NEWTON = 1u << 1,
  ST_NONFINITE = 1u << 2,
  ST_UNSUPPORTED = 1u << 3,
  ST_ZERO_VECTOR = 1u << 4,
  ST_CUDA = 1u << 5,
  ST_ARGUMENT = 1u << 6,
  ST_GRID = 1u << 7,
  ST_TIMEOUT = 1u << 8
};

enum : int { SHAPE_CIRCLE = 0, SHAPE_ELLIPSE = 1, SHAPE_CLUMP = 2, SHAPE_SEGMENT = 3 };
enum : int { ELLIPSE_CLOSEST = 0, ELLIPSE_INTERSECTION = 1 };

struct PState {
  int shape;
  double r, asp, x, y, vx, vy, rot, w;
};

struct Geom {
  int contacted;
  int iters;
  int warm;  // learned warm start: 0 not offered, 1 used, 2 rejected by the residual test,
             // 3 used but the root left its interval (the plain start decided)
  int stuck;  // closest approach: Newton did not terminate (repeat or cap); the root
              // was then found by bisection (newton_quartic, bisect_quartic)
  vec2<double> cp, n, bv1, bv2;
  double overlap;
  vec2<double> rv, nrv, srv;
  double q, q_start;  // closest approach: the quartic's root and Newton's analytic start
};

// BaseParticle::calculateRelativeVelocityAtContactPoint (BaseParticle.cpp:11-25)
__device__ __forceinline__ void relative_velocity(const PState& a, const PState& b,
                                                  vec2<double> ovel, Geom& g) {
  vec2<double> va = V(a.vx, a.vy) + crossw(g.bv1, a.w);
  vec2<double> vb = (V(b.vx, b.vy) + ovel) + crossw(g.bv2, b.w);
  g.rv = va - vb;
  g.nrv = g.n * dot(g.rv, g.n);
  g.srv = g.rv - g.nrv;
}

// CircularParticle::contactWithCircularParticle (CircularParticle.cpp:67-92)
__device__ __forceinline__ bool circle_circle(const PState& a, const PState& b, vec2<double> off,
                                              vec2<double> ovel, Geom& g) {
  vec2<double> pa = V(a.x, a.y);
  vec2<double> pb = V(b.x, b.y) + off;
  vec2<double> branch = pb - pa;
  double distance = len(branch);
  double sumR = a.r + b.r;
  g.overlap = sumR - distance;
  if (g.overlap < 0.0) {
    g.contacted = 0;
    return false;
  }
  g.contacted = 1;
  g.n = unit(branch);
  vec2<double> p1 = pa + g.n * a.r;
  vec2<double> p2 = pb - g.n * b.r;
  g.cp = (p1 + p2) / 2.0;
  g.bv1 = g.cp - pa;
  g.bv2 = g.cp - pb;
  relative_velocity(a, b, ovel, g);
  return true;
}

// A fixed wall segment (SegmentObject.h:13-41): its vertices come as
// (x1, y1, x2, y2); PState holds its (possibly moved) position and its radius
// (half the vertex distance).  _dirVector = (v2 - v1).getUnitVector().
__device__ __forceinline__ vec2<double> seg_dir(double4 s) { return unit(V(s.z, s.w) - V(s.x, s.y)); }

// the segment's point of reference for a projection: a vertex beyond either
// end, else the projection itself (SegmentObject.cpp:51-62,
// CircularParticle.cpp:99-108)
__device__ __forceinline__ vec2<double> seg_ref(const PState& s, double4 v, vec2<double> dir,
                                                double proj) {
  if (proj > s.r) return V(v.z, v.w);
  if (proj < -s.r) return V(v.x, v.y);
  return V(s.x, s.y) + dir * proj;
}

// CircularParticle::contactWithSegmentObject (CircularParticle.cpp:94-129),
// the circle a is P1.  The reference adds the offset to the circle's own
// position when projecting and again to the reference point; kept as written.
__device__ __forceinline__ bool circle_segment(const PState& a, const PState& b, double4 vb,
                                               vec2<double> off, vec2<double> ovel, Geom& g) {
  const vec2<double> pa = V(a.x, a.y);
  const vec2<double> dir = seg_dir(vb);
  const double proj = dot((pa + off) - V(b.x, b.y), dir);
  const vec2<double> ref = seg_ref(b, vb, dir, proj);
  const vec2<double> branch = (ref + off) - pa;
  const double distance = len(branch);
  const double sumR = a.r;
  g.overlap = sumR - distance;
  if (g.overlap < 0.0) {
    g.contacted = 0;
    return false;
  }
  g.contacted = 1;
  g.n = unit(branch);
  g.cp = ref;
  g.bv1 = g.cp - pa;
  g.bv2 = g.cp - (ref + off);
  relative_velocity(a, b, ovel, g);
  return true;
}

// SegmentObject::contactWithCircularParticle (SegmentObject.cpp:45-80), the
// segment a is P1 (its branch vector to the contact point is zero)
__device__ __forceinline__ bool segment_circle(const PState& a, double4 va, const PState& b,
                                               vec2<double> off, vec2<double> ovel, Geom& g) {
  const vec2<double> dir = seg_dir(va);
  const vec2<double> pb = V(b.x, b.y) + off;
  const double proj = dot(pb - V(a.x, a.y), dir);
  const vec2<double> ref = seg_ref(a, va, dir, proj);
  const vec2<double> branch = pb - ref;
  const double distance = len(branch);
  const double sumR = b.r;
  g.overlap = sumR - distance;
  if (g.overlap < 0.0) {
    g.contacted = 0;
    return false;
  }
  g.contacted = 1;
  g.n = unit(branch);
  g.cp = ref;
  g.bv1 = g.cp - ref;
  g.bv2 = g.cp - pb;
  relative_velocity(a, b, ovel, g);
  return true;
}

// EllipticParticle::NewtonRaphsonForQuartic (EllipticParticle.cpp:613-626).
// The reference's iteration is a function of the iterate alone, so an iterate
// equal to an earlier one (not within the tolerance of its predecessor) means
// the loop would cycle forever there; Brent's cycle test (compare each
// iterate with the one saved at the last power-of-two step) finds such a
// repeat within twice the cycle's length after its start.  `stuck` is set
// on a repeat or at kNewtonCap iterations; the operations are the
// reference's, so wherever the reference returns, the result is its own.
__device__ __forceinline__ double newton_quartic(double A, double B, double C, double D, double E,
                                                 double init, int& iters, bool& stuck) {
  double A0 = 4.0 * A;
  double B0 = 3.0 * B;
  double C0 = 2.0 * C;
  double r0 = init;
  double r = 0.0;
  const double tol = 1e-10;
  int it = 0;
  double saved = init;
  int power = 1, lam = 0;
  stuck = false;
  while (fabs(r0 - r) > tol) {
    if (it >= kNewtonCap) {
      stuck = true;
      break;
    }
    r = r0;
    double p2 = r0 * r0;
    double p3 = p2 * r0;
    double p4 = p3 * r0;
    r0 -= (A * p4 + B * p3 + C * p2 + D * r0 + E) / (A0 * p3 + B0 * p2 + C0 * r0 + D);
    ++it;
    if (r0 == saved && fabs(r0 - r) > tol) {
      stuck = true;
      break;
    }
    if (++lam == power) {
      saved = r0;
      power <<= 1;
      lam = 0;
    }
  }
  iters = it;
  return r0;
}

// the quartic A q^4 + B q^3 + C q^2 + D q + E, Horner-free as in the Newton step
__device__ __forceinline__ double quartic_at(double A, double B, double C, double D, double E,
                                             double q) {
  double p2 = q * q;
  double p3 = p2 * q;
  double p4 = p3 * q;
  return A * p4 + B * p3 + C * p2 + D * q + E;
}

// Where the reference's Newton iteration never ends (newton_quartic's
// `stuck`), the root it is meant to find: the quartic's root in
// [min(1, s), max(1, s)], s = sqrt(δ+1) the analytic start, by bisection to
// adjacent doubles (no division, a fixed sequence of operations).  Without a
// sign change on that interval the iterate q is kept.
__device__ __forceinline__ double bisect_quartic(double A, double B, double C, double D, double E,
                                                 double s, double q) {
  double lo = fmin(1.0, s), hi = fmax(1.0, s);
  if (!(lo < hi)) return q;
  double flo = quartic_at(A, B, C, D, E, lo);
  const double fhi = quartic_at(A, B, C, D, E, hi);
  if (flo == 0.0) return lo;
  if (fhi == 0.0) return hi;
  if (!((flo < 0.0) != (fhi < 0.0))) return q;
  for (int k = 0; k < 80; ++k) {
    const double mid = 0.5 * (lo + hi);
    if (!(mid > lo && mid < hi)) break;
    const double fm = quartic_at(A, B, C, D, E, mid);
    if (fm == 0.0) return mid;
    if ((fm < 0.0) == (flo < 0.0)) {
      lo = mid;
      flo = fm;
    } else {
      hi = mid;
    }
  }
  return 0.5 * (lo + hi);
}

// Largest Newton step accepted at a learned warm start, relative to the start
constexpr double kWarmResidual = 0.05;

// EllipticParticle::contactWithEllipticParticle, closest approach
// (Zheng & Palffy-Muhoray), EllipticParticle.cpp:34-285.  (k1x, k1y) and
// (k2x, k2y) are cos/sin of the two orientations.
//
// WARM: `warm` is a predicted root as a fraction of the analytic start
// sqrt(δ+1) (mlp.cuh).  It is clamped to [min(1, s), max(1, s)], s = sqrt(δ+1),
// the interval of the closest-approach root; it is used only when the first
// Newton step from it is below kWarmResidual of it, and a root that leaves the
// interval is discarded for the plain iteration from s.  Newton then stops at
// the same tolerance, so the answer is the plain solver's wherever the plain
// iteration converges inside the interval.  It does not always: after a long
// wander the plain iteration can end at a root outside it (most often a
// negative one), which the reference then uses, and there the warm start's
// answer differs.
template <bool WARM = false>
__device__ __forceinline__ bool ellipse_closest(const PState& a, const PState& b, vec2<double> off,
                                                vec2<double> ovel, double k1x, double k1y,
                                                double k2x, double k2y, Geom& g, uint32_t& st,
                                                float warm = 0.0f) {
  double a1 = a.r, a2 = b.r;
  double b1 = a1 / a.asp, b2 = a2 / b.asp;
  vec2<double> pa = V(a.x, a.y);
  vec2<double> pb = V(b.x, b.y) + off;
  vec2<double> d = pb - pa;
  double dlen = len(d);
  vec2<double> d_hat = d / dlen;
  vec2<double> k1 = V(k1x, k1y);
  vec2<double> k2 = V(k2x, k2y);
  mat2<double> k1k1 = dyad(k1, k1);
  mat2<double> k2k2 = dyad(k2, k2);
  double e1 = sqrt(1.0 - (b1 * b1) / (a1 * a1));
  double e2 = sqrt(1.0 - (b2 * b2) / (a2 * a2));
  mat2<double> I = M(1.0, 0.0, 0.0, 1.0);
  mat2<double> T = (I + k1k1 * (b1 / a1 - 1.0)) / b1;
  double eta = a1 / b1 - 1.0;
  vec2<double> dph = T * d_hat;
  vec2<double> dp0 = T * d;
  mat2<double> P = I + k1k1 * eta;
  mat2<double> Q = I - k2k2 * (e2 * e2);
  mat2<double> Ap = (matmul_ref(matmul_ref(P, Q), P) * (b1 * b1)) / (b2 * b2);
  // matrix2d::eigen (MathMatrix2d.h:112-135)
  double tr = Ap.xx + Ap.yy;
  double dt_ = det(Ap);
  double dl = tr * tr - 4.0 * dt_;
  if (dl < 0) dl = 0.0;
  dl = sqrt(dl);
  double ev1 = (tr + dl) / 2.0;
  double ev2 = (tr - dl) / 2.0;
  double lx, ly;
  if (trunc_abs(ev1) > trunc_abs(ev2)) {
    lx = ev1;
    ly = ev2;
  } else {
    lx = ev2;
    ly = ev1;
  }
  vec2<double> kpp = normalize(V(1.0, (lx - Ap.xx) / Ap.xy), st);
  vec2<double> kpm = normalize(V(1.0, (ly - Ap.xx) / Ap.xy), st);
  double a2p = 1.0 / sqrt(ly);
  double b2p = 1.0 / sqrt(lx);
  if (len(dp0) > 1.0 + a2p) {
    g.contacted = 0;
    return false;
  }
  if (fabs(dot(dp0, kpp)) > 1.0 + b2p) {
    g.contacted = 0;
    return false;
  }
  if (dot(kpm, dph) < 0) kpm = -kpm;
  if (dot(kpp, dph) < 0) kpp = -kpp;
  double delta = (a2p * a2p) / (b2p * b2p) - 1;
  double tanPhi = dot(kpm, dph) / dot(kpp, dph);
  double tanPhi2 = tanPhi * tanPhi;
  double A = -(1.0 + tanPhi2) / (b2p * b2p);
  double B = -2.0 * (1.0 + tanPhi2 + delta) / b2p;
  double C = -tanPhi2 - (1.0 + delta) * (1.0 + delta) + (1.0 + (1.0 + delta) * tanPhi2) / (b2p * b2p);
  double D = 2.0 * (1.0 + tanPhi2) * (1.0 + delta) / b2p;
  double E = (1.0 + tanPhi2 + delta) * (1.0 + delta);
  int it = 0;
  const double start = sqrt(delta + 1.0);
  double init = start;
  double lo = 0.0, hi = 0.0;
  if (WARM) {
    lo = fmin(1.0, start);
    hi = fmax(1.0, start);
    g.warm = 2;
    double q0 = (double)warm * start;
    if (isfinite(q0)) {
      q0 = fmin(fmax(q0, lo), hi);
      const double f = A * q0 * q0 * q0 * q0 + B * q0 * q0 * q0 + C * q0 * q0 + D * q0 + E;
      const double fp = 4.0 * A * q0 * q0 * q0 + 3.0 * B * q0 * q0 + 2.0 * C * q0 + D;
      if (fabs(f) <= kWarmResidual * q0 * fabs(fp)) {
        init = q0;
        g.warm = 1;
      }
    }
  }
  bool stuck = false;
  double q = newton_quartic(A, B, C, D, E, init, it, stuck);
  if (WARM && g.warm == 1 && (stuck || !(q >= lo * (1.0 - 1e-9) && q <= hi * (1.0 + 1e-9)))) {
    int it2 = 0;
    q = newton_quartic(A, B, C, D, E, start, it2, stuck);
    it += it2;
    g.warm = 3;
  }
  if (stuck) {
    q = bisect_quartic(A, B, C, D, E, start, q);
    st |= ST_NEWTON;
  }
  g.iters = it;
  g.stuck = stuck ? 1 : 0;
  g.q = q;
  g.q_start = start;
  double temp = (q * q - 1.0) / delta;
  double d_prime = 0.0;
  if (temp < 0) temp = 0.0;
  if (delta == 0 || !isfinite(temp)) {
    d_prime = 1.0 + a2p;
  } else {
    double u = (1.0 + b2p * (1.0 + delta) / q);
    double v = 1.0 + b2p / q;
    d_prime = sqrt(temp * (u * u) + (1.0 - temp) * (v * v));
  }
  double dk = dot(k1, d_hat);
  double dist = d_prime / sqrt(1.0 - (dk * dk) * (e1 * e1)) * b1;
  double overlap0 = dist - dlen;
  if (overlap0 < 0.0) {
    g.contacted = 0;
    return false;
  }
  vec2<double> tangentPoint;
  if (delta == 0) {
    tangentPoint = inv(T) * d_hat;
  } else {
    double sinPsi2 = (q * q - 1.0) / delta;
    if (sinPsi2 < 0) sinPsi2 = 0.0;
    double cosPsi2 = 1.0 - sinPsi2;
    if (cosPsi2 < 0) cosPsi2 = 0.0;
    mat2<double> Kinv = M(kpm.x, kpp.x, kpm.y, kpp.y);
    tangentPoint = inv(T) * (Kinv * V(sqrt(sinPsi2), sqrt(cosPsi2)));
  }
  vec2<double> contactPoint = (tangentPoint * dlen) / dist;
  mat2<double> A1 = (I - k1k1 * (e1 * e1)) / (b1 * b1);
  vec2<double> cn = normalize(A1 * tangentPoint, st);
  vec2<double> ov = d_hat * overlap0;
  ov = cn * dot(ov, cn);
  g.contacted = 1;
  g.cp = contactPoint + pa;
  g.n = cn;
  g.overlap = len(ov);
  g.bv1 = g.cp - pa;
  g.bv2 = g.cp - pb;
  relative_velocity(a, b, ovel, g);
  return true;
}

// EllipticParticle::solveQuarticGeneral (EllipticParticle.cpp:521-554)
__device__ __forceinline__ bool solve_quartic_general(double a, double b, double c, double d,
                                                      double e, double& aI, double& bI,
                                                      double& gI, double& dI) {
  double delta0 = c * c - 3.0 * b * d + 12.0 * a * e;
  double delta1 = 2.0 * c * c * c - 9.0 * b * c * d + 27.0 * b * b * e + 27.0 * a * d * d -
                  72.0 * a * c * e;
  double delta = (delta1 * delta1 - 4.0 * delta0 * delta0 * delta0) / (-27.0);
  if (delta <= 1e-12 && delta > 0.0) {
    delta = 0.0;
  } else if (delta > 1e-12) {
    return false;
  }
  double p = (8.0 * a * c - 3.0 * b * b) / (8.0 * a * a);
  double q = (b * b * b - 4.0 * a * b * c + 8.0 * a * a * d) / (8.0 * a * a * a);
  double t = (delta1 + sqrt(delta * (-27.0))) / 2.0;
  t = pow(t, 1. / 3.);
  double temp = (-2.0 / 3.0) * p + (t + delta0 / t) / (3.0 * a);
  if (temp <= 0.0) return false;
  double s = 0.5 * sqrt(temp);
  aI = -(-b / (2.0 * a) - 2.0 * s);
  bI = (-b / (4.0 * a) - s) * (-b / (4.0 * a) - s) - 0.25 * (-4.0 * s * s - 2.0 * p + q / s);
  gI = -(-b / (2.0 * a) + 2.0 * s);
  dI = (-b / (4.0 * a) + s) * (-b / (4.0 * a) + s) - 0.25 * (-4.0 * s * s - 2.0 * p - q / s);
  return true;
}

// EllipticParticle::fastQuarticSolver (Strobach 2010), EllipticParticle.cpp:559-609
__device__ __forceinline__ void fast_quartic(double a, double b, double c, double d, double& alpha,
                                             double& beta, double& gamma, double& delta) {
  double e1 = a - alpha - gamma;
  double e2 = b - beta - alpha * gamma - delta;
  double e3 = c - beta * gamma - alpha * delta;
  double e4 = d - beta * delta;
  double e_old = fabs(e1) + fabs(e2) + fabs(e3) + fabs(e4);
  double e_new = 1.0;
  int counter = 0;
  while (fabs((e_old - e_new) / e_old) >= 1e-3) {
    e_old = e_new;
    counter++;
    if (counter > 20) break;
    double u23 = alpha - gamma;
    double u33 = beta - delta - gamma * u23;
    double L43 = -delta * u23 / u33;
    double u44 = beta - delta - L43 * u23;
    double x1 = e1;
    double x2 = e2 - gamma * x1;
    double x3 = e3 - delta * x1 - gamma * x2;
    double x4 = e4 - delta * x2 - L43 * x3;
    double y4 = x4 / u44;
    double y3 = (x3 - u23 * y4) / u33;
    double y2 = x2 - u23 * y3 - y4;
    double y1 = x1 - y3;
    alpha = alpha + y1;
    beta = beta + y2;
    gamma = gamma + y3;
    delta = delta + y4;
    e1 = a - alpha - gamma;
    e2 = b - beta - alpha * gamma - delta;
    e3 = c - beta * gamma - alpha * delta;
    e4 = d - beta * delta;
    e_new = fabs(e1) + fabs(e2) + fabs(e3) + fabs(e4);
    if (e_new < 1e-8) break;
  }
}

// square of a value, standing for pow(v, 2) of the reference (pow with an
// exponent of 2 returns the correctly rounded square)
__device__ __forceinline__ double sq(double v) { return v * v; }

// boundary distance along the line of slope k through cp
// (EllipticParticle.cpp:417-431, :433-447)
__device__ __forceinline__ double chord_half(double cz, double sz, double ax, double bx, double xc,
                                             double yc, vec2<double> cp, double k) {
  double aa = sq(cz / ax) + sq(sz / bx);
  double bb = sq(sz / ax) + sq(cz / bx);
  double cc = cz * sz * (1.0 / ax / ax - 1.0 / bx / bx);
  double alpha = cp.y - yc - k * cp.x;
  double p1 = aa + bb * k * k + 2.0 * cc * k;
  double p2 = -2.0 * aa * xc + 2.0 * bb * k * alpha + 2.0 * cc * (alpha - k * xc);
  double p3 = aa * xc * xc + bb * alpha * alpha - 2.0 * cc * alpha * xc - 1.0;
  double dd = sqrt(p2 * p2 - 4.0 * p1 * p3);
  double xo1 = (-p2 - dd) / (2.0 * p1);
  double xo2 = (-p2 + dd) / (2.0 * p1);
  double yo1 = k * (xo1 - cp.x) + cp.y;
  double yo2 = k * (xo2 - cp.x) + cp.y;
  double d1 = sq(xo1 - cp.x) + sq(yo1 - cp.y);
  double d2 = sq(xo2 - cp.x) + sq(yo2 - cp.y);
  return (d1 > d2) ? sqrt(d2) : sqrt(d1);
}

// EllipticParticle::contactWithEllipticParticle0, intersection (Strobach),
// EllipticParticle.cpp:288-484.  (czi, szi), (czj, szj): cos/sin of the
// orientations.
__device__ __forceinline__ bool ellipse_intersection(const PState& A_, const PState& B_,
                                                     vec2<double> off, vec2<double> ovel,
                                                     double czi, double szi, double czj,
                                                     double szj, Geom& g) {
  double ai = A_.r, aj = B_.r;
  double bi = ai / A_.asp, bj = aj / B_.asp;
  double xi = A_.x, xj = B_.x + off.x;
  double yi = A_.y, yj = B_.y + off.y;
  double z0 = B_.rot - A_.rot;
  double x0 = (xj - xi) * czi + (yj - yi) * szi;
  double y0 = -(xj - xi) * szi + (yj - yi) * czi;
  double cz0 = cos(z0), sz0 = sin(z0), s2z0 = sin(2.0 * z0);
  double c0 = sq(cz0 / aj) + sq(sz0 / bj);
  double c1 = sq(sz0 / aj) + sq(cz0 / bj);
  double c2 = s2z0 / aj / aj - s2z0 / bj / bj;
  double c3 = -2.0 * x0 * c0 - y0 * c2;
  double c4 = -2.0 * y0 * c1 - x0 * c2;
  double c5 = x0 * x0 * c0 + y0 * y0 * c1 + x0 * y0 * c2 - 1.0;
  double kk = bi * bi / (ai * ai);
  double p0 = kk * c2 * c2 + sq(c0 - c1 * kk);
  double p1 = 2.0 * kk * c2 * c4 + 2.0 * (c0 - c1 * kk) * c3;
  double p2 = -kk * c2 * c2 * ai * ai + kk * c4 * c4 + 2.0 * (c0 - c1 * kk) * (c5 + c1 * kk * ai * ai) +
              c3 * c3;
  double p3 = 2.0 * c3 * (c5 + c1 * kk * ai * ai) - 2.0 * kk * c2 * c4 * ai * ai;
  double p4 = sq((c5 + c1 * kk * ai * ai)) - kk * c4 * c4 * ai * ai;
  double alpha, beta, gamma, delta;
  g.iters = 0;
  if (!solve_quartic_general(p0, p1, p2, p3, p4, alpha, beta, gamma, delta)) {
    g.contacted = 0;
    return false;
  }
  p1 /= p0;
  p2 /= p0;
  p3 /= p0;
  p4 /= p0;
  fast_quartic(p1, p2, p3, p4, alpha, beta, gamma, delta);
  double xr[2], yr[2];
  double delta1 = alpha * alpha - 4.0 * beta;
  double delta2 = gamma * gamma - 4.0 * delta;
  if (delta1 >= delta2) {
    xr[0] = (-alpha - sqrt(delta1)) / 2.0;
    xr[1] = (-alpha + sqrt(delta1)) / 2.0;
  } else {
    xr[0] = (-gamma + sqrt(delta2)) / 2.0;
    xr[1] = (-gamma - sqrt(delta2)) / 2.0;
  }
  if (fabs(xr[0]) / ai > 1.0 && fabs(xr[0]) / ai <= 1.0 + 1e-6) xr[0] = copysign(ai, xr[0]);
  if (fabs(xr[1]) / ai > 1.0 && fabs(xr[1]) / ai <= 1.0 + 1e-6) xr[1] = copysign(ai, xr[1]);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    yr[i] = bi * sqrt(1.0 - sq(xr[i] / ai));
    double err1 = c0 * xr[i] * xr[i] + c1 * yr[i] * yr[i] + c2 * xr[i] * yr[i] + c3 * xr[i] +
                  c4 * yr[i] + c5;
    double err2 = c0 * xr[i] * xr[i] + c1 * yr[i] * yr[i] - c2 * xr[i] * yr[i] + c3 * xr[i] -
                  c4 * yr[i] + c5;
    yr[i] = (fabs(err1) <= fabs(err2)) ? yr[i] : -yr[i];
    if (std_min(fabs(err1), fabs(err2)) > 1e-8 || !isfinite(yr[i]) || fabs(yr[i]) > bi) {
      g.contacted = 0;
      return false;
    }
  }
  vec2<double> cp1 = V(xr[0] * czi - yr[0] * szi + xi, xr[0] * szi + yr[0] * czi + yi);
  vec2<double> cp2 = V(xr[1] * czi - yr[1] * szi + xi, xr[1] * szi + yr[1] * czi + yi);
  g.cp = (cp1 + cp2) / 2.0;
  if (!isfinite(len(g.cp))) {
    g.contacted = 0;
    return false;
  }
  vec2<double> tangent = cp1 - cp2;
  if (len(tangent) == 0.0) {
    g.contacted = 0;
    return false;
  }
  uint32_t dummy = 0;
  tangent = normalize(tangent, dummy);
  g.n = V(tangent.y, -tangent.x);
  if (!isfinite(len(g.n))) {
    g.contacted = 0;
    return false;
  }
  vec2<double> bv = g.cp - V(xi, yi);
  if (dot(g.n, bv) < 0.0) g.n = -g.n;
  double k = g.n.y / g.n.x;
  if (fabs(k) > 100000) k = copysign(100000.0, k);
  if (!isfinite(k)) k = (g.n.y > 0) ? 100000.0 : -100000.0;
  double disti = chord_half(czi, szi, ai, bi, xi, yi, g.cp, k);
  double distj = chord_half(czj, szj, aj, bj, xj, yj, g.cp, k);
  g.overlap = disti + distj;
  if (!isfinite(disti)) g.overlap = 2.0 * distj;
  if (!isfinite(distj)) g.overlap = 2.0 * disti;
  g.contacted = 1;
  g.bv1 = g.cp - V(A_.x, A_.y);
  g.bv2 = g.cp - V(xj, yj);
  relative_velocity(A_, B_, ovel, g);
  if (!isfinite(g.overlap)) {
    g.contacted = 0;
    return false;
  }
  return true;
}

// Contact laws a world can be specialised for: all circles, all ellipses with
// one of the two methods, or any mix (dispatched per pair).
enum : int { LAW_CIRCLE = 0, LAW_CLOSEST = 1, LAW_INTERSECTION = 2, LAW_ANY = 3 };

// calculateContactGeometry for a world whose bodies all have one shape; the
// clump test stays (a clump's geometry is never a contact, GluedParticle.cpp:133-140)
// (SCREENED: the caller has already applied the bounding-circle test)
template <int LAW, bool SCREENED = false, bool WARM = false>
__device__ __forceinline__ bool contact_geometry_law(const PState& a, const PState& b,
                                                     double orad_a, double orad_b,
                                                     vec2<double> off, vec2<double> ovel,
                                                     double2 cs_a, double2 cs_b, Geom& g,
                                                     uint32_t& st, float warm = 0.0f) {
  g = Geom{};
  if (a.shape == SHAPE_CLUMP || b.shape == SHAPE_CLUMP) return false;
  if (LAW == LAW_CIRCLE) return circle_circle(a, b, off, ovel, g);
  // EllipticParticle::calculateContactGeometry (EllipticParticle.cpp:16-32)
  if (!SCREENED) {
    vec2<double> dd = V(a.x, a.y) - (V(b.x, b.y) + off);
    if (!((orad_a + orad_b) > sqrt(len2(dd)))) return false;
  }
  if (LAW == LAW_INTERSECTION)
    return ellipse_intersection(a, b, off, ovel, cs_a.x, cs_a.y, cs_b.x, cs_b.y, g);
  return ellipse_closest<WARM>(a, b, off, ovel, cs_a.x, cs_a.y, cs_b.x, cs_b.y, g, st, warm);
}

// BaseParticle::calculateContactGeometry dispatch (CircularParticle.cpp:25-40,
// EllipticParticle.cpp:16-32 with its coarse bounding-circle test,
// GluedParticle.cpp:133-140, SegmentObject.cpp:12-27).  cs_a/cs_b: (cos, sin)
// of each orientation; va/vb: the vertices of a segment.
__device__ __forceinline__ bool contact_geometry(int method, const PState& a, const PState& b,
                                                 double orad_a, double orad_b, vec2<double> off,
                                                 vec2<double> ovel, double2 cs_a, double2 cs_b,
                                                 Geom& g, uint32_t& st,
                                                 double4 va = double4{}, double4 vb = double4{}) {
  g = Geom{};
  if (a.shape == SHAPE_CLUMP || b.shape == SHAPE_CLUMP) return false;
  if (a.shape == SHAPE_SEGMENT) {
    if (b.shape == SHAPE_SEGMENT) return false;  // SegmentObject.cpp:20-22
    if (b.shape != SHAPE_CIRCLE) {
      st |= ST_UNSUPPORTED;
      return false;
    }
    return segment_circle(a, va, b, off, ovel, g);
  }
  if (a.shape == SHAPE_CIRCLE) {
    if (b.shape == SHAPE_SEGMENT) return circle_segment(a, b, vb, off, ovel, g);
    if (b.shape != SHAPE_CIRCLE) {
      st |= ST_UNSUPPORTED;
      return false;
    }
    return circle_circle(a, b, off, ovel, g);
  }
  if (b.shape != SHAPE_ELLIPSE) {
    st |= ST_UNSUPPORTED;
    return false;
  }
  vec2<double> dd = V(a.x, a.y) - (V(b.x, b.y) + off);
  if (!((orad_a + orad_b) > sqrt(len2(dd)))) return false;
  if (method == ELLIPSE_INTERSECTION)
    return ellipse_intersection(a, b, off, ovel, cs_a.x, cs_a.y, cs_b.x, cs_b.y, g);
  return ellipse_closest(a, b, off, ovel, cs_a.x, cs_a.y, cs_b.x, cs_b.y, g, st);
}

}  // namespace xdem
