/* xdem_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU checker of the CUDA path.
 *
 * A C restatement of xDEM's per-timestep path.  Every routine cites the
 * reference function it restates and keeps that function's floating-point
 * operation order, and it calls the same libm functions (cos, sin, atan2, pow,
 * sqrt), so that with -ffp-contract=off its per-contact results are
 * bit-identical to the compiled reference.  See xdem_oracle.h for the three
 * deliberate differences.  Never linked by the product.
 */
#include "xdem_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* 2-D helpers (MathVector.h, MathMatrix2d.h)                                 */
/* ------------------------------------------------------------------------- */
typedef struct { double x, y; } v2;
typedef struct { double xx, xy, yx, yy; } m2;

static inline v2 V(double x, double y) { v2 r = {x, y}; return r; }
static inline v2 vadd(v2 a, v2 b) { return V(a.x + b.x, a.y + b.y); }
static inline v2 vsub(v2 a, v2 b) { return V(a.x - b.x, a.y - b.y); }
static inline v2 vneg(v2 a) { return V(-a.x, -a.y); }
static inline v2 vmul(v2 a, double f) { return V(a.x * f, a.y * f); }
static inline v2 vdiv(v2 a, double f) { return V(a.x / f, a.y / f); }
static inline double vdot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline double vcross(v2 a, v2 b) { return a.x * b.y - a.y * b.x; }
/* vector2d::cross(omega) (MathVector.h:202-205) */
static inline v2 vcrossw(v2 a, double w) { return V(-w * a.y, w * a.x); }
static inline double vlen2(v2 a) { return a.x * a.x + a.y * a.y; }
static inline double vlen(v2 a) { return sqrt(vlen2(a)); }
/* getUnitVector (MathVector.h:169-178) */
static inline v2 vunit(v2 a) {
  double l2 = vlen2(a);
  if (l2 != 0.0) return vdiv(a, sqrt(l2));
  return V(0.0, 0.0);
}
/* normalize (MathVector.h:180-190): zero length is an error */
static inline v2 vnormalize(v2 a, uint32_t* st) {
  double l2 = vlen2(a);
  if (l2 != 0.0) return vdiv(a, sqrt(l2));
  *st |= XDEM_ERR_ZERO_VECTOR;
  return a;
}

static inline m2 M(double xx, double xy, double yx, double yy) {
  m2 r = {xx, xy, yx, yy};
  return r;
}
static inline m2 madd(m2 a, m2 b) { return M(a.xx + b.xx, a.xy + b.xy, a.yx + b.yx, a.yy + b.yy); }
static inline m2 msub(m2 a, m2 b) { return M(a.xx - b.xx, a.xy - b.xy, a.yx - b.yx, a.yy - b.yy); }
static inline m2 mmuls(m2 a, double f) { return M(a.xx * f, a.xy * f, a.yx * f, a.yy * f); }
static inline m2 mdivs(m2 a, double f) { return M(a.xx / f, a.xy / f, a.yx / f, a.yy / f); }
static inline v2 mmulv(m2 a, v2 v) { return V(a.xx * v.x + a.xy * v.y, a.yx * v.x + a.yy * v.y); }
/* matrix2d::operator*(matrix2d) as written (MathMatrix2d.h:85-91): the yy
   entry uses other.yx() */
static inline m2 mmulm(m2 a, m2 o) {
  return M(a.xx * o.xx + a.xy * o.yx, a.xx * o.xy + a.xy * o.yy, a.yx * o.xx + a.yy * o.yx,
           a.yx * o.yx + a.yy * o.yy);
}
static inline m2 mdyad(v2 a, v2 b) { return M(a.x * b.x, a.x * b.y, a.y * b.x, a.y * b.y); }
static inline double mdet(m2 a) { return a.xx * a.yy - a.xy * a.yx; }
/* matrix2d::inv (MathMatrix2d.h:137-140) */
static inline m2 minv(m2 a) { return mdivs(M(a.yy, -a.xy, -a.yx, a.xx), mdet(a)); }
static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
/* int abs(int) applied to a double argument: the conversion truncates toward
   zero; x86-64 turns NaN and out-of-range values into INT_MIN, whose abs()
   stays INT_MIN */
static inline int trunc_abs(double x) {
  if (!(fabs(x) < 2147483648.0)) return INT32_MIN;
  int i = (int)x;
  return i < 0 ? -i : i;
}

/* ------------------------------------------------------------------------- */
/* Contact geometry (ContactGeometry.h)                                       */
/* ------------------------------------------------------------------------- */
typedef struct {
  int contacted;
  v2 cp, n, bv1, bv2;
  double overlap;
  v2 rv, nrv, srv;
  int iters;
  /* closest approach: the quartic A..E, the analytic start s, the root q and
     whether Newton did not terminate (xo_closest_quartic) */
  double quartic[5], q_start, q;
  int stuck;
} geom_t;

typedef struct {
  int shape;
  double r, asp, x, y, vx, vy, rot, w;
  v2 s1, s2; /* segment: _vertex1, _vertex2 */
} pstate_t;

/* BaseParticle::calculateRelativeVelocityAtContactPoint (BaseParticle.cpp:11-25) */
static void relative_velocity(const pstate_t* a, const pstate_t* b, v2 ovel, geom_t* g) {
  v2 va = vadd(V(a->vx, a->vy), vcrossw(g->bv1, a->w));
  v2 vb = vadd(vadd(V(b->vx, b->vy), ovel), vcrossw(g->bv2, b->w));
  g->rv = vsub(va, vb);
  g->nrv = vmul(g->n, vdot(g->rv, g->n));
  g->srv = vsub(g->rv, g->nrv);
}

/* CircularParticle::contactWithCircularParticle (CircularParticle.cpp:67-92) */
static int circle_circle(const pstate_t* a, const pstate_t* b, v2 off, v2 ovel, geom_t* g) {
  v2 pa = V(a->x, a->y);
  v2 pb = vadd(V(b->x, b->y), off);
  v2 branch = vsub(pb, pa);
  double distance = vlen(branch);
  double sumR = a->r + b->r;
  g->overlap = sumR - distance;
  if (g->overlap < 0.0) { g->contacted = 0; return 0; }
  g->contacted = 1;
  g->n = vunit(branch);
  v2 p1 = vadd(pa, vmul(g->n, a->r));
  v2 p2 = vsub(pb, vmul(g->n, b->r));
  g->cp = vdiv(vadd(p1, p2), 2.0);
  g->bv1 = vsub(g->cp, pa);
  g->bv2 = vsub(g->cp, pb);
  relative_velocity(a, b, ovel, g);
  return 1;
}

/* EllipticParticle::NewtonRaphsonForQuartic (EllipticParticle.cpp:613-626).
   The reference's loop has no cap and never ends on some deeply overlapping
   pairs.  Its iteration is a function of the iterate alone, so an iterate
   equal to an earlier one (and not within the tolerance of its predecessor)
   means the loop cycles forever; Brent's test (compare each iterate with the
   one saved at the last power-of-two step) finds the repeat.  *stuck is set on
   a repeat or at XO_NEWTON_CAP iterations; otherwise the result is the
   reference's. */
double xo_newton_quartic(double A, double B, double C, double D, double E, double init,
                         int32_t* iters, int32_t* stuck) {
  double A0 = 4.0 * A;
  double B0 = 3.0 * B;
  double C0 = 2.0 * C;
  double r0 = init;
  double r = 0.0;
  double tol = 1e-10;
  int it = 0;
  double saved = init;
  int power = 1, lam = 0;
  int st = 0;
  while (fabs(r0 - r) > tol) {
    if (it >= XO_NEWTON_CAP) {
      st = 1;
      break;
    }
    r = r0;
    r0 -= (A * (r0 * r0 * r0 * r0) + B * (r0 * r0 * r0) + C * (r0 * r0) + D * r0 + E) /
          (A0 * (r0 * r0 * r0) + B0 * (r0 * r0) + C0 * r0 + D);
    ++it;
    if (r0 == saved && fabs(r0 - r) > tol) {
      st = 1;
      break;
    }
    if (++lam == power) {
      saved = r0;
      power <<= 1;
      lam = 0;
    }
  }
  if (iters) *iters = it;
  if (stuck) *stuck = st;
  return r0;
}

static double quartic_at(double A, double B, double C, double D, double E, double q) {
  return A * (q * q * q * q) + B * (q * q * q) + C * (q * q) + D * q + E;
}

/* Where the Newton iteration never ends: the quartic's root in
   [min(1, s), max(1, s)] (s = sqrt(δ+1), the analytic start) by bisection to
   adjacent doubles; without a sign change there the iterate q is kept. */
double xo_bisect_quartic(double A, double B, double C, double D, double E, double s, double q) {
  double lo = fmin(1.0, s), hi = fmax(1.0, s);
  if (!(lo < hi)) return q;
  double flo = quartic_at(A, B, C, D, E, lo);
  double fhi = quartic_at(A, B, C, D, E, hi);
  if (flo == 0.0) return lo;
  if (fhi == 0.0) return hi;
  if (!((flo < 0.0) != (fhi < 0.0))) return q;
  for (int k = 0; k < 80; ++k) {
    double mid = 0.5 * (lo + hi);
    if (!(mid > lo && mid < hi)) break;
    double fm = quartic_at(A, B, C, D, E, mid);
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

/* EllipticParticle::contactWithEllipticParticle, closest approach
   (Zheng & Palffy-Muhoray), EllipticParticle.cpp:34-285 */
static int ellipse_closest(const pstate_t* a, const pstate_t* b, v2 off, v2 ovel, geom_t* g,
                           uint32_t* st) {
  double a1 = a->r, a2 = b->r;
  double b1 = a1 / a->asp, b2 = a2 / b->asp;
  double z1 = a->rot, z2 = b->rot;
  v2 pa = V(a->x, a->y);
  v2 pb = vadd(V(b->x, b->y), off);
  v2 d = vsub(pb, pa);
  v2 d_hat = vdiv(d, vlen(d));
  v2 k1 = V(cos(z1), sin(z1));
  v2 k2 = V(cos(z2), sin(z2));
  m2 k1k1 = mdyad(k1, k1);
  m2 k2k2 = mdyad(k2, k2);
  double e1 = sqrt(1.0 - (b1 * b1) / (a1 * a1));
  double e2 = sqrt(1.0 - (b2 * b2) / (a2 * a2));
  m2 I = M(1.0, 0.0, 0.0, 1.0);
  m2 T = mdivs(madd(I, mmuls(k1k1, b1 / a1 - 1.0)), b1);
  double eta = a1 / b1 - 1.0;
  v2 d_prime_hat = mmulv(T, d_hat);
  v2 d_prime0 = mmulv(T, d);
  m2 P = madd(I, mmuls(k1k1, eta));
  m2 Q = msub(I, mmuls(k2k2, e2 * e2));
  m2 A_prime = mdivs(mmuls(mmulm(mmulm(P, Q), P), b1 * b1), b2 * b2);
  /* matrix2d::eigen (MathMatrix2d.h:112-135) */
  double tr = A_prime.xx + A_prime.yy;
  double det = mdet(A_prime);
  double dl = tr * tr - 4.0 * det;
  if (dl < 0) dl = 0.0;
  dl = sqrt(dl);
  double ev1 = (tr + dl) / 2.0;
  double ev2 = (tr - dl) / 2.0;
  v2 lambda;
  /* MathMatrix2d.h:122 is compiled where only int abs(int) is declared, so
     the eigenvalues are compared by their truncated integer magnitudes */
  if (trunc_abs(ev1) > trunc_abs(ev2)) lambda = V(ev1, ev2);
  else lambda = V(ev2, ev1);
  v2 kpp = vnormalize(V(1.0, (lambda.x - A_prime.xx) / A_prime.xy), st);
  v2 kpm = vnormalize(V(1.0, (lambda.y - A_prime.xx) / A_prime.xy), st);
  double a2p = 1.0 / sqrt(lambda.y);
  double b2p = 1.0 / sqrt(lambda.x);
  if (vlen(d_prime0) > 1.0 + a2p) { g->contacted = 0; return 0; }
  if (fabs(vdot(d_prime0, kpp)) > 1.0 + b2p) { g->contacted = 0; return 0; }
  if (vdot(kpm, d_prime_hat) < 0) kpm = vneg(kpm);
  if (vdot(kpp, d_prime_hat) < 0) kpp = vneg(kpp);
  double delta = (a2p * a2p) / (b2p * b2p) - 1;
  double tanPhi = vdot(kpm, d_prime_hat) / vdot(kpp, d_prime_hat);
  double tanPhi2 = tanPhi * tanPhi;
  double A = -(1.0 + tanPhi2) / (b2p * b2p);
  double B = -2.0 * (1.0 + tanPhi2 + delta) / b2p;
  double C = -tanPhi2 - (1.0 + delta) * (1.0 + delta) + (1.0 + (1.0 + delta) * tanPhi2) / (b2p * b2p);
  double D = 2.0 * (1.0 + tanPhi2) * (1.0 + delta) / b2p;
  double E = (1.0 + tanPhi2 + delta) * (1.0 + delta);
  int32_t it = 0, stuck = 0;
  double start = sqrt(delta + 1.0);
  double q = xo_newton_quartic(A, B, C, D, E, start, &it, &stuck);
  if (stuck) {
    q = xo_bisect_quartic(A, B, C, D, E, start, q);
    *st |= XDEM_ERR_NEWTON;
  }
  g->iters = it;
  g->quartic[0] = A; g->quartic[1] = B; g->quartic[2] = C; g->quartic[3] = D; g->quartic[4] = E;
  g->q_start = start;
  g->q = q;
  g->stuck = stuck;
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
  double dk = vdot(k1, d_hat);
  double dist = d_prime / sqrt(1.0 - (dk * dk) * (e1 * e1)) * b1;
  double dlen = vlen(d);
  double overlap0 = dist - dlen;
  if (overlap0 < 0.0) { g->contacted = 0; return 0; }
  v2 tangentPoint;
  if (delta == 0) {
    tangentPoint = mmulv(minv(T), d_hat);
  } else {
    double sinPsi2 = (q * q - 1.0) / delta;
    if (sinPsi2 < 0) sinPsi2 = 0.0;
    double cosPsi2 = 1.0 - sinPsi2;
    if (cosPsi2 < 0) cosPsi2 = 0.0;
    m2 Kinv = M(kpm.x, kpp.x, kpm.y, kpp.y);
    tangentPoint = mmulv(minv(T), mmulv(Kinv, V(sqrt(sinPsi2), sqrt(cosPsi2))));
  }
  v2 contactPoint = vdiv(vmul(tangentPoint, dlen), dist);
  m2 A1 = mdivs(msub(I, mmuls(k1k1, e1 * e1)), b1 * b1);
  v2 cn = vnormalize(mmulv(A1, tangentPoint), st);
  v2 ov = vmul(d_hat, overlap0);
  ov = vmul(cn, vdot(ov, cn));
  g->contacted = 1;
  g->cp = vadd(contactPoint, pa);
  g->n = cn;
  g->overlap = vlen(ov);
  g->bv1 = vsub(g->cp, pa);
  g->bv2 = vsub(g->cp, pb);
  relative_velocity(a, b, ovel, g);
  return 1;
}

/* EllipticParticle::solveQuarticGeneral (EllipticParticle.cpp:521-554) */
static int solve_quartic_general(double a, double b, double c, double d, double e, double* aI,
                                 double* bI, double* gI, double* dI) {
  double delta0 = c * c - 3.0 * b * d + 12.0 * a * e;
  double delta1 = 2.0 * c * c * c - 9.0 * b * c * d + 27.0 * b * b * e + 27.0 * a * d * d -
                  72.0 * a * c * e;
  double delta = (delta1 * delta1 - 4.0 * delta0 * delta0 * delta0) / (-27.0);
  if (delta <= 1e-12 && delta > 0.0) {
    delta = 0.0;
  } else if (delta > 1e-12) {
    return 0;
  }
  double p = (8.0 * a * c - 3.0 * b * b) / (8.0 * a * a);
  double q = (b * b * b - 4.0 * a * b * c + 8.0 * a * a * d) / (8.0 * a * a * a);
  double t = (delta1 + sqrt(delta * (-27.0))) / 2.0;
  t = pow(t, 1. / 3.);
  double temp = (-2.0 / 3.0) * p + (t + delta0 / t) / (3.0 * a);
  if (temp <= 0.0) return 0;
  double s = 0.5 * sqrt(temp);
  *aI = -(-b / (2.0 * a) - 2.0 * s);
  *bI = (-b / (4.0 * a) - s) * (-b / (4.0 * a) - s) - 0.25 * (-4.0 * s * s - 2.0 * p + q / s);
  *gI = -(-b / (2.0 * a) + 2.0 * s);
  *dI = (-b / (4.0 * a) + s) * (-b / (4.0 * a) + s) - 0.25 * (-4.0 * s * s - 2.0 * p - q / s);
  return 1;
}

/* EllipticParticle::fastQuarticSolver (Strobach 2010), EllipticParticle.cpp:559-609 */
static double fast_quartic(double a, double b, double c, double d, double aI, double bI,
                           double gI, double dI, double* alpha_, double* beta_, double* gamma_,
                           double* delta_) {
  double alpha = aI, beta = bI, gamma = gI, delta = dI;
  double e1 = a - alpha - gamma;
  double e2 = b - beta - alpha * gamma - delta;
  double e3 = c - beta * gamma - alpha * delta;
  double e4 = d - beta * delta;
  double e_old = fabs(e1) + fabs(e2) + fabs(e3) + fabs(e4);
  double e_new = 1.0;
  int counter = 0;
  double u23, u33, L43, u44, x1, x2, x3, x4, y1, y2, y3, y4;
  while (fabs((e_old - e_new) / e_old) >= 1e-3) {
    e_old = e_new;
    counter++;
    if (counter > 20) break;
    u23 = alpha - gamma;
    u33 = beta - delta - gamma * u23;
    L43 = -delta * u23 / u33;
    u44 = beta - delta - L43 * u23;
    x1 = e1;
    x2 = e2 - gamma * x1;
    x3 = e3 - delta * x1 - gamma * x2;
    x4 = e4 - delta * x2 - L43 * x3;
    y4 = x4 / u44;
    y3 = (x3 - u23 * y4) / u33;
    y2 = x2 - u23 * y3 - y4;
    y1 = x1 - y3;
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
  *alpha_ = alpha;
  *beta_ = beta;
  *gamma_ = gamma;
  *delta_ = delta;
  return e_new;
}

/* boundary distance along the line of slope k through cp, for one ellipse
   (EllipticParticle.cpp:417-431 and :433-447) */
static double chord_half(double cz, double sz, double ax, double bx, double xc, double yc,
                         v2 cp, double k) {
  double aa = pow(cz / ax, 2) + pow(sz / bx, 2);
  double bb = pow(sz / ax, 2) + pow(cz / bx, 2);
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
  double d1 = pow(xo1 - cp.x, 2) + pow(yo1 - cp.y, 2);
  double d2 = pow(xo2 - cp.x, 2) + pow(yo2 - cp.y, 2);
  return (d1 > d2) ? sqrt(d2) : sqrt(d1);
}

/* EllipticParticle::contactWithEllipticParticle0, intersection (Strobach),
   EllipticParticle.cpp:288-484 */
static int ellipse_intersection(const pstate_t* A_, const pstate_t* B_, v2 off, v2 ovel,
                                geom_t* g) {
  double ai = A_->r, aj = B_->r;
  double bi = ai / A_->asp, bj = aj / B_->asp;
  double xi = A_->x, xj = B_->x + off.x;
  double yi = A_->y, yj = B_->y + off.y;
  double zi = A_->rot, zj = B_->rot;
  double szi = sin(zi), czi = cos(zi);
  double szj = sin(zj), czj = cos(zj);
  double z0 = zj - zi;
  double x0 = (xj - xi) * czi + (yj - yi) * szi;
  double y0 = -(xj - xi) * szi + (yj - yi) * czi;
  double c0 = pow(cos(z0) / aj, 2) + pow(sin(z0) / bj, 2);
  double c1 = pow(sin(z0) / aj, 2) + pow(cos(z0) / bj, 2);
  double c2 = sin(2.0 * z0) / aj / aj - sin(2.0 * z0) / bj / bj;
  double c3 = -2.0 * x0 * c0 - y0 * c2;
  double c4 = -2.0 * y0 * c1 - x0 * c2;
  double c5 = x0 * x0 * c0 + y0 * y0 * c1 + x0 * y0 * c2 - 1.0;
  double kk = bi * bi / (ai * ai);
  double p0 = kk * c2 * c2 + pow(c0 - c1 * kk, 2);
  double p1 = 2.0 * kk * c2 * c4 + 2.0 * (c0 - c1 * kk) * c3;
  double p2 = -kk * c2 * c2 * ai * ai + kk * c4 * c4 + 2.0 * (c0 - c1 * kk) * (c5 + c1 * kk * ai * ai) +
              c3 * c3;
  double p3 = 2.0 * c3 * (c5 + c1 * kk * ai * ai) - 2.0 * kk * c2 * c4 * ai * ai;
  double p4 = pow((c5 + c1 * kk * ai * ai), 2) - kk * c4 * c4 * ai * ai;
  double aI, bI, gI, dI;
  g->iters = 0;
  if (!solve_quartic_general(p0, p1, p2, p3, p4, &aI, &bI, &gI, &dI)) {
    g->contacted = 0;
    return 0;
  }
  p1 /= p0;
  p2 /= p0;
  p3 /= p0;
  p4 /= p0;
  p0 /= p0;
  double alpha, beta, gamma, delta;
  fast_quartic(p1, p2, p3, p4, aI, bI, gI, dI, &alpha, &beta, &gamma, &delta);
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
  for (int i = 0; i < 2; i++) {
    yr[i] = bi * sqrt(1.0 - pow(xr[i] / ai, 2));
    double err1 = c0 * xr[i] * xr[i] + c1 * yr[i] * yr[i] + c2 * xr[i] * yr[i] + c3 * xr[i] +
                  c4 * yr[i] + c5;
    double err2 = c0 * xr[i] * xr[i] + c1 * yr[i] * yr[i] - c2 * xr[i] * yr[i] + c3 * xr[i] -
                  c4 * yr[i] + c5;
    yr[i] = (fabs(err1) <= fabs(err2)) ? yr[i] : -yr[i];
    if (dmin(fabs(err1), fabs(err2)) > 1e-8) { g->contacted = 0; return 0; }
    if (!isfinite(yr[i])) { g->contacted = 0; return 0; }
    if (fabs(yr[i]) > bi) { g->contacted = 0; return 0; }
  }
  v2 cp1 = V(xr[0] * czi - yr[0] * szi + xi, xr[0] * szi + yr[0] * czi + yi);
  v2 cp2 = V(xr[1] * czi - yr[1] * szi + xi, xr[1] * szi + yr[1] * czi + yi);
  g->cp = vdiv(vadd(cp1, cp2), 2.0);
  if (!isfinite(vlen(g->cp))) { g->contacted = 0; return 0; }
  v2 tangent = vsub(cp1, cp2);
  if (vlen(tangent) == 0.0) { g->contacted = 0; return 0; }
  uint32_t dummy = 0;
  tangent = vnormalize(tangent, &dummy);
  g->n = V(tangent.y, -tangent.x);
  if (!isfinite(vlen(g->n))) { g->contacted = 0; return 0; }
  v2 bv = vsub(g->cp, V(xi, yi));
  if (vdot(g->n, bv) < 0.0) g->n = vneg(g->n);
  double k = g->n.y / g->n.x;
  if (fabs(k) > 100000) k = copysign(100000, k);
  if (!isfinite(k)) k = (g->n.y > 0) ? 100000 : -100000;
  double disti = chord_half(czi, szi, ai, bi, xi, yi, g->cp, k);
  double distj = chord_half(czj, szj, aj, bj, xj, yj, g->cp, k);
  g->overlap = disti + distj;
  if (!isfinite(disti)) g->overlap = 2.0 * distj;
  if (!isfinite(distj)) g->overlap = 2.0 * disti;
  g->contacted = 1;
  g->bv1 = vsub(g->cp, V(A_->x, A_->y));
  g->bv2 = vsub(g->cp, V(xj, yj));
  relative_velocity(A_, B_, ovel, g);
  if (!isfinite(g->overlap)) { g->contacted = 0; return 0; }
  return 1;
}
/* SegmentObject::_dirVector = (v2 - v1).getUnitVector() (SegmentObject.h:37,
   MathVector.h:169-178) */
static v2 seg_dir(const pstate_t* s) { return vunit(vsub(s->s2, s->s1)); }

/* the point of the segment nearest to q along its direction: a vertex beyond
   either end, else the projection (SegmentObject.cpp:51-62,
   CircularParticle.cpp:99-108) */
static v2 seg_ref(const pstate_t* s, v2 dir, double proj) {
  if (proj > s->r) return s->s2;
  if (proj < -s->r) return s->s1;
  return vadd(V(s->x, s->y), vmul(dir, proj));
}

/* CircularParticle::contactWithSegmentObject (CircularParticle.cpp:94-129):
   the circle is P1.  The reference adds the offset to the circle's own
   position when projecting and again to the reference point (the segment's
   image would take the offset once); restated as written. */
static int circle_segment(const pstate_t* a, const pstate_t* b, v2 off, v2 ovel, geom_t* g) {
  v2 dir = seg_dir(b);
  double proj = vdot(vsub(vadd(V(a->x, a->y), off), V(b->x, b->y)), dir);
  v2 ref = seg_ref(b, dir, proj);
  v2 branch = vsub(vadd(ref, off), V(a->x, a->y));
  double distance = vlen(branch);
  double sumR = a->r;
  g->overlap = sumR - distance;
  if (g->overlap < 0.0) { g->contacted = 0; return 0; }
  g->contacted = 1;
  g->n = vunit(branch);
  g->cp = ref;
  g->bv1 = vsub(g->cp, V(a->x, a->y));
  g->bv2 = vsub(g->cp, vadd(ref, off));
  relative_velocity(a, b, ovel, g);
  return 1;
}

/* SegmentObject::contactWithCircularParticle (SegmentObject.cpp:45-80): the
   segment is P1; its branch vector to the contact point is zero. */
static int segment_circle(const pstate_t* a, const pstate_t* b, v2 off, v2 ovel, geom_t* g) {
  v2 dir = seg_dir(a);
  v2 pb = vadd(V(b->x, b->y), off);
  double proj = vdot(vsub(pb, V(a->x, a->y)), dir);
  v2 ref = seg_ref(a, dir, proj);
  v2 branch = vsub(pb, ref);
  double distance = vlen(branch);
  double sumR = b->r;
  g->overlap = sumR - distance;
  if (g->overlap < 0.0) { g->contacted = 0; return 0; }
  g->contacted = 1;
  g->n = vunit(branch);
  g->cp = ref;
  g->bv1 = vsub(g->cp, ref);
  g->bv2 = vsub(g->cp, pb);
  relative_velocity(a, b, ovel, g);
  return 1;
}

/* BaseParticle::calculateContactGeometry dispatch (CircularParticle.cpp:25-40,
   EllipticParticle.cpp:16-32, GluedParticle.cpp:133-140,
   SegmentObject.cpp:12-27) */
static int contact_geometry(int method, const pstate_t* a, const pstate_t* b, double orad_a,
                            double orad_b, v2 off, v2 ovel, geom_t* g, uint32_t* st) {
  memset(g, 0, sizeof(*g));
  if (a->shape == XDEM_SHAPE_CLUMP || b->shape == XDEM_SHAPE_CLUMP) return 0;
  if (a->shape == XDEM_SHAPE_SEGMENT) {
    if (b->shape == XDEM_SHAPE_SEGMENT) return 0;
    if (b->shape != XDEM_SHAPE_CIRCLE) { *st |= XDEM_ERR_UNSUPPORTED_PAIR; return 0; }
    return segment_circle(a, b, off, ovel, g);
  }
  if (a->shape == XDEM_SHAPE_CIRCLE) {
    if (b->shape == XDEM_SHAPE_SEGMENT) return circle_segment(a, b, off, ovel, g);
    if (b->shape != XDEM_SHAPE_CIRCLE) { *st |= XDEM_ERR_UNSUPPORTED_PAIR; return 0; }
    return circle_circle(a, b, off, ovel, g);
  }
  if (b->shape != XDEM_SHAPE_ELLIPSE) { *st |= XDEM_ERR_UNSUPPORTED_PAIR; return 0; }
  /* takeCoarseDetection with offset (BaseParticle.h:131-132) */
  v2 dd = vsub(V(a->x, a->y), vadd(V(b->x, b->y), off));
  if (!((orad_a + orad_b) > sqrt(vlen2(dd)))) { g->contacted = 0; return 0; }
  if (method == XDEM_ELLIPSE_INTERSECTION) return ellipse_intersection(a, b, off, ovel, g);
  return ellipse_closest(a, b, off, ovel, g, st);
}

int32_t xo_pair_geometry(int32_t npairs, int32_t method, const double* pi, const double* pj,
                         const double* off, double* out) {
  uint32_t st = 0;
  for (int k = 0; k < npairs; ++k) {
    const double* a = pi + 9 * k;
    const double* b = pj + 9 * k;
    pstate_t A = {(int)a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], {0, 0}, {0, 0}};
    pstate_t B = {(int)b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8], {0, 0}, {0, 0}};
    geom_t g;
    int c = contact_geometry(method, &A, &B, a[1], b[1], V(off[4 * k], off[4 * k + 1]),
                             V(off[4 * k + 2], off[4 * k + 3]), &g, &st);
    double* o = out + 17 * k;
    o[0] = c ? 1.0 : 0.0;
    o[1] = g.n.x; o[2] = g.n.y; o[3] = g.cp.x; o[4] = g.cp.y;
    o[5] = g.bv1.x; o[6] = g.bv1.y; o[7] = g.bv2.x; o[8] = g.bv2.y;
    o[9] = g.overlap;
    o[10] = g.rv.x; o[11] = g.rv.y; o[12] = g.nrv.x; o[13] = g.nrv.y;
    o[14] = g.srv.x; o[15] = g.srv.y;
    o[16] = (double)g.iters;
  }
  return (int32_t)st;
}

int32_t xo_closest_quartic(int32_t npairs, const double* pi, const double* pj, const double* off,
                           double* out) {
  uint32_t st = 0;
  for (int k = 0; k < npairs; ++k) {
    const double* a = pi + 9 * k;
    const double* b = pj + 9 * k;
    pstate_t A = {(int)a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], {0, 0}, {0, 0}};
    pstate_t B = {(int)b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8], {0, 0}, {0, 0}};
    geom_t g;
    int c = contact_geometry(XDEM_ELLIPSE_CLOSEST_APPROACH, &A, &B, a[1], b[1],
                             V(off[4 * k], off[4 * k + 1]), V(off[4 * k + 2], off[4 * k + 3]),
                             &g, &st);
    double* o = out + 10 * k;
    for (int i = 0; i < 5; ++i) o[i] = g.quartic[i];
    o[5] = g.q_start;
    o[6] = g.q;
    o[7] = (double)g.iters;
    o[8] = (double)g.stuck;
    o[9] = c ? 1.0 : 0.0;
  }
  return (int32_t)st;
}

/* ------------------------------------------------------------------------- */
/* World state                                                                */
/* ------------------------------------------------------------------------- */
typedef struct {
  int j;
  v2 n, cp, b, bv1, bv2, s, fn, ft, f;
  double t1, t2, damp;
} contact_t;

enum { CAND_REGULAR = 0, CAND_TOP = 1, CAND_BOTTOM = 2 };

struct xo_world {
  xdem_params prm;
  int threads;
  int n;
  int *shape, *up, *setting, *rattler, *num_sub;
  double *orad, *rad, *asp, *x, *y, *vx, *vy, *rot, *w, *vol, *m, *im, *I, *iI, *bx, *by;
  double *s1x, *s1y, *s2x, *s2y; /* segment vertices (zero for other shapes) */
  /* contacts: CSR by owner, partners ascending */
  int64_t *cstart;
  contact_t* con;
  int64_t ncon;
  /* per-particle sums (BaseWorld::_totalForce/_totalTorque/_numContactPerParticle) */
  double *fx, *fy, *tq;
  int* ncp;
  /* candidates (findPossibleContacts) */
  int* cand_n;
  int* cand;
  unsigned char* cand_kind;
  /* world scalars */
  double xmin, xmax, ymin, ymax, xlen, ylen, maxsize, total_volume;
  double shift, shift_vel, strain, shift_rate;
  double velX, velY, vmass, max_strain_rate;
  double stress[4];
  double kn, kt, e, mu, factor, g, dt;
  uint32_t status;
};

static void recalc_factor(xo_world* w) {
  /* ContactModel_LinearDissipativeFrictioanl ctor / recalculateFactor
     (ContactModel_LinearDissipativeFrictional.h:18-23, .cpp:66-71) */
  double lg = log(w->e);
  w->factor = 2.0 * sqrt(w->kn) * fabs(lg) / sqrt(M_PI * M_PI + lg * lg);
}

xo_world* xo_create(const xdem_params* prm, int32_t threads) {
  xo_world* w = (xo_world*)calloc(1, sizeof(xo_world));
  w->prm = *prm;
  w->threads = threads > 0 ? threads : 1;
  w->xmin = prm->xmin; w->xmax = prm->xmax; w->ymin = prm->ymin; w->ymax = prm->ymax;
  w->xlen = w->xmax - w->xmin;
  w->ylen = w->ymax - w->ymin;
  w->kn = prm->normal_stiffness; w->kt = prm->shear_stiffness;
  w->e = prm->restitution_coeff; w->mu = prm->frictional_coeff;
  w->g = prm->global_damping; w->dt = prm->dt;
  recalc_factor(w);
  w->shift_rate = prm->shift_strain_rate;
  w->shift_vel = w->shift_rate * w->ylen;
  return w;
}

static void free_particles(xo_world* w) {
  void* ps[] = {w->shape, w->up, w->setting, w->rattler, w->num_sub, w->orad, w->rad, w->asp,
                w->x, w->y, w->vx, w->vy, w->rot, w->w, w->vol, w->m, w->im, w->I, w->iI,
                w->bx, w->by, w->cstart, w->con, w->fx, w->fy, w->tq, w->ncp, w->cand_n,
                w->cand, w->cand_kind, w->s1x, w->s1y, w->s2x, w->s2y};
  for (size_t k = 0; k < sizeof(ps) / sizeof(ps[0]); ++k) free(ps[k]);
}

void xo_destroy(xo_world* w) {
  if (!w) return;
  free_particles(w);
  free(w);
}

uint32_t xo_status(xo_world* w) {
  uint32_t s = w->status;
  w->status = 0;
  return s;
}

#define ALLOC(p, cnt) (p) = calloc((size_t)(cnt) > 0 ? (size_t)(cnt) : 1, sizeof(*(p)))

int32_t xo_set_particles(xo_world* w, const xdem_particles* P) {
  free_particles(w);
  int n = P->n;
  w->n = n;
  ALLOC(w->shape, n); ALLOC(w->up, n); ALLOC(w->setting, n); ALLOC(w->rattler, n);
  ALLOC(w->num_sub, n); ALLOC(w->orad, n); ALLOC(w->rad, n); ALLOC(w->asp, n);
  ALLOC(w->x, n); ALLOC(w->y, n); ALLOC(w->vx, n); ALLOC(w->vy, n); ALLOC(w->rot, n);
  ALLOC(w->w, n); ALLOC(w->vol, n); ALLOC(w->m, n); ALLOC(w->im, n); ALLOC(w->I, n);
  ALLOC(w->iI, n); ALLOC(w->bx, n); ALLOC(w->by, n);
  ALLOC(w->s1x, n); ALLOC(w->s1y, n); ALLOC(w->s2x, n); ALLOC(w->s2y, n);
  ALLOC(w->cstart, n + 1); ALLOC(w->con, 1); w->ncon = 0;
  ALLOC(w->fx, n); ALLOC(w->fy, n); ALLOC(w->tq, n); ALLOC(w->ncp, n);
  ALLOC(w->cand_n, n); ALLOC(w->cand, (size_t)n * XO_CANDIDATE_CAP * 3);
  ALLOC(w->cand_kind, (size_t)n * XO_CANDIDATE_CAP * 3);
  double maxr = 0.0, vol = 0.0;
  for (int i = 0; i < n; ++i) {
    w->shape[i] = P->shape[i]; w->up[i] = P->up_level[i]; w->setting[i] = P->setting[i];
    w->rattler[i] = P->is_rattler ? P->is_rattler[i] : 0;
    w->num_sub[i] = P->num_sub ? P->num_sub[i] : 0;
    w->orad[i] = P->outer_radius[i]; w->rad[i] = P->radius[i]; w->asp[i] = P->aspect_ratio[i];
    w->x[i] = P->x[i]; w->y[i] = P->y[i]; w->vx[i] = P->vx[i]; w->vy[i] = P->vy[i];
    w->rot[i] = P->rot[i]; w->w[i] = P->rot_vel[i];
    w->vol[i] = P->volume[i]; w->m[i] = P->mass[i]; w->im[i] = P->inv_mass[i];
    w->I[i] = P->inertia[i]; w->iI[i] = P->inv_inertia[i];
    w->bx[i] = P->branch_x ? P->branch_x[i] : 0.0;
    w->by[i] = P->branch_y ? P->branch_y[i] : 0.0;
    if (w->shape[i] == XDEM_SHAPE_SEGMENT) {
      if (!P->seg_x1 || !P->seg_y1 || !P->seg_x2 || !P->seg_y2) return XDEM_ERR_ARGUMENT;
      w->s1x[i] = P->seg_x1[i]; w->s1y[i] = P->seg_y1[i];
      w->s2x[i] = P->seg_x2[i]; w->s2y[i] = P->seg_y2[i];
    }
    /* updateMaximumParticleSize (BaseWorld.cpp:201-219) */
    if (w->orad[i] > maxr) maxr = w->orad[i];
    /* updateTotalParticleVolume (BaseWorld.cpp:188-199) */
    if (!(w->setting[i] & XDEM_SKIP_MACRO_SUM)) vol += w->vol[i];
  }
  w->maxsize = w->prm.max_particle_size > 0 ? w->prm.max_particle_size : maxr * 2.01;
  w->total_volume = vol;
  return XDEM_OK;
}

int32_t xo_get_particles(xo_world* w, xdem_particles* P) {
  P->n = w->n;
  for (int i = 0; i < w->n; ++i) {
    if (P->x) P->x[i] = w->x[i];
    if (P->y) P->y[i] = w->y[i];
    if (P->vx) P->vx[i] = w->vx[i];
    if (P->vy) P->vy[i] = w->vy[i];
    if (P->rot) P->rot[i] = w->rot[i];
    if (P->rot_vel) P->rot_vel[i] = w->w[i];
    if (P->is_rattler) P->is_rattler[i] = w->rattler[i];
    if (P->mass) P->mass[i] = w->m[i];
    if (P->inertia) P->inertia[i] = w->I[i];
    if (P->branch_x) P->branch_x[i] = w->bx[i];
    if (P->branch_y) P->branch_y[i] = w->by[i];
    if (P->seg_x1) P->seg_x1[i] = w->s1x[i];
    if (P->seg_y1) P->seg_y1[i] = w->s1y[i];
    if (P->seg_x2) P->seg_x2[i] = w->s2x[i];
    if (P->seg_y2) P->seg_y2[i] = w->s2y[i];
  }
  return XDEM_OK;
}

static int cmp_key(const void* a, const void* b) {
  const int64_t* x = (const int64_t*)a;
  const int64_t* y = (const int64_t*)b;
  return (x[0] > y[0]) - (x[0] < y[0]);
}

int32_t xo_set_contacts(xo_world* w, const xdem_contacts* C) {
  int64_t nc = C->count;
  int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * 2 * (nc > 0 ? nc : 1));
  for (int64_t k = 0; k < nc; ++k) {
    keys[2 * k] = ((int64_t)C->id_i[k] << 32) | (uint32_t)C->id_j[k];
    keys[2 * k + 1] = k;
  }
  qsort(keys, (size_t)nc, 2 * sizeof(int64_t), cmp_key);
  free(w->con);
  w->con = (contact_t*)calloc((size_t)(nc > 0 ? nc : 1), sizeof(contact_t));
  memset(w->cstart, 0, sizeof(int64_t) * (w->n + 1));
  for (int64_t q = 0; q < nc; ++q) {
    int64_t k = keys[2 * q + 1];
    contact_t* c = &w->con[q];
    c->j = C->id_j[k];
    c->n = V(C->normal_x[k], C->normal_y[k]);
    c->cp = V(C->point_x[k], C->point_y[k]);
    c->b = V(C->branch_x[k], C->branch_y[k]);
    c->bv1 = V(C->bv1_x[k], C->bv1_y[k]);
    c->bv2 = V(C->bv2_x[k], C->bv2_y[k]);
    c->s = V(C->shear_x[k], C->shear_y[k]);
    c->fn = V(C->fn_x[k], C->fn_y[k]);
    c->ft = V(C->ft_x[k], C->ft_y[k]);
    c->f = vadd(c->fn, c->ft);
    c->t1 = C->torque_i[k];
    c->t2 = C->torque_j[k];
    c->damp = C->damping[k];
    w->cstart[C->id_i[k] + 1]++;
  }
  for (int i = 0; i < w->n; ++i) w->cstart[i + 1] += w->cstart[i];
  w->ncon = nc;
  free(keys);
  return XDEM_OK;
}

int32_t xo_get_contacts(xo_world* w, xdem_contacts* C) {
  C->count = w->ncon;
  if (C->capacity < w->ncon) return XDEM_ERR_CAPACITY;
  for (int i = 0; i < w->n; ++i) {
    for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k) {
      contact_t* c = &w->con[k];
      C->id_i[k] = i; C->id_j[k] = c->j;
      C->normal_x[k] = c->n.x; C->normal_y[k] = c->n.y;
      C->point_x[k] = c->cp.x; C->point_y[k] = c->cp.y;
      C->branch_x[k] = c->b.x; C->branch_y[k] = c->b.y;
      C->bv1_x[k] = c->bv1.x; C->bv1_y[k] = c->bv1.y;
      C->bv2_x[k] = c->bv2.x; C->bv2_y[k] = c->bv2.y;
      C->shear_x[k] = c->s.x; C->shear_y[k] = c->s.y;
      C->fn_x[k] = c->fn.x; C->fn_y[k] = c->fn.y;
      C->ft_x[k] = c->ft.x; C->ft_y[k] = c->ft.y;
      C->torque_i[k] = c->t1; C->torque_j[k] = c->t2;
      C->damping[k] = c->damp;
    }
  }
  return XDEM_OK;
}

int32_t xo_get_force_and_torque(xo_world* w, double* fx, double* fy, double* t, int32_t* nc) {
  for (int i = 0; i < w->n; ++i) {
    fx[i] = w->fx[i]; fy[i] = w->fy[i]; t[i] = w->tq[i];
    if (nc) nc[i] = w->ncp[i];
  }
  return XDEM_OK;
}

void xo_get_boundary(xo_world* w, double* box) {
  box[0] = w->xmin; box[1] = w->xmax; box[2] = w->ymin; box[3] = w->ymax;
}
void xo_get_stress(xo_world* w, double* s) { memcpy(s, w->stress, sizeof(w->stress)); }
void xo_get_lees_edwards(xo_world* w, double* out) {
  out[0] = w->shift; out[1] = w->shift_vel; out[2] = w->strain; out[3] = w->shift_rate;
}
void xo_set_lees_edwards(xo_world* w, const double* in) {
  w->shift = in[0]; w->shift_vel = in[1]; w->strain = in[2]; w->shift_rate = in[3];
}
/* PeriodicControlWorld::setVirtualBoundaryMass (PeriodicControlWorld.cpp:58-71) */
void xo_set_virtual_boundary_mass(xo_world* w, double mass) {
  if (mass >= 0) { w->vmass = mass; return; }
  double m = 0.0;
  for (int i = 0; i < w->n; ++i) {
    if (w->setting[i] & XDEM_SKIP_MACRO_SUM) continue;
    m += w->m[i];
  }
  w->vmass = m / ((double)w->n * 10.0);
}
void xo_set_max_strain_rate(xo_world* w, double r) { w->max_strain_rate = r; }

/* BaseWorld::getKineticEnergy (BaseWorld.cpp:302-310), sequential sum */
double xo_kinetic_energy(xo_world* w) {
  double ke = 0.0;
  for (int i = 0; i < w->n; ++i)
    ke += 0.5 * (w->m[i] * vlen2(V(w->vx[i], w->vy[i])) + w->I[i] * w->w[i] * w->w[i]);
  return ke;
}

int64_t xo_count_contacts(xo_world* w) { return w->ncon; }

/* ------------------------------------------------------------------------- */
/* Sub-steps                                                                  */
/* ------------------------------------------------------------------------- */

/* PeriodicBoundaryWorld::modifyParticlePosition (PeriodicBoundaryWorld.cpp:129-142)
   and LeesEdwardsBoundaryWorld::modifyParticlePosition (:304-333) */
static void modify_particle_position(xo_world* w) {
  int le = w->prm.world_kind == XDEM_WORLD_LEES_EDWARDS;
  for (int i = 0; i < w->n; ++i) {
    if (le) {
      if (w->y[i] < w->ymin) {
        w->y[i] += w->ylen;
        w->x[i] += w->shift;
      } else if (w->y[i] > w->ymax) {
        w->y[i] += -w->ylen;
        w->x[i] += -w->shift;
      }
      if (w->x[i] < w->xmin) w->x[i] += w->xlen;
      else if (w->x[i] > w->xmax) w->x[i] += -w->xlen;
    } else {
      if (w->x[i] < w->xmin) w->x[i] += w->xlen;
      else if (w->x[i] > w->xmax) w->x[i] += -w->xlen;
      if (w->y[i] < w->ymin) w->y[i] += w->ylen;
      else if (w->y[i] > w->ymax) w->y[i] += -w->ylen;
    }
  }
}

/* LeesEdwardsBoundaryWorld::apply/removeBackgroudVelocity (:508-530) */
static void background_velocity(xo_world* w, int apply) {
  for (int i = 0; i < w->n; ++i) {
    if (apply) w->vx[i] = w->vx[i] + w->shift_rate * w->y[i];
    else w->vx[i] = w->vx[i] - w->shift_rate * w->y[i];
  }
}

/* cell index of a coordinate; a coordinate at the upper edge would give
   numGrid in the reference (out of range), clamped here */
static inline int cell_of(double v, double vmin, double len, int ng) {
  int c = (int)floor((v - vmin) / len);
  if (c < 0) c = 0;
  if (c > ng - 1) c = ng - 1;
  return c;
}

/* findPossibleContacts: PeriodicBoundaryWorld.cpp:12-85 and
   LeesEdwardsBoundaryWorld.cpp:34-205 (cell lists, 3x3 scan, id/upLevel
   filters, 200-candidate cap) */
static void find_possible_contacts(xo_world* w) {
  int le = w->prm.world_kind == XDEM_WORLD_LEES_EDWARDS;
  w->xlen = w->xmax - w->xmin;
  w->ylen = w->ymax - w->ymin;
  int nx = (int)floor(w->xlen / w->maxsize);
  int ny = (int)floor(w->ylen / w->maxsize);
  if (nx < 3 || ny < 3) {
    w->status |= XDEM_ERR_GRID;
    memset(w->cand_n, 0, sizeof(int) * (size_t)w->n);
    return;
  }
  int ncell = nx * ny;
  double lx = w->xlen / nx, ly = w->ylen / ny;
  int n = w->n;
  int* pc = (int*)malloc(sizeof(int) * 2 * n);
  int* lec = (int*)malloc(sizeof(int) * n); /* LE column (row 0: top list, row ny-1: bottom list) */
  int* cnt = (int*)calloc((size_t)ncell + 2 * nx + 1, sizeof(int));
  for (int i = 0; i < n; ++i) {
    int ix = cell_of(w->x[i], w->xmin, lx, nx);
    int iy = cell_of(w->y[i], w->ymin, ly, ny);
    pc[2 * i] = ix;
    pc[2 * i + 1] = iy;
    lec[i] = -1;
    if (le && iy == 0) {
      double t = w->x[i] + w->shift;
      if (t < w->xmin) t += w->xlen;
      else if (t > w->xmax) t -= w->xlen;
      lec[i] = cell_of(t, w->xmin, lx, nx);
    } else if (le && iy == ny - 1) {
      double t = w->x[i] - w->shift;
      if (t < w->xmin) t += w->xlen;
      else if (t > w->xmax) t -= w->xlen;
      lec[i] = cell_of(t, w->xmin, lx, nx);
    }
  }
  /* bins: regular cells, then boxLE_top (nx), then boxLE_bottom (nx); members
     in ascending particle id as the reference's single-thread fill */
  int nb = ncell + 2 * nx;
  int* start = (int*)calloc((size_t)nb + 1, sizeof(int));
  for (int i = 0; i < n; ++i) {
    start[pc[2 * i + 1] * nx + pc[2 * i] + 1]++;
    if (lec[i] >= 0) {
      int b = (pc[2 * i + 1] == 0) ? ncell + lec[i] : ncell + nx + lec[i];
      start[b + 1]++;
    }
  }
  for (int b = 0; b < nb; ++b) start[b + 1] += start[b];
  int* mem = (int*)malloc(sizeof(int) * (size_t)(start[nb] > 0 ? start[nb] : 1));
  memcpy(cnt, start, sizeof(int) * nb);
  for (int i = 0; i < n; ++i) {
    mem[cnt[pc[2 * i + 1] * nx + pc[2 * i]]++] = i;
    if (lec[i] >= 0) {
      int b = (pc[2 * i + 1] == 0) ? ncell + lec[i] : ncell + nx + lec[i];
      mem[cnt[b]++] = i;
    }
  }
  for (int i = 0; i < n; ++i) {
    int nreg = 0, ntop = 0, nbot = 0;
    int* list = w->cand + (size_t)i * XO_CANDIDATE_CAP * 3;
    unsigned char* kind = w->cand_kind + (size_t)i * XO_CANDIDATE_CAP * 3;
    int total = 0;
    w->cand_n[i] = 0;
    if (w->setting[i] & XDEM_SKIP_CONTACT_DETECTION) continue;
    int ix = pc[2 * i], iy = pc[2 * i + 1];
    for (int dx = -1; dx <= 1; ++dx) {
      int jx = ix + dx;
      if (jx == -1) jx = nx - 1;
      else if (jx == nx) jx = 0;
      for (int dy = -1; dy <= 1; ++dy) {
        int jy = iy + dy;
        int b, k = CAND_REGULAR;
        if (le && (jy == -1 || jy == ny)) {
          if (jy == -1) { b = ncell + nx + jx; k = CAND_BOTTOM; }
          else { b = ncell + jx; k = CAND_TOP; }
        } else {
          if (jy == -1) jy = ny - 1;
          else if (jy == ny) jy = 0;
          b = jy * nx + jx;
        }
        for (int q = start[b]; q < start[b + 1]; ++q) {
          int j = mem[q];
          if (w->setting[j] & XDEM_SKIP_CONTACT_DETECTION) continue;
          if (i >= j) continue;
          if (w->up[i] == w->up[j]) continue;
          if (k == CAND_REGULAR) {
            if (nreg + 1 >= XO_CANDIDATE_CAP) { w->status |= XDEM_ERR_CAPACITY; continue; }
            nreg++;
          } else if (k == CAND_TOP) {
            if (ntop + 1 >= XO_CANDIDATE_CAP) { w->status |= XDEM_ERR_CAPACITY; continue; }
            ntop++;
          } else {
            if (nbot + 1 >= XO_CANDIDATE_CAP) { w->status |= XDEM_ERR_CAPACITY; continue; }
            nbot++;
          }
          list[total] = j;
          kind[total] = (unsigned char)k;
          total++;
        }
      }
    }
    w->cand_n[i] = total;
  }
  free(pc); free(lec); free(cnt); free(start); free(mem);
}

/* per-candidate offset: PeriodicBoundaryWorld.cpp:97-101 (minimum image) and
   LeesEdwardsBoundaryWorld.cpp:233-279 (sheared images) */
static void candidate_offset(const xo_world* w, int i, int j, int kind, v2* off, v2* ovel) {
  *ovel = V(0.0, 0.0);
  if (kind == CAND_REGULAR) {
    double ox = 0.0, oy = 0.0;
    if (w->x[j] - w->x[i] > w->xlen / 2.0) ox = -w->xlen;
    else if (w->x[j] - w->x[i] < -w->xlen / 2.0) ox = w->xlen;
    if (w->y[j] - w->y[i] > w->ylen / 2.0) oy = -w->ylen;
    else if (w->y[j] - w->y[i] < -w->ylen / 2.0) oy = w->ylen;
    *off = V(ox, oy);
    return;
  }
  double sgn = (kind == CAND_TOP) ? 1.0 : -1.0;
  v2 o = (kind == CAND_TOP) ? V(w->shift, w->ylen) : V(-w->shift, -w->ylen);
  double t = o.x + w->x[j];
  if (t < w->xmin) { o.x += w->xlen; t += w->xlen; }
  else if (t > w->xmax) { o.x += -w->xlen; t -= w->xlen; }
  if (t - w->x[i] > w->xlen / 2.0) o.x += -w->xlen;
  else if (t - w->x[i] < -w->xlen / 2.0) o.x += w->xlen;
  *off = o;
  *ovel = V(sgn * w->shift_vel, 0.0);
}

static inline pstate_t pstate(const xo_world* w, int i) {
  pstate_t p = {w->shape[i], w->rad[i], w->asp[i], w->x[i], w->y[i],
                w->vx[i], w->vy[i], w->rot[i], w->w[i],
                {w->s1x[i], w->s1y[i]}, {w->s2x[i], w->s2y[i]}};
  return p;
}

/* ContactModel_LinearDissipativeFrictioanl::calculateDampingConstact
   (ContactModel_LinearDissipativeFrictional.cpp:73-82) with the flag
   selection of BaseParticle.cpp:53-64 */
static double damping_constant(const xo_world* w, int i, int j) {
  int si = w->setting[i] & XDEM_SKIP_TIME_INTEGRAL, sj = w->setting[j] & XDEM_SKIP_TIME_INTEGRAL;
  double mi = w->m[i], mj = w->m[j];
  if (!si && sj) return sqrt(mi) * w->factor;
  if (si && !sj) return sqrt(mj) * w->factor;
  return sqrt((mi * mj) / (mi + mj)) * w->factor;
}

/* BaseParticle::calculateContactForceAndTorque (BaseParticle.cpp:27-98) with
   ContactModel_LinearDissipativeFrictioanl::calculateNormalForce/ShearForce
   (ContactModel_LinearDissipativeFrictional.cpp:3-46) and
   ContactInformation::calculateTotalForceAndTorque (ContactInformation.h:62-68).
   old == NULL: a new contact. */
static void contact_force(const xo_world* w, int i, int j, v2 off, const geom_t* g,
                          const contact_t* old, contact_t* c) {
  double dt = w->dt;
  c->j = j;
  if (!old) {
    c->n = g->n; c->cp = g->cp; c->bv1 = g->bv1; c->bv2 = g->bv2;
    c->s = V(0.0, 0.0);
    double rvn = vdot(g->rv, g->n);
    if (!isnormal(rvn)) c->s = vmul(g->srv, dt);
    else c->s = vmul(g->srv, dmin(dt, g->overlap / rvn));
    c->damp = damping_constant(w, i, j);
  } else {
    *c = *old;
    double dot = vdot(c->n, g->n);
    double det = vcross(c->n, g->n);
    double angle = atan2(det, dot);
    m2 R = M(cos(angle), -sin(angle), sin(angle), cos(angle));
    c->s = mmulv(R, c->s);
    c->s = vadd(c->s, vmul(g->srv, dt));
    c->n = g->n; c->cp = g->cp; c->bv1 = g->bv1; c->bv2 = g->bv2;
  }
  c->b = vsub(V(w->x[i], w->y[i]), vadd(V(w->x[j], w->y[j]), off));
  /* normal force */
  c->fn = vadd(vmul(vmul(vneg(g->n), w->kn), g->overlap), vmul(vneg(g->nrv), c->damp));
  /* shear force */
  double maxFs = vlen(c->fn) * w->mu;
  v2 el = vmul(vneg(c->s), w->kt);
  v2 di = vmul(vneg(g->srv), c->damp);
  v2 fs = vadd(el, di);
  if (vlen(fs) > maxFs) {
    fs = vmul(vunit(fs), maxFs);
    if (vlen(el) > maxFs) c->s = vdiv(vneg(fs), w->kt);
    else c->s = vdiv(vneg(el), w->kt);
  }
  c->ft = fs;
  c->f = vadd(c->fn, c->ft);
  c->t1 = vcross(c->bv1, c->f);
  c->t2 = vcross(c->bv2, vneg(c->f));
}

static const contact_t* find_old(const xo_world* w, int i, int j) {
  int64_t lo = w->cstart[i], hi = w->cstart[i + 1] - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) / 2;
    int mj = w->con[mid].j;
    if (mj == j) return &w->con[mid];
    if (mj < j) lo = mid + 1;
    else hi = mid - 1;
  }
  return NULL;
}

static int cmp_contact(const void* a, const void* b) {
  int x = ((const contact_t*)a)->j, y = ((const contact_t*)b)->j;
  return (x > y) - (x < y);
}

/* updateContacts: PeriodicBoundaryWorld.cpp:87-107, LeesEdwardsBoundaryWorld.cpp:207-283.
   A history entry whose pair is not a candidate survives unchanged, as the
   reference's map entry does. */
static void update_contacts(xo_world* w) {
  int n = w->n;
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  off[0] = 0;
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + w->cand_n[i] + (w->cstart[i + 1] - w->cstart[i]);
  contact_t* buf = (contact_t*)malloc(sizeof(contact_t) * (size_t)(off[n] > 0 ? off[n] : 1));
  int* cnt = (int*)calloc((size_t)n, sizeof(int));
  uint32_t st_all = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(w->threads) reduction(| : st_all)
  for (int i = 0; i < n; ++i) {
    uint32_t st = 0;
    contact_t* out = buf + off[i];
    int k = 0;
    const int* list = w->cand + (size_t)i * XO_CANDIDATE_CAP * 3;
    const unsigned char* kind = w->cand_kind + (size_t)i * XO_CANDIDATE_CAP * 3;
    int nold = (int)(w->cstart[i + 1] - w->cstart[i]);
    unsigned char* seen = (unsigned char*)calloc((size_t)(nold > 0 ? nold : 1), 1);
    pstate_t a = pstate(w, i);
    for (int q = 0; q < w->cand_n[i]; ++q) {
      int j = list[q];
      v2 o, ov;
      candidate_offset(w, i, j, kind[q], &o, &ov);
      pstate_t b = pstate(w, j);
      geom_t g;
      const contact_t* old = find_old(w, i, j);
      if (old) seen[old - (w->con + w->cstart[i])] = 1;
      if (contact_geometry(w->prm.ellipse_method, &a, &b, w->orad[i], w->orad[j], o, ov, &g, &st)) {
        contact_force(w, i, j, o, &g, old, &out[k]);
        k++;
      }
    }
    for (int q = 0; q < nold; ++q)
      if (!seen[q]) out[k++] = w->con[w->cstart[i] + q];
    free(seen);
    qsort(out, (size_t)k, sizeof(contact_t), cmp_contact);
    cnt[i] = k;
    st_all |= st;
  }
  w->status |= st_all;
  int64_t total = 0;
  for (int i = 0; i < n; ++i) total += cnt[i];
  contact_t* con = (contact_t*)malloc(sizeof(contact_t) * (size_t)(total > 0 ? total : 1));
  int64_t p = 0;
  for (int i = 0; i < n; ++i) {
    w->cstart[i] = p;
    memcpy(con + p, buf + off[i], sizeof(contact_t) * cnt[i]);
    p += cnt[i];
  }
  w->cstart[n] = p;
  free(w->con);
  w->con = con;
  w->ncon = total;
  free(buf); free(off); free(cnt);
}

/* BaseWorld::collectForceAndTorque (BaseWorld.cpp:17-57) in the fixed order
   described in xdem_oracle.h */
static void collect_force_and_torque(xo_world* w) {
  int n = w->n;
  for (int i = 0; i < n; ++i) {
    w->fx[i] = 0.0; w->fy[i] = 0.0; w->tq[i] = 0.0; w->ncp[i] = 0;
    w->rattler[i] = 1;
  }
  for (int i = 0; i < n; ++i) {
    for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k) {
      const contact_t* c = &w->con[k];
      int j = c->j;
      w->fx[i] += c->f.x; w->fy[i] += c->f.y;
      w->fx[j] += -c->f.x; w->fy[j] += -c->f.y;
      w->tq[i] += c->t1;
      w->tq[j] += c->t2;
      w->ncp[i]++; w->ncp[j]++;
      w->rattler[i] = 0; w->rattler[j] = 0;
    }
  }
}

/* GluedParticle::isRattlerParticle (GluedParticle.cpp:141-147) */
static int is_rattler(const xo_world* w, int i) {
  if (w->shape[i] == XDEM_SHAPE_CLUMP) {
    for (int k = 1; k <= w->num_sub[i]; ++k)
      if (!w->rattler[i + k]) return 0;
    return 1;
  }
  return w->rattler[i];
}

/* BaseWorld::takeTimeIntegral (BaseWorld.cpp:59-77) with
   BaseParticle::takeTimeIntegral (BaseParticle.cpp:107-118) and
   GluedParticle::takeTimeIntegral (GluedParticle.cpp:91-125) */
static void take_time_integral(xo_world* w) {
  double dt = w->dt, g = w->g;
  for (int i = 0; i < w->n; ++i) {
    if (w->setting[i] & XDEM_SKIP_TIME_INTEGRAL) continue;
    if (w->shape[i] == XDEM_SHAPE_CLUMP) {
      v2 F = V(0.0, 0.0);
      double T = 0.0;
      for (int k = 1; k <= w->num_sub[i]; ++k) {
        v2 fk = V(w->fx[i + k], w->fy[i + k]);
        F = vadd(F, fk);
        T += w->tq[i + k];
        T += vcross(V(w->bx[i + k], w->by[i + k]), fk);
      }
      v2 v = vdiv(vadd(vmul(V(w->vx[i], w->vy[i]), 1.0 - g * dt), vmul(vmul(F, w->im[i]), dt)),
                  1.0 + g * dt);
      w->vx[i] = v.x; w->vy[i] = v.y;
      w->x[i] += v.x * dt; w->y[i] += v.y * dt;
      w->w[i] = (w->w[i] * (1.0 - g * dt) + T * w->iI[i] * dt) / (1.0 + g * dt);
      w->rot[i] += w->w[i] * dt;
      double angle = w->w[i] * dt;
      m2 R = M(cos(angle), -sin(angle), sin(angle), cos(angle));
      for (int k = 1; k <= w->num_sub[i]; ++k) {
        v2 b = mmulv(R, V(w->bx[i + k], w->by[i + k]));
        w->bx[i + k] = b.x; w->by[i + k] = b.y;
        v2 sv = vadd(v, vcrossw(b, w->w[i]));
        w->vx[i + k] = sv.x; w->vy[i + k] = sv.y;
        w->x[i + k] = w->x[i] + b.x; w->y[i + k] = w->y[i] + b.y;
        w->w[i + k] = w->w[i];
        w->rot[i + k] += angle;
      }
      continue;
    }
    v2 v = vdiv(vadd(vmul(V(w->vx[i], w->vy[i]), 1.0 - g * dt),
                     vmul(vmul(V(w->fx[i], w->fy[i]), w->im[i]), dt)),
                1.0 + g * dt);
    w->vx[i] = v.x; w->vy[i] = v.y;
    w->x[i] += v.x * dt; w->y[i] += v.y * dt;
    w->w[i] = (w->w[i] * (1.0 - g * dt) + w->tq[i] * w->iI[i] * dt) / (1.0 + g * dt);
    w->rot[i] += w->w[i] * dt;
  }
  /* a non-finite state (the reference carries NaN on without a word) */
  for (int i = 0; i < w->n; ++i)
    if (!isfinite(w->x[i]) || !isfinite(w->y[i]) || !isfinite(w->vx[i]) || !isfinite(w->vy[i]) ||
        !isfinite(w->rot[i]) || !isfinite(w->w[i])) {
      w->status |= XDEM_ERR_NONFINITE;
      break;
    }
}

/* BaseWorld::resetVelocityOfRattlers / scaleVelocityOfRattlers (BaseWorld.cpp:79-106) */
static void rattlers(xo_world* w, int reset, double scale) {
  for (int i = 0; i < w->n; ++i) {
    if (w->setting[i] & XDEM_SKIP_MACRO_SUM) continue;
    if (!is_rattler(w, i)) continue;
    if (reset) {
      w->vx[i] = 0.0; w->vy[i] = 0.0; w->w[i] = 0.0;
    } else {
      w->vx[i] *= scale; w->vy[i] *= scale; w->w[i] *= scale;
    }
  }
}

/* BaseWorld::updateTotalStress (BaseWorld.cpp:158-176) with
   BaseParticle::getStressFromContactList (BaseParticle.cpp:143-151) and
   GluedParticle::getStressFromContactList (GluedParticle.cpp:127-139) */
static void update_total_stress(xo_world* w) {
  m2 tot = M(0.0, 0.0, 0.0, 0.0);
  for (int i = 0; i < w->n; ++i) {
    if (w->setting[i] & XDEM_SKIP_MACRO_SUM) continue;
    m2 s = M(0.0, 0.0, 0.0, 0.0);
    if (w->shape[i] == XDEM_SHAPE_CLUMP) {
      for (int q = 1; q <= w->num_sub[i]; ++q) {
        int sp = i + q;
        v2 bv = V(w->bx[sp], w->by[sp]);
        for (int64_t k = w->cstart[sp]; k < w->cstart[sp + 1]; ++k)
          s = madd(s, mdyad(w->con[k].f, vadd(w->con[k].b, bv)));
      }
    } else {
      for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k)
        s = madd(s, mdyad(w->con[k].f, w->con[k].b));
    }
    tot = madd(tot, s);
  }
  tot = mdivs(tot, w->xlen * w->ylen);
  w->stress[0] = tot.xx; w->stress[1] = tot.xy; w->stress[2] = tot.yx; w->stress[3] = tot.yy;
}

static void scale_positions(xo_world* w, double sx, double sy) {
  for (int i = 0; i < w->n; ++i) {
    w->x[i] *= sx;
    w->y[i] *= sy;
  }
}

#define MAX_SCALE_RATE 100000000.0

/* PeriodicControlWorld box laws (PeriodicControlWorld.cpp:124-237) */
static void box_law(xo_world* w, int law, double p0, double p1) {
  double dt = w->dt;
  if (law == XDEM_BOX_STRAIN) {
    double sx = 1.0 + p0 * w->xlen * dt;
    double sy = 1.0 + p1 * w->ylen * dt;
    w->xmin *= sx; w->xmax *= sx; w->ymin *= sy; w->ymax *= sy;
    w->xlen = w->xmax - w->xmin; w->ylen = w->ymax - w->ymin;
    scale_positions(w, sx, sy);
  } else if (law == XDEM_BOX_STRESS_UNIFORM) {
    double hydro = (w->stress[0] + w->stress[3]) / 2.0;
    double dv = (p0 - hydro) * w->xlen * dt;
    w->velX += dv;
    w->velY = w->velX;
    double scale = (w->xmin + dv * dt) / w->xmin;
    w->xmin += dv * dt; w->xmax = -w->xmin; w->xlen = w->xmax - w->xmin;
    w->ymin += dv * dt; w->ymax = -w->ymin; w->ylen = w->ymax - w->ymin;
    scale_positions(w, scale, scale);
  } else if (law == XDEM_BOX_STRESS_XY) {
    double pre = w->xmin;
    double sxx = w->stress[0];
    if (fabs(sxx) < p0) w->velX *= (1.0 - dt * 1.0);
    double dv = (p0 - sxx) * w->xlen / w->vmass * dt;
    w->velX = dv;
    if (fabs(w->velX) / w->xlen > MAX_SCALE_RATE * dt) w->velX = MAX_SCALE_RATE * dt * w->xlen;
    w->xmin += w->velX * dt; w->xmax = -w->xmin; w->xlen = w->xmax - w->xmin;
    double scale = w->xmin / pre;
    scale_positions(w, scale, 1.0);
    pre = w->ymin;
    double syy = w->stress[3];
    if (fabs(syy) < p0) w->velY *= (1.0 - dt * 1.0);
    dv = (p0 - syy) * w->ylen / w->vmass * dt;
    w->velY = dv;
    if (fabs(w->velY) / w->ylen > MAX_SCALE_RATE * dt) w->velY = MAX_SCALE_RATE * dt * w->ylen;
    w->ymin += w->velY * dt; w->ymax = -w->ymin; w->ylen = w->ymax - w->ymin;
    scale = w->ymin / pre;
    scale_positions(w, 1.0, scale);
  } else if (law == XDEM_BOX_STRESS_UNIFORM_LIMIT) {
    double prex = w->xmin;
    double hydro = (w->stress[0] + w->stress[3]) / 2.0;
    double dv = (p0 - hydro) * w->xlen * dt;
    w->velX += dv;
    if ((fabs(w->velX) / (w->xlen / 2.0)) > w->max_strain_rate)
      w->velX = fabs(w->velX) / w->velX * (w->xlen / 2.0) * w->max_strain_rate;
    w->velY = w->velX;
    w->xmin += w->velX * dt; w->xmax = -w->xmin; w->xlen = w->xmax - w->xmin;
    w->ymin += w->velY * dt; w->ymax = -w->ymin; w->ylen = w->ymax - w->ymin;
    double scale = w->xmin / prex;
    scale_positions(w, scale, scale);
  }
}

/* LeesEdwardsBoundaryWorld::updateLeesEdwardBoundary (:285-296) */
static void update_le_boundary(xo_world* w) {
  w->shift_vel = w->shift_rate * w->ylen;
  w->strain += w->shift_rate * w->dt;
  w->shift += w->shift_vel * w->dt;
  if (w->shift > w->xmax) w->shift -= w->xlen;
  else if (w->shift < w->xmin) w->shift += w->xlen;
}

/* scaleBoundarySizeToGivenSolidFraction (PeriodicBoundaryWorld.cpp:276-284) */
static void scale_to_fraction(xo_world* w, double phi) {
  double cur = w->total_volume / (w->xlen * w->ylen);
  double scale = sqrt(cur / phi);
  scale_positions(w, scale, scale);
  w->xmin *= scale; w->xmax *= scale; w->ymin *= scale; w->ymax *= scale;
  w->xlen = w->xmax - w->xmin; w->ylen = w->ymax - w->ymin;
}

/* takeTimeStep of each world kind (PeriodicBoundaryWorld.cpp:119-127,
   PeriodicControlWorld.cpp:114-122, LeesEdwardsBoundaryWorld.cpp:21-31) */
static void take_time_step(xo_world* w) {
  int kind = w->prm.world_kind;
  modify_particle_position(w);
  if (kind == XDEM_WORLD_LEES_EDWARDS) background_velocity(w, 1);
  find_possible_contacts(w);
  update_contacts(w);
  if (kind == XDEM_WORLD_LEES_EDWARDS) background_velocity(w, 0);
  collect_force_and_torque(w);
  take_time_integral(w);
  if (kind == XDEM_WORLD_PERIODIC_CONTROL) rattlers(w, 1, 0.0);
  if (kind == XDEM_WORLD_LEES_EDWARDS) update_le_boundary(w);
}

enum {
  RH_MODIFY = 0, RH_APPLY_BG = 1, RH_REMOVE_BG = 2, RH_FIND = 3, RH_UPDATE = 4, RH_COLLECT = 5,
  RH_INTEGRATE = 6, RH_RESET_RATTLERS = 7, RH_SCALE_RATTLERS = 8, RH_STRESS = 9,
  RH_BOX_LAW = 10, RH_LE_BOUNDARY = 11, RH_TAKE_STEP = 12, RH_SCALE_TO_FRACTION = 13
};

int32_t xo_call(xo_world* w, int32_t which, double a, double b, double c) {
  switch (which) {
    case RH_MODIFY: modify_particle_position(w); break;
    case RH_APPLY_BG: background_velocity(w, 1); break;
    case RH_REMOVE_BG: background_velocity(w, 0); break;
    case RH_FIND: find_possible_contacts(w); break;
    case RH_UPDATE: update_contacts(w); break;
    case RH_COLLECT: collect_force_and_torque(w); break;
    case RH_INTEGRATE: take_time_integral(w); break;
    case RH_RESET_RATTLERS: rattlers(w, 1, 0.0); break;
    case RH_SCALE_RATTLERS: rattlers(w, 0, a); break;
    case RH_STRESS: update_total_stress(w); break;
    case RH_BOX_LAW: box_law(w, (int)a, b, c); break;
    case RH_LE_BOUNDARY: update_le_boundary(w); break;
    case RH_TAKE_STEP: take_time_step(w); break;
    case RH_SCALE_TO_FRACTION: scale_to_fraction(w, a); break;
    default: return XDEM_ERR_ARGUMENT;
  }
  return (int32_t)w->status;
}

int32_t xo_run(xo_world* w, int32_t nsteps, const xdem_control* ctl, int32_t* steps_done) {
  int s = 0;
  for (; s < nsteps; ++s) {
    if (ctl->scale_rattlers) rattlers(w, 0, ctl->rattler_scale);
    if (ctl->sequence == XDEM_SEQ_SUBSTEPS) {
      modify_particle_position(w);
      find_possible_contacts(w);
      update_contacts(w);
      collect_force_and_torque(w);
      take_time_integral(w);
    } else {
      take_time_step(w);
    }
    if (ctl->reset_rattlers) rattlers(w, 1, 0.0);
    if (ctl->update_stress) update_total_stress(w);
    if (ctl->box_law != XDEM_BOX_NONE) box_law(w, ctl->box_law, ctl->p0, ctl->p1);
    if (ctl->stop_on_pressure && (w->stress[0] + w->stress[3]) / 2.0 >= ctl->stop_pressure) {
      ++s;
      break;
    }
  }
  if (steps_done) *steps_done = s;
  return (int32_t)w->status;
}

/* QuadronAnalysis rattler removal, coordination number and solid fraction
   (QuadronAnalysis.cpp:663-668, :980-986, :144-165, :703-713, :724-732).
   Removing particles with exactly one active contact until none is left
   leaves the same set in any order, so the peeling below uses a queue. */
void xo_quadron_z_phi(xo_world* w, double* out) {
  int n = w->n;
  int64_t nc = w->ncon;
  int* deg = (int*)calloc((size_t)n, sizeof(int));
  int* active = (int*)malloc(sizeof(int) * n);
  unsigned char* cact = (unsigned char*)malloc((size_t)(nc > 0 ? nc : 1));
  int64_t* adj_start = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  for (int i = 0; i < n; ++i)
    for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k) {
      adj_start[i + 1]++;
      adj_start[w->con[k].j + 1]++;
    }
  for (int i = 0; i < n; ++i) adj_start[i + 1] += adj_start[i];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  memcpy(fill, adj_start, sizeof(int64_t) * (n + 1));
  int64_t* adj = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * nc > 0 ? 2 * nc : 1));
  for (int i = 0; i < n; ++i)
    for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k) {
      adj[fill[i]++] = k;
      adj[fill[w->con[k].j]++] = k;
    }
  int* owner = (int*)malloc(sizeof(int) * (size_t)(nc > 0 ? nc : 1));
  for (int i = 0; i < n; ++i)
    for (int64_t k = w->cstart[i]; k < w->cstart[i + 1]; ++k) owner[k] = i;
  for (int64_t k = 0; k < nc; ++k) cact[k] = 1;
  for (int i = 0; i < n; ++i) {
    deg[i] = (int)(adj_start[i + 1] - adj_start[i]);
    active[i] = deg[i] > 0;
  }
  int* queue = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int qh = 0, qt = 0;
  for (int i = 0; i < n; ++i)
    if (active[i] && deg[i] == 1) queue[qt++] = i;
  while (qh < qt) {
    int p = queue[qh++];
    if (!active[p] || deg[p] != 1) continue;
    active[p] = 0;
    for (int64_t a = adj_start[p]; a < adj_start[p + 1]; ++a) {
      int64_t k = adj[a];
      if (!cact[k]) continue;
      cact[k] = 0;
      int o = owner[k] == p ? w->con[k].j : owner[k];
      deg[p]--;
      deg[o]--;
      if (active[o] && deg[o] == 0) active[o] = 0; /* its only contact was this one */
      else if (active[o] && deg[o] == 1) queue[qt++] = o;
    }
  }
  int np = 0;
  int64_t ncact = 0;
  double vol = 0.0;
  for (int i = 0; i < n; ++i)
    if (active[i]) { np++; vol += w->vol[i]; }
  for (int64_t k = 0; k < nc; ++k) ncact += cact[k];
  out[0] = np == 0 ? 0.0 : (double)ncact / np * 2.0;
  out[1] = vol / (w->xlen * w->ylen);
  free(deg); free(active); free(cact); free(adj_start); free(fill); free(adj); free(owner);
  free(queue);
}
