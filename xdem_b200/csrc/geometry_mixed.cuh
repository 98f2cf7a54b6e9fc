// geometry_mixed.cuh — contact geometry of the mixed-precision path.
//
// Positions, velocities, the tangential spring and the Lees-Edwards shift stay
// FP64; the geometry's heavy arithmetic runs in FP32, and the two quantities
// whose conditioning needs FP64 are evaluated in FP64 from the FP32 result:
//
//  * circles: the overlap r_i + r_j - |d| (a difference of O(1) numbers that
//    is O(1e-3)) is the reference's FP64 expression (CircularParticle.cpp:
//    67-77), so the contact decision is the FP64 one; normal, contact point
//    and relative velocity are FP32.
//
//  * ellipses, closest approach: the distance of closest approach along d̂
//    is the root of Perram and Wertheim's contact function
//        F(λ) = λ(1-λ) dᵀ C(λ)⁻¹ d,   C(λ) = (1-λ) A_i⁻¹ + λ A_j⁻¹,
//    σ = |d| / sqrt(max_λ F) (J. Comput. Phys. 58, 409 (1985)), the same
//    quantity the reference builds from Zheng and Palffy-Muhoray's quartic
//    (EllipticParticle.cpp:34-285): the tangent point is
//    p_i + (1-λ*) A_i⁻¹ C⁻¹ d and the normal C⁻¹ d / |C⁻¹ d|, exactly the
//    reference's contactPoint and normal (EllipticParticle.cpp:188-221).
//    λ* is found by Newton in FP32 on d/dλ log F; F is then evaluated once in
//    FP64 at that λ.  F is stationary at λ*, so an FP32 error ε in λ moves
//    F by O(ε²) (~1e-12 relative) and the FP64 overlap σ - |d| keeps ~1e-10
//    relative accuracy where an all-FP32 difference would lose 1e-4.
//
//    The reference orders the two eigenvalues of its matrix A' by their
//    truncated integer magnitudes (int abs on a double, MathMatrix2d.h:122),
//    which exchanges them whenever both share an integer part; its two
//    rejection tests (EllipticParticle.cpp:77-84) then discard some pairs that
//    touch, and deep overlaps come out differently.  For such pairs the two
//    tests are evaluated here in FP32 with the exchanged semi-axes: a pair
//    they reject has no contact, as in the reference; a pair they pass, if
//    its overlap is below a tenth of the contact distance, has the reference's
//    geometry, which the contact function reproduces.  A pair within FP32
//    error of a test's threshold or of an integer eigenvalue, or overlapping
//    deeper, is handed to the reference's FP64 construction (a separate pass,
//    so that warps stay converged), which keeps the contact set the FP64
//    path's.
#pragma once
#include "geometry.cuh"

namespace xdem {

// Geometry result of the mixed path: FP64 overlap and contact-point offset
// base, FP32 directions and velocities.
struct GeomM {
  int iters;
  float2 n;      // unit normal (from i towards j)
  float2 cpo;    // contact point - p_i
  float2 bv1;    // contact point - p_i
  float2 bv2;    // contact point - (p_j + offset)
  double overlap;
  float2 rv, nrv, srv;
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// relative velocity at the contact point (BaseParticle.cpp:11-25) in FP32
__device__ __forceinline__ void relative_velocity_m(const PState& a, const PState& b,
                                                    vec2<double> ovel, GeomM& g) {
  const float wa = (float)a.w, wb = (float)b.w;
  const float vax = (float)a.vx - wa * g.bv1.y, vay = (float)a.vy + wa * g.bv1.x;
  const float vbx = (float)(b.vx + ovel.x) - wb * g.bv2.y;
  const float vby = (float)(b.vy + ovel.y) + wb * g.bv2.x;
  g.rv = f2(vax - vbx, vay - vby);
  const float vn = g.rv.x * g.n.x + g.rv.y * g.n.y;
  g.nrv = f2(g.n.x * vn, g.n.y * vn);
  g.srv = f2(g.rv.x - g.nrv.x, g.rv.y - g.nrv.y);
}

// circle-circle with the FP64 overlap (CircularParticle.cpp:67-92)
__device__ __forceinline__ bool circle_circle_m(const PState& a, const PState& b, vec2<double> off,
                                                vec2<double> ovel, GeomM& g) {
  const double dx = (b.x + off.x) - a.x, dy = (b.y + off.y) - a.y;
  const double distance = sqrt(dx * dx + dy * dy);
  const double overlap = (a.r + b.r) - distance;
  if (overlap < 0.0) return false;
  g.overlap = overlap;
  g.iters = 0;
  const float inv = distance != 0.0 ? (float)(1.0 / distance) : 0.0f;
  g.n = f2((float)dx * inv, (float)dy * inv);
  // midpoint of the two surface points
  const float ra = (float)a.r, rb = (float)b.r, fdx = (float)dx, fdy = (float)dy;
  const float h = 0.5f * (ra - rb);
  g.cpo = f2(0.5f * fdx + g.n.x * h, 0.5f * fdy + g.n.y * h);
  g.bv1 = g.cpo;
  g.bv2 = f2(g.cpo.x - fdx, g.cpo.y - fdy);
  relative_velocity_m(a, b, ovel, g);
  return true;
}

// Outcome of the mixed closest-approach routine.
enum : int { PW_NONE = 0, PW_CONTACT = 1, PW_FALLBACK = 2 };

constexpr int kLambdaCap = 8;

// Closest approach of two ellipses by the contact function (see the file
// comment).  csa/csb: FP64 (cos, sin) of the two orientations.
__device__ __forceinline__ int ellipse_closest_m(const PState& a, const PState& b,
                                                 vec2<double> off, vec2<double> ovel, double2 csa,
                                                 double2 csb, GeomM& g) {
  // ---- FP64 inputs of the contact function -----------------------------
  const double a1 = a.r, a2 = b.r;
  const double b1 = a1 / a.asp, b2 = a2 / b.asp;
  const double dx = (b.x + off.x) - a.x, dy = (b.y + off.y) - a.y;

  // ---- reference eigenvalue ordering, FP32 -----------------------------
  // A' = (b1²/b2²) P Q P with P = I + η k1k1ᵀ, Q = I - e2² k2k2ᵀ
  // (EllipticParticle.cpp:59-71); its eigenvalues from the trace and
  // det A' = (a1 b1 / (a2 b2))²
  const float c1 = (float)csa.x, s1 = (float)csa.y, c2 = (float)csb.x, s2 = (float)csb.y;
  bool exchanged;
  {
    const float fa1 = (float)a1, fb1 = (float)b1, fa2 = (float)a2, fb2 = (float)b2;
    const float eta = fa1 / fb1 - 1.0f;
    const float e22 = 1.0f - (fb2 * fb2) / (fa2 * fa2);
    const float sc = (fb1 * fb1) / (fb2 * fb2);
    // A' = sc P Q P, P = I + η k1k1ᵀ, Q = I - e2² k2k2ᵀ (symmetric)
    const float Pxx = 1.0f + eta * c1 * c1, Pxy = eta * c1 * s1, Pyy = 1.0f + eta * s1 * s1;
    const float Qxx = 1.0f - e22 * c2 * c2, Qxy = -e22 * c2 * s2, Qyy = 1.0f - e22 * s2 * s2;
    const float Mxx = Pxx * Qxx + Pxy * Qxy, Mxy = Pxx * Qxy + Pxy * Qyy;
    const float Myx = Pxy * Qxx + Pyy * Qxy, Myy = Pxy * Qxy + Pyy * Qyy;
    const float Axx = sc * (Mxx * Pxx + Mxy * Pxy), Axy = sc * (Mxx * Pxy + Mxy * Pyy);
    const float Ayy = sc * (Myx * Pxy + Myy * Pyy);
    const float tr = Axx + Ayy;
    const float rt = (fa1 * fb1) / (fa2 * fb2);
    const float dt_ = rt * rt;  // det A' = (a1 b1 / (a2 b2))²
    float disc = tr * tr - 4.0f * dt_;
    disc = disc > 0.0f ? sqrtf(disc) : 0.0f;
    const float ev1 = 0.5f * (tr + disc), ev2 = 0.5f * (tr - disc);
    // FP32 error bound of the two eigenvalues (a few ulp of the trace)
    const float tol = 1e-5f * fmaxf(tr, 1.0f);
    const float f1lo = floorf(ev1 - tol), f1hi = floorf(ev1 + tol);
    const float f2lo = floorf(ev2 - tol), f2hi = floorf(ev2 + tol);
    if (f1lo != f1hi || f2lo != f2hi) return PW_FALLBACK;  // ambiguous in FP32
    exchanged = f1lo == f2lo;
    if (exchanged) {
      // the reference's rejection tests with its exchanged axes
      // (EllipticParticle.cpp:73-84): lx = ev2, ly = ev1
      if (fabsf(Axy) < 1e-4f * tr) return PW_FALLBACK;  // ill-conditioned eigenvector
      const float lx = ev2, ly = ev1;
      const float a2p = rsqrtf(ly), b2p = rsqrtf(lx);
      float kx = 1.0f, ky = (lx - Axx) / Axy;
      const float ik = rsqrtf(kx * kx + ky * ky);
      kx *= ik;
      ky *= ik;
      const float fdx = (float)dx, fdy = (float)dy;
      const float k1d = c1 * fdx + s1 * fdy, g1 = fb1 / fa1 - 1.0f;
      const float px = (fdx + c1 * k1d * g1) / fb1, py = (fdy + s1 * k1d * g1) / fb1;
      const float dn = sqrtf(px * px + py * py);
      const float r1 = dn - (1.0f + a2p);
      const float r2 = fabsf(px * kx + py * ky) - (1.0f + b2p);
      const float rtol = 2e-5f * (1.0f + dn);
      if (fabsf(r1) <= rtol || fabsf(r2) <= rtol) return PW_FALLBACK;
      if (r1 > 0.0f || r2 > 0.0f) {
        g.iters = 0;
        return PW_NONE;
      }
    }
  }

  // ---- λ* by Newton on d/dλ log F, FP32 ----------------------------------
  // With u = (k·d)², w = (k×d)², α = a², β = b²:
  //   N(λ) = (1-λ)(α1 w1 + β1 u1) + λ(α2 w2 + β2 u2)          = dᵀ adj C(λ) d
  //   D(λ) = (1-λ)² α1β1 + λ² α2β2 + λ(1-λ) M12,
  //   M12  = α1β2 + α2β1 + (α1-β1)(α2-β2) (k1×k2)²             = det C(λ)
  //   F(λ) = λ(1-λ) N(λ) / D(λ)
  float lam;
  int it = 0;
  {
    const float fdx = (float)dx, fdy = (float)dy;
    const float L = fdx * fdx + fdy * fdy;
    const float il = rsqrtf(L);
    const float ex = fdx * il, ey = fdy * il;  // d̂
    const float k1d = c1 * ex + s1 * ey, k1c = c1 * ey - s1 * ex;
    const float k2d = c2 * ex + s2 * ey, k2c = c2 * ey - s2 * ex;
    const float al1 = (float)(a1 * a1), be1 = (float)(b1 * b1);
    const float al2 = (float)(a2 * a2), be2 = (float)(b2 * b2);
    const float u1 = k1d * k1d, w1 = k1c * k1c, u2 = k2d * k2d, w2 = k2c * k2c;
    const float N0 = al1 * w1 + be1 * u1, N1 = al2 * w2 + be2 * u2;
    const float kx = c1 * s2 - s1 * c2;
    const float M12 = al1 * be2 + al2 * be1 + (al1 - be1) * (al2 - be2) * (kx * kx);
    const float D0 = al1 * be1, D1 = al2 * be2;
    const float dN = N1 - N0;
    const float Dpp = 2.0f * (D0 + D1 - M12);
    // start from the support-function ratio (exact for two circles)
    const float h1 = sqrtf(al1 * u1 + be1 * w1), h2 = sqrtf(al2 * u2 + be2 * w2);
    lam = h1 / (h1 + h2);
#pragma unroll 1
    for (; it < kLambdaCap; ++it) {
      const float om = 1.0f - lam;
      const float N = fmaf(lam, dN, N0);
      const float D = om * om * D0 + lam * lam * D1 + lam * om * M12;
      const float Dp = -2.0f * om * D0 + 2.0f * lam * D1 + (om - lam) * M12;
      const float il_ = 1.0f / lam, io = 1.0f / om;
      const float rN = dN / N, rD = Dp / D;
      const float h = il_ - io + rN - rD;
      const float hp = -il_ * il_ - io * io - rN * rN - Dpp / D + rD * rD;
      const float step = h / hp;
      lam = fminf(fmaxf(lam - step, 1e-6f), 1.0f - 1e-6f);
      if (fabsf(step) < 2e-7f) {
        ++it;
        break;
      }
    }
  }

  // ---- FP64 evaluation of F at λ*, overlap ---------------------------------
  const double lamd = (double)lam, omd = 1.0 - lamd;
  const double A1 = a1 * a1, B1 = b1 * b1, A2 = a2 * a2, B2 = b2 * b2;
  const double k1d = csa.x * dx + csa.y * dy, k1c = csa.x * dy - csa.y * dx;
  const double k2d = csb.x * dx + csb.y * dy, k2c = csb.x * dy - csb.y * dx;
  const double N = omd * (A1 * (k1c * k1c) + B1 * (k1d * k1d)) + lamd * (A2 * (k2c * k2c) + B2 * (k2d * k2d));
  const double kx = csa.x * csb.y - csa.y * csb.x;
  const double M12 = A1 * B2 + A2 * B1 + (A1 - B1) * (A2 - B2) * (kx * kx);
  const double D = omd * omd * (A1 * B1) + lamd * lamd * (A2 * B2) + lamd * omd * M12;
  const double L = dx * dx + dy * dy;
  const double dlen = sqrt(L);
  const double sigma = sqrt(L * D / (lamd * omd * N));
  const double overlap0 = sigma - dlen;
  g.iters = it;
  if (!(overlap0 >= 0.0)) return PW_NONE;
  // deep overlaps of exchanged pairs: the reference's construction decides
  if (exchanged && overlap0 > 0.1 * sigma) return PW_FALLBACK;

  // ---- normal, tangent point, relative velocity, FP32 ----------------------
  {
    const float l = lam, o = 1.0f - lam;
    const float fdx = (float)dx, fdy = (float)dy;
    // inverse shape matrices A⁻¹ = β I + (α-β) k kᵀ
    const float al1 = (float)A1, be1 = (float)B1, al2 = (float)A2, be2 = (float)B2;
    const float g1 = al1 - be1, g2 = al2 - be2;
    const float Ai_xx = be1 + g1 * c1 * c1, Ai_yy = be1 + g1 * s1 * s1, Ai_xy = g1 * c1 * s1;
    const float Bi_xx = be2 + g2 * c2 * c2, Bi_yy = be2 + g2 * s2 * s2, Bi_xy = g2 * c2 * s2;
    const float Cxx = o * Ai_xx + l * Bi_xx, Cyy = o * Ai_yy + l * Bi_yy, Cxy = o * Ai_xy + l * Bi_xy;
    // v = adj(C) d ∝ C⁻¹ d
    const float vx = Cyy * fdx - Cxy * fdy, vy = -Cxy * fdx + Cxx * fdy;
    const float detC = Cxx * Cyy - Cxy * Cxy;
    const float iv = rsqrtf(vx * vx + vy * vy);
    g.n = f2(vx * iv, vy * iv);
    const float sc = o / detC;
    g.cpo = f2(sc * (Ai_xx * vx + Ai_xy * vy), sc * (Ai_xy * vx + Ai_yy * vy));
    // normalOverlap = overlap0 |d̂·n| (EllipticParticle.cpp:214-219)
    const float cosn = fabsf(fdx * g.n.x + fdy * g.n.y) * (float)(1.0 / dlen);
    g.overlap = overlap0 * (double)cosn;
    g.bv1 = g.cpo;
    g.bv2 = f2(g.cpo.x - fdx, g.cpo.y - fdy);
  }
  relative_velocity_m(a, b, ovel, g);
  return PW_CONTACT;
}

// FP64 result of the reference construction, in the mixed layout
__device__ __forceinline__ void geom_to_m(const Geom& s, const PState& a, GeomM& g) {
  g.iters = s.iters;
  g.n = f2((float)s.n.x, (float)s.n.y);
  g.cpo = f2((float)(s.cp.x - a.x), (float)(s.cp.y - a.y));
  g.bv1 = f2((float)s.bv1.x, (float)s.bv1.y);
  g.bv2 = f2((float)s.bv2.x, (float)s.bv2.y);
  g.overlap = s.overlap;
  g.rv = f2((float)s.rv.x, (float)s.rv.y);
  g.nrv = f2((float)s.nrv.x, (float)s.nrv.y);
  g.srv = f2((float)s.srv.x, (float)s.srv.y);
}

}  // namespace xdem
