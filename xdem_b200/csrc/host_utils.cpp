// host_utils.cpp — host-only set-up helpers of the C-ABI: seeded random
// sequential addition and the particle-property formulas of the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/xdem_gpu.h"

namespace {

constexpr double kPi = 3.14159265358979323846;  // M_PI

// splitmix64: a small, well-mixed, seedable generator
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

// EllipticParticle::pointInsideParticle (EllipticParticle.cpp:486-495) and
// CircularParticle::pointInsideParticle (CircularParticle.cpp:42-45)
bool point_inside(int shape, double r, double asp, double x, double y, double rot, double px,
                  double py) {
  if (shape == XDEM_SHAPE_CIRCLE) {
    double dx = x - px, dy = y - py;
    return std::sqrt(dx * dx + dy * dy) < r;
  }
  double cosa = std::cos(rot);
  double sina = std::sin(rot);
  double dd = (r / asp) * (r / asp);
  double DD = r * r;
  double a = std::pow(cosa * (px - x) + sina * (py - y), 2);
  double b = std::pow(sina * (px - x) - cosa * (py - y), 2);
  return (a / dd + b / DD) <= 1.0;
}

}  // namespace

extern "C" {

int32_t xdem_rsa_positions(int32_t n, const double* radius, const double box[4], uint64_t seed,
                           int64_t max_attempts, double* x, double* y) {
  if (n < 0 || !radius || !box || !x || !y) return XDEM_ERR_ARGUMENT;
  double xmin = box[0], xmax = box[1], ymin = box[2], ymax = box[3];
  double lx = xmax - xmin, ly = ymax - ymin;
  double rmax = 0.0;
  for (int i = 0; i < n; ++i) rmax = std::fmax(rmax, radius[i]);
  if (!(lx > 0) || !(ly > 0) || !(rmax > 0)) return XDEM_ERR_ARGUMENT;
  int nx = std::max(1, (int)std::floor(lx / (2.0 * rmax)));
  int ny = std::max(1, (int)std::floor(ly / (2.0 * rmax)));
  double cx = lx / nx, cy = ly / ny;
  std::vector<std::vector<int>> cells((size_t)nx * ny);
  SplitMix64 rng(seed);
  for (int i = 0; i < n; ++i) {
    bool placed = false;
    for (int64_t att = 0; att < max_attempts && !placed; ++att) {
      double px = xmin + rng.uniform() * lx;
      double py = ymin + rng.uniform() * ly;
      int ix = std::min(nx - 1, (int)((px - xmin) / cx));
      int iy = std::min(ny - 1, (int)((py - ymin) / cy));
      bool ok = true;
      for (int dx = -1; dx <= 1 && ok; ++dx)
        for (int dy = -1; dy <= 1 && ok; ++dy) {
          int jx = ((ix + dx) % nx + nx) % nx, jy = ((iy + dy) % ny + ny) % ny;
          for (int j : cells[(size_t)jy * nx + jx]) {
            double ddx = x[j] - px, ddy = y[j] - py;
            if (ddx > lx / 2) ddx -= lx;
            else if (ddx < -lx / 2) ddx += lx;
            if (ddy > ly / 2) ddy -= ly;
            else if (ddy < -ly / 2) ddy += ly;
            double s = radius[i] + radius[j];
            if (ddx * ddx + ddy * ddy < s * s) {
              ok = false;
              break;
            }
          }
        }
      if (ok) {
        x[i] = px;
        y[i] = py;
        cells[(size_t)iy * nx + ix].push_back(i);
        placed = true;
      }
    }
    if (!placed) return XDEM_ERR_CAPACITY;
  }
  return XDEM_OK;
}

// CircularParticle::calculateParticleProperties (CircularParticle.cpp:16-23),
// EllipticParticle::calculateParticleProperties (EllipticParticle.cpp:7-14)
// and SegmentObject::calculateParticleProperties (SegmentObject.cpp:4-10)
int32_t xdem_particle_properties(int32_t n, const int32_t* shape, const double* radius,
                                 const double* aspect, double density, double* volume,
                                 double* mass, double* inv_mass, double* inertia,
                                 double* inv_inertia) {
  if (n < 0 || !shape || !radius || !aspect || !volume || !mass || !inv_mass || !inertia ||
      !inv_inertia)
    return XDEM_ERR_ARGUMENT;
  for (int i = 0; i < n; ++i) {
    double r = radius[i];
    if (shape[i] == XDEM_SHAPE_CIRCLE) {
      volume[i] = kPi * r * r;
      mass[i] = volume[i] * density;
      inv_mass[i] = 1.0 / mass[i];
      inertia[i] = mass[i] * r * r / 2.0;
      inv_inertia[i] = 1.0 / inertia[i];
    } else if (shape[i] == XDEM_SHAPE_ELLIPSE) {
      double k = aspect[i];
      volume[i] = kPi * r * r / k;
      mass[i] = volume[i] * density;
      inv_mass[i] = 1.0 / mass[i];
      inertia[i] = mass[i] * (r * r + r * r / k / k) / 4.0;
      inv_inertia[i] = 1.0 / inertia[i];
    } else if (shape[i] == XDEM_SHAPE_SEGMENT) {
      // SegmentObject::calculateParticleProperties (SegmentObject.cpp:4-10):
      // linear volume, a rod's inertia
      volume[i] = r * 2.0;
      mass[i] = volume[i] * density;
      inv_mass[i] = 1.0 / mass[i];
      inertia[i] = mass[i] * r * r / 3.0;
      inv_inertia[i] = 1.0 / inertia[i];
    } else {
      return XDEM_ERR_ARGUMENT;
    }
  }
  return XDEM_OK;
}

// GluedParticle::calculateParticleProperties (GluedParticle.cpp:7-80): mass
// centre, mass and inertia of a clump by a 100-cell quadrature over the union of
// its sub-particles (inertia sums dm * distance, as the reference does).
// out_clump: x, y, volume, mass, inv_mass, inertia, inv_inertia.
int32_t xdem_clump_properties(int32_t nsub, const int32_t* sub_shape, const double* sub_radius,
                              const double* sub_aspect, const double* sub_x, const double* sub_y,
                              const double* sub_rot, double density, double* out_clump,
                              double* branch_x, double* branch_y) {
  if (nsub <= 0 || !sub_shape || !sub_radius || !sub_aspect || !sub_x || !sub_y || !sub_rot ||
      !out_clump || !branch_x || !branch_y)
    return XDEM_ERR_ARGUMENT;
  double xmin = 1e10, xmax = -1e10, ymin = 1e10, ymax = -1e10, rmax = 0.0;
  for (int k = 0; k < nsub; ++k) {
    double r = sub_radius[k];
    xmin = (sub_x[k] - r) < xmin ? (sub_x[k] - r) : xmin;
    xmax = (sub_x[k] + r) > xmax ? (sub_x[k] + r) : xmax;
    ymin = (sub_y[k] - r) < ymin ? (sub_y[k] - r) : ymin;
    ymax = (sub_y[k] + r) > ymax ? (sub_y[k] + r) : ymax;
    rmax = r > rmax ? r : rmax;
  }
  xmin -= 0.1 * rmax;
  xmax += 0.1 * rmax;
  ymin -= 0.1 * rmax;
  ymax += 0.1 * rmax;
  double lx = xmax - xmin, ly = ymax - ymin;
  double dl = (lx < ly ? lx : ly) / 100;
  int nx = (int)std::floor(lx / dl);
  int ny = (int)std::floor(ly / dl);
  double dlx = lx / nx, dly = ly / ny;
  std::vector<double> xx(nx), yy(ny);
  for (int i = 0; i < nx; ++i) xx[i] = xmin + dlx * (i + 0.5);
  for (int j = 0; j < ny; ++j) yy[j] = ymin + dly * (j + 0.5);
  double dvolume = dlx * dly;
  double dmass = dvolume * density;
  double mcx = 0.0, mcy = 0.0, volume = 0.0, mass = 0.0, inertia = 0.0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nsub; ++k)
        if (point_inside(sub_shape[k], sub_radius[k], sub_aspect[k], sub_x[k], sub_y[k],
                         sub_rot[k], xx[i], yy[j])) {
          mcx += xx[i] * dmass;
          mcy += yy[j] * dmass;
          volume += dvolume;
          mass += dmass;
          break;
        }
  mcx /= mass;
  mcy /= mass;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nsub; ++k)
        if (point_inside(sub_shape[k], sub_radius[k], sub_aspect[k], sub_x[k], sub_y[k],
                         sub_rot[k], xx[i], yy[j])) {
          double dx = mcx - xx[i], dy = mcy - yy[j];
          inertia += dmass * std::sqrt(dx * dx + dy * dy);
          break;
        }
  out_clump[0] = mcx;
  out_clump[1] = mcy;
  out_clump[2] = volume;
  out_clump[3] = mass;
  out_clump[4] = 1.0 / mass;
  out_clump[5] = inertia;
  out_clump[6] = 1.0 / inertia;
  for (int k = 0; k < nsub; ++k) {
    branch_x[k] = sub_x[k] - mcx;
    branch_y[k] = sub_y[k] - mcy;
  }
  return XDEM_OK;
}

// named ranges for profilers (NVTX; no effect unless a tool is attached)
int32_t xdem_range_push(const char* name) {
  nvtxRangePushA(name ? name : "");
  return XDEM_OK;
}
int32_t xdem_range_pop(void) {
  nvtxRangePop();
  return XDEM_OK;
}

}  // extern "C"
