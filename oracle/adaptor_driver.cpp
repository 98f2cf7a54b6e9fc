// adaptor_driver.cpp — TEST INFRASTRUCTURE ONLY.
//
// Runs driver loops written the way the reference's own drivers are
// (mainIsoCircPack_WCCM.cpp:46-126: random generation by takeTimeStep, then a
// second world on the same particles compressed by sub-steps under stress
// control; LeesEdwardsBoundaryWorld shear; clumps as in
// mainClumpParticleTest.cpp:95-150) twice from identical seeded inputs: once
// with the reference's world classes (the unmodified sources compiled by
// oracle/Makefile) and once with the drop-in GPU worlds of
// include/xdem_gpu_world.hpp.  The driver code is one template used for both;
// only the world types differ.  Prints one JSON line with the largest
// relative differences of the particle states, the contact maps, the stress
// and the box; exits 0 when every difference is within the case's tolerance.
//
//     adaptor_driver <case>    case: discs_compression | ellipses_lees_edwards | clumps_control
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "xdem_gpu_world.hpp"

namespace {

struct Particles {
  std::vector<CircularParticle> discs;
  std::vector<EllipticParticle> ellipses;
  std::vector<GluedParticle> clumps;
  std::vector<BaseParticle*> handlers;
};

// particles on a jittered square lattice in [-L/2, L/2)^2 (seeded)
void lattice(int n, double spacing, double& half, std::vector<vector2d>& pos, unsigned seed) {
  const int side = static_cast<int>(std::ceil(std::sqrt(static_cast<double>(n))));
  half = 0.5 * side * spacing;
  std::default_random_engine engine(seed);
  std::uniform_real_distribution<double> jitter(-0.05 * spacing, 0.05 * spacing);
  pos.clear();
  for (int k = 0; k < n; ++k) {
    const int ix = k % side, iy = k / side;
    pos.push_back(vector2d(-half + (ix + 0.5) * spacing + jitter(engine),
                           -half + (iy + 0.5) * spacing + jitter(engine)));
  }
}

void make_discs(Particles& P, int n, ContactModel* m, double& half) {
  std::vector<vector2d> pos;
  lattice(n, 1.25, half, pos, 11);
  std::default_random_engine engine(5);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::normal_distribution<double> vel(0.0, 0.05);
  P.discs.resize(n);
  for (int i = 0; i < n; ++i) {
    const double r = u(engine) < 0.5 ? 0.5 : 0.7;
    P.discs[i] = CircularParticle(i, r, pos[i], vector2d(vel(engine), vel(engine)), 0.0, 0.0, m);
    P.discs[i].calculateParticleProperties(1.0);
  }
  for (auto& d : P.discs) P.handlers.push_back(&d);
}

void make_ellipses(Particles& P, int n, ContactModel* m, double& half) {
  std::vector<vector2d> pos;
  lattice(n, 1.9, half, pos, 13);
  std::default_random_engine engine(7);
  std::uniform_real_distribution<double> b(0.5, 0.7), asp(1.0, 2.0), th(0.0, M_PI);
  std::normal_distribution<double> vel(0.0, 0.02);
  P.ellipses.resize(n);
  for (int i = 0; i < n; ++i) {
    const double k = asp(engine), a = k * b(engine);
    P.ellipses[i] = EllipticParticle(i, a, k, pos[i], vector2d(vel(engine), vel(engine)),
                                     th(engine), 0.0, m);
    P.ellipses[i].calculateParticleProperties(1.0);
  }
  for (auto& e : P.ellipses) P.handlers.push_back(&e);
}

// clumps of two or three circular sub-discs (GluedParticle), built as the
// reference's clump driver builds its clumps
void make_clumps(Particles& P, int nclump, ContactModel* m, double& half) {
  std::vector<vector2d> pos;
  lattice(nclump, 2.2, half, pos, 17);
  std::default_random_engine engine(9);
  std::uniform_int_distribution<int> count(2, 3);
  std::uniform_real_distribution<double> r(0.3, 0.6), off(-0.5, 0.5);
  std::vector<int> nsub(nclump);
  int total = 0;
  for (int i = 0; i < nclump; ++i) {
    nsub[i] = count(engine);
    total += nsub[i];
  }
  P.clumps.resize(nclump);
  P.discs.resize(total);
  int id = 0, d = 0;
  for (int i = 0; i < nclump; ++i) {
    P.clumps[i] = GluedParticle(id, vector2d(0.0, 0.0), 0.0);
    P.clumps[i].appendSetting(SETTING::SKIP_CONTACT_DETECTION);
    P.handlers.push_back(&P.clumps[i]);
    const int cid = id++;
    for (int k = 0; k < nsub[i]; ++k) {
      P.discs[d] = CircularParticle(id++, r(engine), pos[i] + vector2d(off(engine), off(engine)),
                                    vector2d(0.0, 0.0), 0.0, 0.0, m);
      P.discs[d].calculateParticleProperties(1.0);
      P.discs[d].setUpLevel(cid);
      P.discs[d].appendSetting(SETTING::SKIP_TIME_INTEGRAL);
      P.discs[d].appendSetting(SETTING::SKIP_MACRO_SUM);
      P.handlers.push_back(&P.discs[d]);
      P.clumps[i].pushBackSubParticle(&P.discs[d]);
      ++d;
    }
    P.clumps[i].calculateParticleProperties(1.0);
  }
}

struct Outcome {
  std::vector<BaseParticle*> particles;
  matrix2d stress;
  double box[4];
  int contacts;
};

// mainIsoCircPack_WCCM.cpp:46-126 in small: random generation, then
// compression by sub-steps with stressControlX/Y and rattler scaling
template <class PBW, class PCW>
void discs_compression(Particles& P, ContactModel* m, double half, Outcome& out) {
  const double dt = 2e-4;
  PBW rg(dt, P.handlers, m);
  rg.setWorldBoundary(-half, half, -half, half);
  rg.scaleBoundarySizeToGivenSolidFraction(0.80);
  for (int s = 0; s < 150; ++s) {
    rg.takeTimeStep();
    rg.resetVelocityOfRattlers();
  }
  PCW cw(dt, P.handlers, m);
  cw.setWorldBoundary(rg.getXmin(), rg.getXmax(), rg.getYmin(), rg.getYmax());
  cw.updateTotalParticleVolume();
  cw.setVirtualBoundaryMass();
  BaseParticle::_GlobalDamping_ = 0.1;
  for (int s = 0; s < 150; ++s) {
    cw.scaleVelocityOfRattlers(0.99);
    cw.modifyParticlePosition();
    cw.findPossibleContacts();
    cw.updateContacts();
    cw.collectForceAndTorque();
    cw.takeTimeIntegral();
    cw.updateTotalStress();
    cw.updatePeriodicBoundary_stressControlX(50.0);
    cw.updatePeriodicBoundary_stressControlY(50.0);
  }
  BaseParticle::_GlobalDamping_ = 0.0;
  out.stress = cw.getStress();
  out.box[0] = cw.getXmin();
  out.box[1] = cw.getXmax();
  out.box[2] = cw.getYmin();
  out.box[3] = cw.getYmax();
  out.contacts = cw.countActucalContacts();
  out.particles = P.handlers;
}

template <class LEW>
void ellipses_lees_edwards(Particles& P, ContactModel* m, double half, Outcome& out) {
  LEW w(1e-4, P.handlers, m);
  w.setWorldBoundary(-half, half, -half, half);
  w.scaleBoundarySizeToGivenSolidFraction(0.72);
  w.setShiftStrainRate(0.3);
  for (int s = 0; s < 120; ++s) {
    w.takeTimeStep();
    w.updateTotalStress();
  }
  out.stress = w.getStress();
  out.box[0] = w.getTotalShift();
  out.box[1] = w.getTotalStrain();
  out.box[2] = w.getXmin();
  out.box[3] = w.getYmax();
  out.contacts = w.countActucalContacts();
  out.particles = P.handlers;
}

template <class PCW>
void clumps_control(Particles& P, ContactModel* m, double half, Outcome& out) {
  PCW w(2e-4, P.handlers, m);
  w.setWorldBoundary(-half, half, -half, half);
  w.scaleBoundarySizeToGivenSolidFraction(0.62);
  w.setVirtualBoundaryMass();
  for (int s = 0; s < 120; ++s) {
    w.modifyParticlePosition();
    w.findPossibleContacts();
    w.updateContacts();
    w.collectForceAndTorque();
    w.takeTimeIntegral();
    w.resetVelocityOfRattlers();
    w.updateTotalStress();
    w.updatePeriodicBoundary_stressControlUniform(20.0);
  }
  out.stress = w.getStress();
  out.box[0] = w.getXmin();
  out.box[1] = w.getXmax();
  out.box[2] = w.getYmin();
  out.box[3] = w.getYmax();
  out.contacts = w.countActucalContacts();
  out.particles = P.handlers;
}

double rel(double a, double b, double scale) { return std::fabs(a - b) / std::max(scale, 1e-300); }

struct Diff {
  double state = 0.0, contact = 0.0, stress = 0.0, box = 0.0;
  int key_mismatch = 0;
};

// largest relative difference per group (relative to the group's largest
// magnitude in the reference run)
Diff compare(const Outcome& r, const Outcome& g) {
  Diff d;
  const size_t n = r.particles.size();
  double sp = 0.0, sv = 0.0, sr = 0.0, sw = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const BaseParticle* p = r.particles[i];
    sp = std::max({sp, std::fabs(p->getPosX()), std::fabs(p->getPosY())});
    sv = std::max({sv, std::fabs(p->getVelX()), std::fabs(p->getVelY())});
    sr = std::max(sr, std::fabs(p->getRot()));
    sw = std::max(sw, std::fabs(p->getRotVel()));
  }
  double sf = 0.0;
  for (size_t i = 0; i < n; ++i)
    for (const auto& kv : xdem_gpu::ParticleAccess::contacts(r.particles[i]))
      sf = std::max({sf, std::fabs(kv.second._normalForce.x()), std::fabs(kv.second._normalForce.y()),
                     std::fabs(kv.second._shearForce.x()), std::fabs(kv.second._shearForce.y())});
  for (size_t i = 0; i < n; ++i) {
    const BaseParticle *a = r.particles[i], *b = g.particles[i];
    d.state = std::max({d.state, rel(a->getPosX(), b->getPosX(), sp), rel(a->getPosY(), b->getPosY(), sp),
                        rel(a->getVelX(), b->getVelX(), sv), rel(a->getVelY(), b->getVelY(), sv),
                        rel(a->getRot(), b->getRot(), sr), rel(a->getRotVel(), b->getRotVel(), sw)});
    auto& ca = xdem_gpu::ParticleAccess::contacts(r.particles[i]);
    auto& cb = xdem_gpu::ParticleAccess::contacts(g.particles[i]);
    if (ca.size() != cb.size()) d.key_mismatch++;
    for (const auto& kv : ca) {
      auto it = cb.find(kv.first);
      if (it == cb.end()) {
        d.key_mismatch++;
        continue;
      }
      const ContactInformation &x = kv.second, &y = it->second;
      d.contact = std::max({d.contact, rel(x._normalForce.x(), y._normalForce.x(), sf),
                            rel(x._normalForce.y(), y._normalForce.y(), sf),
                            rel(x._shearForce.x(), y._shearForce.x(), sf),
                            rel(x._shearForce.y(), y._shearForce.y(), sf)});
    }
  }
  const double ss = std::max({std::fabs(r.stress.xx()), std::fabs(r.stress.xy()),
                              std::fabs(r.stress.yx()), std::fabs(r.stress.yy())});
  d.stress = std::max({rel(r.stress.xx(), g.stress.xx(), ss), rel(r.stress.xy(), g.stress.xy(), ss),
                       rel(r.stress.yx(), g.stress.yx(), ss), rel(r.stress.yy(), g.stress.yy(), ss)});
  double sb = 0.0;
  for (int k = 0; k < 4; ++k) sb = std::max(sb, std::fabs(r.box[k]));
  for (int k = 0; k < 4; ++k) d.box = std::max(d.box, rel(r.box[k], g.box[k], sb));
  return d;
}

}  // namespace

int main(int argc, char** argv) {
  const std::string which = argc > 1 ? argv[1] : "discs_compression";
  ContactModel model_r(1e4, 5e3, 0.372336, 0.5), model_g(1e4, 5e3, 0.372336, 0.5);
  Particles pr, pg;
  Outcome r, g;
  double half = 0.0;
  double tol = 1e-9;
  if (which == "discs_compression") {
    make_discs(pr, 400, &model_r, half);
    make_discs(pg, 400, &model_g, half);
    discs_compression<PeriodicBoundaryWorld, PeriodicControlWorld>(pr, &model_r, half, r);
    discs_compression<GpuPeriodicBoundaryWorld, GpuPeriodicControlWorld>(pg, &model_g, half, g);
  } else if (which == "ellipses_lees_edwards") {
    make_ellipses(pr, 300, &model_r, half);
    make_ellipses(pg, 300, &model_g, half);
    ellipses_lees_edwards<LeesEdwardsBoundaryWorld>(pr, &model_r, half, r);
    ellipses_lees_edwards<GpuLeesEdwardsBoundaryWorld>(pg, &model_g, half, g);
  } else if (which == "clumps_control") {
    make_clumps(pr, 120, &model_r, half);
    make_clumps(pg, 120, &model_g, half);
    clumps_control<PeriodicControlWorld>(pr, &model_r, half, r);
    clumps_control<GpuPeriodicControlWorld>(pg, &model_g, half, g);
  } else {
    std::printf("{\"case\": \"%s\", \"error\": \"unknown case\"}\n", which.c_str());
    return 2;
  }
  const Diff d = compare(r, g);
  const bool ok = d.key_mismatch == 0 && d.state <= tol && d.contact <= tol && d.stress <= tol &&
                  d.box <= tol && r.contacts == g.contacts && r.contacts > 0;
  std::printf(
      "{\"case\": \"%s\", \"particles\": %zu, \"contacts_ref\": %d, \"contacts_gpu\": %d, "
      "\"key_mismatch\": %d, \"state\": %.3e, \"contact_forces\": %.3e, \"stress\": %.3e, "
      "\"box\": %.3e, \"tol\": %.1e, \"ok\": %s}\n",
      which.c_str(), r.particles.size(), r.contacts, g.contacts, d.key_mismatch, d.state, d.contact,
      d.stress, d.box, tol, ok ? "true" : "false");
  return ok ? 0 : 1;
}
