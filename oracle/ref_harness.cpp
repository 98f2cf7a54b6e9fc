// ref_harness.cpp — TEST INFRASTRUCTURE ONLY (the oracle's strongest form).
//
// Drives the UNMODIFIED reference xDEM classes, compiled from their own sources
// by oracle/Makefile into oracle/_ref/libxdem_ref.so, behind a C API that uses
// the same structs as include/xdem_gpu.h.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load the result; the product never links
// it.
//
// The harness needs private/protected members of the reference classes (the
// contact maps, _totalForce, clump branch vectors, the Strobach contact routine
// that EllipticParticle.cpp:27 does not dispatch), so it widens access for this
// translation unit only.  Class layout is unaffected.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#include <omp.h>

#define private public
#define protected public
#include "CircularParticle.h"
#include "EllipticParticle.h"
#include "GluedParticle.h"
#include "PeriodicBoundaryWorld.h"
#include "PeriodicControlWorld.h"
#include "LeesEdwardsBoundaryWorld.h"
#include "QuadronAnalysis.h"
#undef private
#undef protected

#include "../include/xdem_gpu.h"

namespace {

// EllipticParticle with the intersection (Strobach) contact routine in place of
// closest approach: the reference selects the routine by editing
// EllipticParticle.cpp:27; this subclass is that edit.
class IntersectionEllipse : public EllipticParticle {
 public:
  using EllipticParticle::EllipticParticle;
  bool calculateContactGeometry(const BaseParticle* otherParticle, ContactGeometry& cg,
                                const vector2d& offset, const vector2d& offsetVel) override {
    if (const EllipticParticle* other = dynamic_cast<const EllipticParticle*>(otherParticle)) {
      if (!takeCoarseDetection(otherParticle, offset)) {
        cg.isContacted = false;
        return false;
      }
      return contactWithEllipticParticle0(other, cg, offset, offsetVel);
    }
    printf("Todo: more particle types...\n");
    exit(-1);
  }
};

struct Harness {
  xdem_params prm{};
  std::unique_ptr<ContactModel> model;
  std::vector<std::unique_ptr<BaseParticle>> owned;
  std::vector<BaseParticle*> handlers;
  std::unique_ptr<BaseWorld> world;
  int kind = 0;
  int threads = 1;

  PeriodicBoundaryWorld* periodic() { return static_cast<PeriodicBoundaryWorld*>(world.get()); }
  PeriodicControlWorld* control() { return static_cast<PeriodicControlWorld*>(world.get()); }
  LeesEdwardsBoundaryWorld* le() { return static_cast<LeesEdwardsBoundaryWorld*>(world.get()); }
};

std::unique_ptr<BaseParticle> make_particle(int shape, int method, int id, double radius,
                                            double aspect, double x, double y, double vx,
                                            double vy, double rot, double rotVel,
                                            ContactModel* m) {
  vector2d p(x, y), v(vx, vy);
  if (shape == XDEM_SHAPE_CIRCLE)
    return std::unique_ptr<BaseParticle>(new CircularParticle(id, radius, p, v, rot, rotVel, m));
  if (shape == XDEM_SHAPE_ELLIPSE) {
    if (method == XDEM_ELLIPSE_INTERSECTION)
      return std::unique_ptr<BaseParticle>(
          new IntersectionEllipse(id, radius, aspect, p, v, rot, rotVel, m));
    return std::unique_ptr<BaseParticle>(
        new EllipticParticle(id, radius, aspect, p, v, rot, rotVel, m));
  }
  GluedParticle* g = new GluedParticle(id, v, rotVel);
  g->_position = p;
  g->_rotation = rot;
  g->_contactModel = m;
  return std::unique_ptr<BaseParticle>(g);
}

ContactInformation* find_contact(BaseParticle* p, int other) {
  auto it = p->_contactInfo.find(other);
  return it == p->_contactInfo.end() ? nullptr : &it->second;
}

}  // namespace

extern "C" {

void* refh_create(const xdem_params* prm, int32_t num_threads) {
  Harness* h = new Harness();
  h->prm = *prm;
  h->kind = prm->world_kind;
  h->threads = num_threads > 0 ? num_threads : 1;
  h->model.reset(new ContactModel(prm->normal_stiffness, prm->shear_stiffness,
                                  prm->restitution_coeff, prm->frictional_coeff));
  BaseParticle::_GlobalDamping_ = prm->global_damping;
  return h;
}

void refh_destroy(void* hp) { delete static_cast<Harness*>(hp); }

// calculateParticleProperties(density) for circles/ellipses/segments
// (CircularParticle.cpp:16-23, EllipticParticle.cpp:7-14,
// SegmentObject.cpp:4-10); a segment of radius r spans (-r, 0)..(r, 0).
void refh_particle_properties(int32_t n, const int32_t* shape, const double* radius,
                              const double* aspect, double density, double* volume,
                              double* mass, double* inv_mass, double* inertia,
                              double* inv_inertia) {
  ContactModel m;
  for (int i = 0; i < n; ++i) {
    std::unique_ptr<BaseParticle> p;
    if (shape[i] == XDEM_SHAPE_SEGMENT)
      p.reset(new SegmentObject(i, vector2d(-radius[i], 0.0), vector2d(radius[i], 0.0),
                                vector2d(0.0, 0.0), 0.0, &m));
    else
      p = make_particle(shape[i], 0, i, radius[i], aspect[i], 0, 0, 0, 0, 0, 0, &m);
    p->calculateParticleProperties(density);
    volume[i] = p->_volume;
    mass[i] = p->_mass;
    inv_mass[i] = p->_invMass;
    inertia[i] = p->_inertia;
    inv_inertia[i] = p->_invInertia;
  }
}

// GluedParticle::calculateParticleProperties (GluedParticle.cpp:7-80) for one
// clump with nsub sub-particles (circles or ellipses).  Outputs the clump's
// centre, volume, mass, inertia and every sub's branch vector; the subs take
// the clump's mass and inertia (GluedParticle.cpp:73-74).
void refh_clump_properties(int32_t nsub, const int32_t* sub_shape, const double* sub_radius,
                           const double* sub_aspect, const double* sub_x, const double* sub_y,
                           const double* sub_rot, double density, double* out_clump /*7*/,
                           double* branch_x, double* branch_y) {
  ContactModel m;
  std::vector<std::unique_ptr<BaseParticle>> subs;
  GluedParticle g(0, vector2d(0, 0), 0.0);
  for (int k = 0; k < nsub; ++k) {
    subs.push_back(make_particle(sub_shape[k], 0, k + 1, sub_radius[k], sub_aspect[k], sub_x[k],
                                 sub_y[k], 0, 0, sub_rot[k], 0, &m));
    subs.back()->calculateParticleProperties(density);
    g.pushBackSubParticle(subs.back().get());
  }
  g.calculateParticleProperties(density);
  out_clump[0] = g._position.x();
  out_clump[1] = g._position.y();
  out_clump[2] = g._volume;
  out_clump[3] = g._mass;
  out_clump[4] = g._invMass;
  out_clump[5] = g._inertia;
  out_clump[6] = g._invInertia;
  for (int k = 0; k < nsub; ++k) {
    branch_x[k] = g._branchVectors[k].x();
    branch_y[k] = g._branchVectors[k].y();
  }
}

// Build the particle objects and the world (BaseWorld ctor, BaseWorld.h:44-56).
int32_t refh_set_particles(void* hp, const xdem_particles* P) {
  Harness* h = static_cast<Harness*>(hp);
  h->owned.clear();
  h->handlers.clear();
  ContactModel* m = h->model.get();
  for (int i = 0; i < P->n; ++i) {
    std::unique_ptr<BaseParticle> p;
    if (P->shape[i] == XDEM_SHAPE_SEGMENT) {
      // the wall constructor derives position, radii, rotation and direction
      // from the vertices (SegmentObject.h:24-40)
      if (!P->seg_x1 || !P->seg_y1 || !P->seg_x2 || !P->seg_y2) return XDEM_ERR_ARGUMENT;
      p.reset(new SegmentObject(i, vector2d(P->seg_x1[i], P->seg_y1[i]),
                                vector2d(P->seg_x2[i], P->seg_y2[i]),
                                vector2d(P->vx[i], P->vy[i]), P->rot_vel[i], m));
    } else {
      p = make_particle(P->shape[i], h->prm.ellipse_method, i, P->radius[i], P->aspect_ratio[i],
                        P->x[i], P->y[i], P->vx[i], P->vy[i], P->rot[i], P->rot_vel[i], m);
    }
    p->_upLevel = P->up_level[i];
    p->_setting = static_cast<SETTING>(P->setting[i]);
    p->_outerRadius = P->outer_radius[i];
    p->_volume = P->volume[i];
    p->_mass = P->mass[i];
    p->_invMass = P->inv_mass[i];
    p->_inertia = P->inertia[i];
    p->_invInertia = P->inv_inertia[i];
    p->_isRattler = P->is_rattler ? (P->is_rattler[i] != 0) : false;
    h->handlers.push_back(p.get());
    h->owned.push_back(std::move(p));
  }
  // clumps: attach sub-particles and branch vectors
  if (P->num_sub) {
    for (int i = 0; i < P->n; ++i) {
      if (P->shape[i] != XDEM_SHAPE_CLUMP) continue;
      GluedParticle* g = static_cast<GluedParticle*>(h->handlers[i]);
      for (int k = 1; k <= P->num_sub[i]; ++k) {
        g->pushBackSubParticle(h->handlers[i + k]);
        g->_branchVectors.push_back(vector2d(P->branch_x[i + k], P->branch_y[i + k]));
      }
    }
  }
  switch (h->kind) {
    case XDEM_WORLD_PERIODIC:
      h->world.reset(new PeriodicBoundaryWorld(h->prm.dt, h->handlers, m));
      break;
    case XDEM_WORLD_PERIODIC_CONTROL:
      h->world.reset(new PeriodicControlWorld(h->prm.dt, h->handlers, m));
      break;
    case XDEM_WORLD_LEES_EDWARDS:
      h->world.reset(new LeesEdwardsBoundaryWorld(h->prm.dt, h->handlers, m));
      break;
    default:
      return XDEM_ERR_ARGUMENT;
  }
  h->world->set_OMP_NumThreadsAndSizeChunk(h->threads, 100);
  h->world->setWorldBoundary(h->prm.xmin, h->prm.xmax, h->prm.ymin, h->prm.ymax);
  if (h->prm.max_particle_size > 0) h->world->_maxParticleSize = h->prm.max_particle_size;
  if (h->kind == XDEM_WORLD_LEES_EDWARDS) h->le()->setShiftStrainRate(h->prm.shift_strain_rate);
  // collectForceAndTorque has not run yet: empty force arrays, like a fresh world
  h->world->_totalForce.assign(P->n, vector2d(0.0, 0.0));
  h->world->_totalTorque.assign(P->n, 0.0);
  h->world->_numContactPerParticle.assign(P->n, 0);
  return XDEM_OK;
}

void refh_set_threads(void* hp, int32_t threads) {
  Harness* h = static_cast<Harness*>(hp);
  h->threads = threads;
  if (h->world) h->world->set_OMP_NumThreadsAndSizeChunk(threads, 100);
}

int32_t refh_get_particles(void* hp, xdem_particles* P) {
  Harness* h = static_cast<Harness*>(hp);
  int n = static_cast<int>(h->handlers.size());
  P->n = n;
  for (int i = 0; i < n; ++i) {
    BaseParticle* p = h->handlers[i];
    if (P->x) P->x[i] = p->_position.x();
    if (P->y) P->y[i] = p->_position.y();
    if (P->vx) P->vx[i] = p->_velocity.x();
    if (P->vy) P->vy[i] = p->_velocity.y();
    if (P->rot) P->rot[i] = p->_rotation;
    if (P->rot_vel) P->rot_vel[i] = p->_rotationVel;
    if (P->is_rattler) P->is_rattler[i] = p->_isRattler ? 1 : 0;
    if (P->mass) P->mass[i] = p->_mass;
    if (P->inertia) P->inertia[i] = p->_inertia;
    if (P->branch_x || P->branch_y) {
      if (P->branch_x) P->branch_x[i] = 0.0;
      if (P->branch_y) P->branch_y[i] = 0.0;
    }
    if (SegmentObject* s = dynamic_cast<SegmentObject*>(p)) {
      if (P->seg_x1) P->seg_x1[i] = s->_vertex1.x();
      if (P->seg_y1) P->seg_y1[i] = s->_vertex1.y();
      if (P->seg_x2) P->seg_x2[i] = s->_vertex2.x();
      if (P->seg_y2) P->seg_y2[i] = s->_vertex2.y();
    }
  }
  if (P->branch_x || P->branch_y) {
    for (int i = 0; i < n; ++i) {
      if (GluedParticle* g = dynamic_cast<GluedParticle*>(h->handlers[i])) {
        for (size_t k = 0; k < g->_branchVectors.size(); ++k) {
          if (P->branch_x) P->branch_x[i + 1 + k] = g->_branchVectors[k].x();
          if (P->branch_y) P->branch_y[i + 1 + k] = g->_branchVectors[k].y();
        }
      }
    }
  }
  return XDEM_OK;
}

int32_t refh_set_contacts(void* hp, const xdem_contacts* C) {
  Harness* h = static_cast<Harness*>(hp);
  for (auto* p : h->handlers) p->_contactInfo.clear();
  for (int64_t k = 0; k < C->count; ++k) {
    ContactInformation ci;
    ci._otherID = C->id_j[k];
    ci._contactNormal = vector2d(C->normal_x[k], C->normal_y[k]);
    ci._contactPoint = vector2d(C->point_x[k], C->point_y[k]);
    ci._branchVector = vector2d(C->branch_x[k], C->branch_y[k]);
    ci._branchVectorFromP1 = vector2d(C->bv1_x[k], C->bv1_y[k]);
    ci._branchVectorFromP2 = vector2d(C->bv2_x[k], C->bv2_y[k]);
    ci._shearOverlap = vector2d(C->shear_x[k], C->shear_y[k]);
    ci._normalForce = vector2d(C->fn_x[k], C->fn_y[k]);
    ci._shearForce = vector2d(C->ft_x[k], C->ft_y[k]);
    ci._force = ci._normalForce + ci._shearForce;
    ci._forceOnP1 = ci._force;
    ci._forceOnP2 = -ci._force;
    ci._torqueOnP1 = C->torque_i[k];
    ci._torqueOnP2 = C->torque_j[k];
    ci._dampingConstant = C->damping[k];
    h->handlers[C->id_i[k]]->_contactInfo.emplace(C->id_j[k], ci);
  }
  return XDEM_OK;
}

int32_t refh_get_contacts(void* hp, xdem_contacts* C) {
  Harness* h = static_cast<Harness*>(hp);
  int64_t total = 0;
  for (auto* p : h->handlers) total += static_cast<int64_t>(p->_contactInfo.size());
  C->count = total;
  if (C->capacity < total) return XDEM_ERR_CAPACITY;
  int64_t k = 0;
  for (auto* p : h->handlers) {
    std::vector<int> keys;
    for (auto& it : p->_contactInfo) keys.push_back(it.first);
    std::sort(keys.begin(), keys.end());
    for (int j : keys) {
      const ContactInformation& ci = p->_contactInfo.at(j);
      C->id_i[k] = p->_id;
      C->id_j[k] = j;
      C->normal_x[k] = ci._contactNormal.x();
      C->normal_y[k] = ci._contactNormal.y();
      C->point_x[k] = ci._contactPoint.x();
      C->point_y[k] = ci._contactPoint.y();
      C->branch_x[k] = ci._branchVector.x();
      C->branch_y[k] = ci._branchVector.y();
      C->bv1_x[k] = ci._branchVectorFromP1.x();
      C->bv1_y[k] = ci._branchVectorFromP1.y();
      C->bv2_x[k] = ci._branchVectorFromP2.x();
      C->bv2_y[k] = ci._branchVectorFromP2.y();
      C->shear_x[k] = ci._shearOverlap.x();
      C->shear_y[k] = ci._shearOverlap.y();
      C->fn_x[k] = ci._normalForce.x();
      C->fn_y[k] = ci._normalForce.y();
      C->ft_x[k] = ci._shearForce.x();
      C->ft_y[k] = ci._shearForce.y();
      C->torque_i[k] = ci._torqueOnP1;
      C->torque_j[k] = ci._torqueOnP2;
      C->damping[k] = ci._dampingConstant;
      ++k;
    }
  }
  return XDEM_OK;
}

int32_t refh_get_force_and_torque(void* hp, double* fx, double* fy, double* t, int32_t* nc) {
  Harness* h = static_cast<Harness*>(hp);
  BaseWorld* w = h->world.get();
  for (size_t i = 0; i < h->handlers.size(); ++i) {
    fx[i] = w->_totalForce[i].x();
    fy[i] = w->_totalForce[i].y();
    t[i] = w->_totalTorque[i];
    if (nc) nc[i] = w->_numContactPerParticle.empty() ? 0 : w->_numContactPerParticle[i];
  }
  return XDEM_OK;
}

void refh_get_boundary(void* hp, double* box) {
  BaseWorld* w = static_cast<Harness*>(hp)->world.get();
  box[0] = w->_xmin;
  box[1] = w->_xmax;
  box[2] = w->_ymin;
  box[3] = w->_ymax;
}

void refh_get_stress(void* hp, double* s) {
  matrix2d m = static_cast<Harness*>(hp)->world->getStress();
  s[0] = m.xx();
  s[1] = m.xy();
  s[2] = m.yx();
  s[3] = m.yy();
}

void refh_get_lees_edwards(void* hp, double* out) {
  Harness* h = static_cast<Harness*>(hp);
  if (h->kind != XDEM_WORLD_LEES_EDWARDS) {
    out[0] = out[1] = out[2] = out[3] = 0.0;
    return;
  }
  LeesEdwardsBoundaryWorld* w = h->le();
  out[0] = w->_totalShift;
  out[1] = w->_shiftVel;
  out[2] = w->_totalStrain;
  out[3] = w->_shiftStrainRate;
}

void refh_set_lees_edwards(void* hp, const double* in) {
  Harness* h = static_cast<Harness*>(hp);
  if (h->kind != XDEM_WORLD_LEES_EDWARDS) return;
  LeesEdwardsBoundaryWorld* w = h->le();
  w->_totalShift = in[0];
  w->_shiftVel = in[1];
  w->_totalStrain = in[2];
  w->_shiftStrainRate = in[3];
}

void refh_set_virtual_boundary_mass(void* hp, double mass) {
  Harness* h = static_cast<Harness*>(hp);
  if (mass < 0) h->control()->setVirtualBoundaryMass();
  else h->control()->setVirtualBoundaryMass(mass);
}

void refh_set_max_strain_rate(void* hp, double r) {
  static_cast<Harness*>(hp)->control()->setMaxStrainRate(r);
}

double refh_get_control_mass(void* hp) { return static_cast<Harness*>(hp)->control()->_mass; }

double refh_kinetic_energy(void* hp) { return static_cast<Harness*>(hp)->world->getKineticEnergy(); }

int64_t refh_count_contacts(void* hp) {
  return static_cast<Harness*>(hp)->world->countActucalContacts();
}

// Sub-step dispatcher: one reference method per code.
enum {
  RH_MODIFY = 0, RH_APPLY_BG = 1, RH_REMOVE_BG = 2, RH_FIND = 3, RH_UPDATE = 4, RH_COLLECT = 5,
  RH_INTEGRATE = 6, RH_RESET_RATTLERS = 7, RH_SCALE_RATTLERS = 8, RH_STRESS = 9,
  RH_BOX_LAW = 10, RH_LE_BOUNDARY = 11, RH_TAKE_STEP = 12, RH_SCALE_TO_FRACTION = 13
};

static void box_law(Harness* h, int law, double p0, double p1) {
  PeriodicControlWorld* c = h->control();
  switch (law) {
    case XDEM_BOX_STRAIN: c->updatePeriodicBoundary_strainControl(p0, p1); break;
    case XDEM_BOX_STRESS_XY:
      c->updatePeriodicBoundary_stressControlX(p0);
      c->updatePeriodicBoundary_stressControlY(p0);
      break;
    case XDEM_BOX_STRESS_UNIFORM: c->updatePeriodicBoundary_stressControlUniform(p0); break;
    case XDEM_BOX_STRESS_UNIFORM_LIMIT:
      c->updatePeriodicBoundary_stressControlUniform_strainLimit(p0);
      break;
    default: break;
  }
}

int32_t refh_call(void* hp, int32_t which, double a, double b, double c) {
  Harness* h = static_cast<Harness*>(hp);
  BaseWorld* w = h->world.get();
  switch (which) {
    case RH_MODIFY: w->modifyParticlePosition(); break;
    case RH_APPLY_BG: h->le()->applyBackgroudVelocity(); break;
    case RH_REMOVE_BG: h->le()->removeBackgroudVelocity(); break;
    case RH_FIND: w->findPossibleContacts(); break;
    case RH_UPDATE: w->updateContacts(); break;
    case RH_COLLECT: w->collectForceAndTorque(); break;
    case RH_INTEGRATE: w->takeTimeIntegral(); break;
    case RH_RESET_RATTLERS: w->resetVelocityOfRattlers(); break;
    case RH_SCALE_RATTLERS: w->scaleVelocityOfRattlers(a); break;
    case RH_STRESS: w->updateTotalStress(); break;
    case RH_BOX_LAW: box_law(h, static_cast<int>(a), b, c); break;
    case RH_LE_BOUNDARY: h->le()->updateLeesEdwardBoundary(); break;
    case RH_TAKE_STEP: w->takeTimeStep(); break;
    case RH_SCALE_TO_FRACTION: h->periodic()->scaleBoundarySizeToGivenSolidFraction(a); break;
    default: return XDEM_ERR_ARGUMENT;
  }
  return XDEM_OK;
}

// The driver loops of xdem_run, built from the reference's own methods.
int32_t refh_run(void* hp, int32_t nsteps, const xdem_control* ctl, int32_t* steps_done) {
  Harness* h = static_cast<Harness*>(hp);
  BaseWorld* w = h->world.get();
  int s = 0;
  for (; s < nsteps; ++s) {
    if (ctl->scale_rattlers) w->scaleVelocityOfRattlers(ctl->rattler_scale);
    if (ctl->sequence == XDEM_SEQ_SUBSTEPS) {
      w->modifyParticlePosition();
      w->findPossibleContacts();
      w->updateContacts();
      w->collectForceAndTorque();
      w->takeTimeIntegral();
    } else {
      w->takeTimeStep();
    }
    if (ctl->reset_rattlers) w->resetVelocityOfRattlers();
    if (ctl->update_stress) w->updateTotalStress();
    if (ctl->box_law != XDEM_BOX_NONE) box_law(h, ctl->box_law, ctl->p0, ctl->p1);
    if (ctl->stop_on_pressure && w->getStress().trace() / 2.0 >= ctl->stop_pressure) {
      ++s;
      break;
    }
  }
  if (steps_done) *steps_done = s;
  return XDEM_OK;
}

// One pair through BaseParticle::calculateContactGeometry (virtual dispatch as
// in BaseParticle.cpp:29).  Row layouts as xdem_pair_geometry.
int32_t refh_pair_geometry(int32_t npairs, int32_t method, const double* pi, const double* pj,
                           const double* off, double* out) {
  ContactModel m;
  for (int k = 0; k < npairs; ++k) {
    const double* a = pi + 9 * k;
    const double* b = pj + 9 * k;
    auto p1 = make_particle(static_cast<int>(a[0]), method, 0, a[1], a[2], a[3], a[4], a[5],
                            a[6], a[7], a[8], &m);
    auto p2 = make_particle(static_cast<int>(b[0]), method, 1, b[1], b[2], b[3], b[4], b[5],
                            b[6], b[7], b[8], &m);
    ContactGeometry cg;
    bool c = p1->calculateContactGeometry(p2.get(), cg, vector2d(off[4 * k], off[4 * k + 1]),
                                          vector2d(off[4 * k + 2], off[4 * k + 3]));
    double* o = out + 17 * k;
    o[0] = c ? 1.0 : 0.0;
    o[1] = cg.contactNormal.x();
    o[2] = cg.contactNormal.y();
    o[3] = cg.contactPoint.x();
    o[4] = cg.contactPoint.y();
    o[5] = cg.branchVectorFromP1.x();
    o[6] = cg.branchVectorFromP1.y();
    o[7] = cg.branchVectorFromP2.x();
    o[8] = cg.branchVectorFromP2.y();
    o[9] = cg.normalOverlap;
    o[10] = cg.relVel.x();
    o[11] = cg.relVel.y();
    o[12] = cg.normalRelVel.x();
    o[13] = cg.normalRelVel.y();
    o[14] = cg.shearRelVel.x();
    o[15] = cg.shearRelVel.y();
    o[16] = -1.0;
  }
  return XDEM_OK;
}

// QuadronAnalysis rattler-free coordination number and solid fraction
// (QuadronAnalysis.cpp:360-386 constructor, :663-668 inactivateRattlerParticles,
// :980-986 removeOpenChainParticles, :703-713, :724-732).
void refh_quadron_z_phi(void* hp, double* out) {
  Harness* h = static_cast<Harness*>(hp);
  BaseWorld* w = h->world.get();
  QuadronSystem::setPeriodicBoundarySize(w->_xmin, w->_xmax, w->_ymin, w->_ymax);
  QuadronSystem::QuadronAnalysis qa(h->handlers);
  qa.inactivateRattlerParticles();
  qa.removeOpenChainParticles();
  out[0] = qa.calculateMeanCoordinationNumber();
  out[1] = qa.calculateRattlerFreeSolidFraction();
}

}  // extern "C"
