// xdem_gpu_world.hpp — drop-in GPU worlds for drivers written against the
// reference's C++ classes.
//
//   GpuPeriodicBoundaryWorld    : PeriodicBoundaryWorld     (PeriodicBoundaryWorld.h:8)
//   GpuPeriodicControlWorld     : PeriodicControlWorld      (PeriodicControlWorld.h:5)
//   GpuLeesEdwardsBoundaryWorld : LeesEdwardsBoundaryWorld  (LeesEdwardsBoundaryWorld.h:5)
//
// Each takes the reference constructor's arguments (dt, vector<BaseParticle*>,
// ContactModel*; BaseWorld.h:44-56) and keeps the reference interface: the
// virtual step methods (BaseWorld.h:59-71) are overridden, and the
// non-virtual ones a driver calls on the concrete type
// (collectForceAndTorque, takeTimeIntegral, updateTotalStress, the box laws,
// ...; BaseWorld.h:62-63,95,105, PeriodicControlWorld.h:28-36,
// LeesEdwardsBoundaryWorld.h:31-45) are hidden by same-named members that run
// on the GPU through the C-ABI of xdem_gpu.h.  A driver such as
// mainIsoCircPack_WCCM.cpp:115-126 compiles unchanged when its world's type
// names the Gpu class instead.
//
// Where the state lives.  The particle objects the driver owns stay the
// reference's record.  The first GPU call uploads them (positions,
// velocities, shapes, masses, settings, clump branch vectors, segment
// vertices and every particle's contact map) together with the world's
// scalars (box, time step, contact model, global damping, control and
// Lees-Edwards state).  With host sync on (the default) every GPU call then
// writes the results back into the particle objects and the world's members:
// state, rattler flags, contact maps, the clump branch vectors,
// _totalForce/_totalTorque/_numContactPerParticle, _totalStress, the box and
// the Lees-Edwards scalars, so getters and file output behave as with the
// reference world.  For long runs, setHostSync(false) and pull() before the
// host reads, or run(n) for n graph-captured steps.  After the driver changes
// particles or contacts on the host, push() uploads them again.
//
// Requirements: the reference's headers on the include path, ids equal to
// vector indices (as the reference itself requires, BaseWorld.cpp:72-74),
// clump sub-particles following their clump's id.  Errors that make the
// reference print and exit() (a 200-candidate overflow, an unsupported shape
// pair) make these classes print the status and exit() the same way; a
// closest-approach Newton iteration that would never end in the reference is
// reported once on stderr and the run goes on (xdem_gpu.h, XDEM_ERR_NEWTON).
//
// The reference keeps some of what must be mirrored out of public reach: a
// particle's contact map and rattler flag (protected, BaseParticle.h:33,46),
// a clump's sub-particles and branch vectors (protected, GluedParticle.h:8-9)
// and the contact model's constants (private,
// ContactModel_LinearDissipativeFrictional.h:44-47).  They are read and
// written here through pointers to members, formed in a derived class for the
// protected ones and in an explicit template instantiation (where access is
// not checked) for the private ones; the reference's headers need no edits.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <unordered_map>
#include <vector>

#include "CircularParticle.h"
#include "EllipticParticle.h"
#include "GluedParticle.h"
#include "LeesEdwardsBoundaryWorld.h"
#include "PeriodicBoundaryWorld.h"
#include "PeriodicControlWorld.h"
#include "SegmentObject.h"
#include "xdem_gpu.h"

namespace xdem_gpu {

// ---- access to the members the reference does not expose ------------------
struct ParticleAccess : BaseParticle {
  static std::unordered_map<int, ContactInformation>& contacts(BaseParticle* p) {
    return p->*(&ParticleAccess::_contactInfo);
  }
  static bool& rattler(BaseParticle* p) { return p->*(&ParticleAccess::_isRattler); }
};

struct GluedAccess : GluedParticle {
  static std::vector<BaseParticle*>& subs(GluedParticle* g) {
    return g->*(&GluedAccess::_subParticles);
  }
  static std::vector<vector2d>& branches(GluedParticle* g) {
    return g->*(&GluedAccess::_branchVectors);
  }
};

template <class Tag, typename Tag::type M>
struct MemberOf {
  friend typename Tag::type member_of(Tag) { return M; }
};
struct ShearStiffnessTag {
  typedef double ContactModel::*type;
  friend type member_of(ShearStiffnessTag);
};
struct RestitutionTag {
  typedef double ContactModel::*type;
  friend type member_of(RestitutionTag);
};
struct FrictionTag {
  typedef double ContactModel::*type;
  friend type member_of(FrictionTag);
};
template struct MemberOf<ShearStiffnessTag, &ContactModel::_shearStiffness>;
template struct MemberOf<RestitutionTag, &ContactModel::_restitutionCoeff>;
template struct MemberOf<FrictionTag, &ContactModel::_frictionalCoeff>;

// prints the first set status bit and exits, as the reference does on errors
inline void fail(int32_t st, const char* where) {
  for (int b = 0; b < 31; ++b)
    if (st & (1 << b)) {
      std::printf("[xdem_gpu] %s: %s\n", where, xdem_status_string(1 << b));
      break;
    }
  std::exit(-1);
}

// ---- the world template ----------------------------------------------------
template <class Base, int Kind>
class GpuWorld : public Base {
 public:
  GpuWorld(const double& dt, const std::vector<BaseParticle*> particleHandlers,
           ContactModel* contactModelHandler)
      : Base(dt, particleHandlers, contactModelHandler) {}
  GpuWorld(const GpuWorld&) = delete;
  GpuWorld& operator=(const GpuWorld&) = delete;
  ~GpuWorld() {
    if (h_) xdem_destroy(h_);
  }

  // ---- synchronisation ----------------------------------------------------
  // true (default): every GPU call writes its results back to the host
  void setHostSync(bool on) { host_sync_ = on; }
  // Closest-approach (the reference's dispatch, EllipticParticle.cpp:27) or
  // XDEM_ELLIPSE_INTERSECTION; FP64 or XDEM_PRECISION_MIXED.  Before the
  // first GPU call.
  void setEllipseMethod(int32_t method) { method_ = method; }
  void setPrecision(int32_t precision) { precision_ = precision; }
  xdem_world handle() {
    ensure();
    return h_;
  }

  // host particle objects and world scalars -> device
  void push() {
    if (!h_) {
      ensure();
      return;
    }
    upload_particles();
    upload_scalars();
  }

  // device -> host particle objects and world members
  void pull() {
    if (!h_) return;
    pull_scalars();
    pull_particles();
  }

  // n steps of the world's own takeTimeStep, captured in CUDA graphs
  // (xdem_run); the host copy is refreshed once at the end
  void run(int nsteps) {
    ensure();
    xdem_control ctl{};
    ctl.sequence = XDEM_SEQ_TAKE_TIME_STEP;
    int32_t done = 0;
    check(xdem_run(h_, nsteps, &ctl, &done), "run");
    after();
  }

  // ---- the virtual step methods (BaseWorld.h:59-71) ------------------------
  void takeTimeStep() override {
    ensure();
    check(xdem_take_time_step(h_), "takeTimeStep");
    after();
  }
  void modifyParticlePosition() override {
    ensure();
    check(xdem_modify_particle_position(h_), "modifyParticlePosition");
    after();
  }
  void findPossibleContacts() override {
    ensure();
    check(xdem_find_possible_contacts(h_), "findPossibleContacts");
    after();
  }
  void updateContacts() override {
    ensure();
    check(xdem_update_contacts(h_), "updateContacts");
    after();
  }

  // ---- non-virtual methods, hidden (BaseWorld.h) ----------------------------
  void collectForceAndTorque() {
    ensure();
    check(xdem_collect_force_and_torque(h_), "collectForceAndTorque");
    after();
  }
  void takeTimeIntegral() {
    ensure();
    check(xdem_take_time_integral(h_), "takeTimeIntegral");
    after();
  }
  void resetVelocityOfRattlers() {
    ensure();
    check(xdem_reset_velocity_of_rattlers(h_), "resetVelocityOfRattlers");
    after();
  }
  void scaleVelocityOfRattlers(const double scale) {
    ensure();
    check(xdem_scale_velocity_of_rattlers(h_, scale), "scaleVelocityOfRattlers");
    after();
  }
  const matrix2d updateTotalStress() {
    ensure();
    double s[4];
    check(xdem_update_total_stress(h_, s), "updateTotalStress");
    after();
    return this->_totalStress;
  }
  void setTimeIncrement(const double& dt) {
    Base::setTimeIncrement(dt);
    if (h_) check(xdem_set_time_increment(h_, dt), "setTimeIncrement");
  }
  void setWorldBoundary(const double& xmin, const double& xmax, const double& ymin,
                        const double& ymax) {
    Base::setWorldBoundary(xmin, xmax, ymin, ymax);
    if (h_) {
      const double box[4] = {xmin, xmax, ymin, ymax};
      check(xdem_set_boundary(h_, box), "setWorldBoundary");
    }
  }
  const int countActucalContacts() {
    ensure();
    int64_t n = 0;
    check(xdem_count_contacts(h_, &n), "countActucalContacts");
    return static_cast<int>(n);
  }
  const double getKineticEnergy() {
    ensure();
    double e = 0.0;
    check(xdem_get_kinetic_energy(h_, &e), "getKineticEnergy");
    return e;
  }
  // PeriodicBoundaryWorld.cpp:276-284
  void scaleBoundarySizeToGivenSolidFraction(const double& initSolidFrac) {
    ensure();
    check(xdem_scale_boundary_to_solid_fraction(h_, initSolidFrac),
          "scaleBoundarySizeToGivenSolidFraction");
    after();
  }

  // ---- PeriodicControlWorld (PeriodicControlWorld.h:28-36) -------------------
  void setVirtualBoundaryMass() {
    Base::setVirtualBoundaryMass();
    if (h_) check(xdem_set_virtual_boundary_mass(h_, this->_mass), "setVirtualBoundaryMass");
  }
  void setVirtualBoundaryMass(const double& mass) {
    Base::setVirtualBoundaryMass(mass);
    if (h_) check(xdem_set_virtual_boundary_mass(h_, mass), "setVirtualBoundaryMass");
  }
  void setMaxStrainRate(const double maxStrainRate) {
    Base::setMaxStrainRate(maxStrainRate);
    if (h_) check(xdem_set_max_strain_rate(h_, maxStrainRate), "setMaxStrainRate");
  }
  void updatePeriodicBoundary_strainControl(const double& strainRateX, const double& strainRateY) {
    box_law(XDEM_BOX_STRAIN, strainRateX, strainRateY, "updatePeriodicBoundary_strainControl");
  }
  void updatePeriodicBoundary_stressControlUniform(const double& stress) {
    box_law(XDEM_BOX_STRESS_UNIFORM, stress, 0.0, "updatePeriodicBoundary_stressControlUniform");
  }
  void updatePeriodicBoundary_stressControlUniform_strainLimit(const double& stress) {
    box_law(XDEM_BOX_STRESS_UNIFORM_LIMIT, stress, 0.0,
            "updatePeriodicBoundary_stressControlUniform_strainLimit");
  }
  // stressControlX followed by stressControlY with the same stress, as
  // drivers call them, is one XDEM_BOX_STRESS_XY law on the device; the X
  // call is held until the Y call arrives
  void updatePeriodicBoundary_stressControlX(const double& stress) {
    pending_x_ = true;
    pending_stress_ = stress;
  }
  void updatePeriodicBoundary_stressControlY(const double& stress) {
    if (!pending_x_ || pending_stress_ != stress) {
      std::printf("[xdem_gpu] stressControlY without a matching stressControlX\n");
      std::exit(-1);
    }
    pending_x_ = false;
    box_law(XDEM_BOX_STRESS_XY, stress, 0.0, "updatePeriodicBoundary_stressControlXY");
  }

  // ---- LeesEdwardsBoundaryWorld (LeesEdwardsBoundaryWorld.h:31-45) ------------
  void updateLeesEdwardBoundary() {
    ensure();
    check(xdem_update_lees_edwards_boundary(h_), "updateLeesEdwardBoundary");
    after();
  }
  void applyBackgroudVelocity() {
    ensure();
    check(xdem_apply_background_velocity(h_), "applyBackgroudVelocity");
    after();
  }
  void removeBackgroudVelocity() {
    ensure();
    check(xdem_remove_background_velocity(h_), "removeBackgroudVelocity");
    after();
  }
  void setShiftStrainRate(const double& shiftStrainRate) {
    Base::setShiftStrainRate(shiftStrainRate);
    if (h_) check(xdem_set_shift_strain_rate(h_, shiftStrainRate), "setShiftStrainRate");
  }

 private:
  void check(int32_t st, const char* where) {
    if (st & XDEM_ERR_NEWTON) {
      if (!newton_reported_)
        std::fprintf(stderr, "[xdem_gpu] %s: %s (reported once)\n", where,
                     xdem_status_string(XDEM_ERR_NEWTON));
      newton_reported_ = true;
      st &= ~XDEM_ERR_NEWTON;
    }
    if (st) fail(st, where);
  }

  void after() {
    if (host_sync_) pull();
  }

  void box_law(int32_t law, double p0, double p1, const char* where) {
    static_assert(Kind != XDEM_WORLD_PERIODIC, "box laws belong to PeriodicControlWorld");
    ensure();
    check(xdem_update_boundary(h_, law, p0, p1), where);
    after();
  }

  // the contact model's constants and the global damping, which drivers
  // change between phases (mainIsoCircPack_WCCM.cpp:104-108)
  void model_constants(double c[5]) const {
    ContactModel* m = this->_contactModelHandler;
    c[0] = m->getNormalStiffness();
    c[1] = m->*member_of(ShearStiffnessTag());
    c[2] = m->*member_of(RestitutionTag());
    c[3] = m->*member_of(FrictionTag());
    c[4] = BaseParticle::_GlobalDamping_;
  }

  // the world on the device, created at the first GPU call from the host
  // state; later calls re-send the contact model and global damping when the
  // driver has changed them
  void ensure() {
    if (h_) {
      double c[5];
      model_constants(c);
      if (c[0] != consts_[0] || c[1] != consts_[1] || c[2] != consts_[2] || c[3] != consts_[3])
        check(xdem_set_contact_model(h_, c[0], c[1], c[2], c[3]), "setContactModel");
      if (c[4] != consts_[4]) check(xdem_set_global_damping(h_, c[4]), "setGlobalDamping");
      for (int k = 0; k < 5; ++k) consts_[k] = c[k];
      return;
    }
    model_constants(consts_);
    xdem_params prm{};
    prm.world_kind = Kind;
    prm.ellipse_method = method_;
    prm.precision = precision_;
    prm.dt = this->_dt;
    prm.xmin = this->_xmin;
    prm.xmax = this->_xmax;
    prm.ymin = this->_ymin;
    prm.ymax = this->_ymax;
    prm.normal_stiffness = consts_[0];
    prm.shear_stiffness = consts_[1];
    prm.restitution_coeff = consts_[2];
    prm.frictional_coeff = consts_[3];
    prm.global_damping = consts_[4];
    check(xdem_create(&prm, &h_), "xdem_create");
    upload_particles();
    upload_scalars();
  }

  void upload_scalars() {
    if constexpr (Kind != XDEM_WORLD_PERIODIC) {
      check(xdem_set_virtual_boundary_mass(h_, this->_mass), "setVirtualBoundaryMass");
      check(xdem_set_max_strain_rate(h_, this->_maxStrainRate), "setMaxStrainRate");
    }
    if constexpr (Kind == XDEM_WORLD_LEES_EDWARDS) {
      const double le[4] = {this->_totalShift, this->_shiftVel, this->_totalStrain,
                            this->_shiftStrainRate};
      check(xdem_set_lees_edwards(h_, le), "setLeesEdwards");
    }
  }

  void upload_particles() {
    const std::vector<BaseParticle*>& ps = this->_particleHandlers;
    const int n = static_cast<int>(ps.size());
    std::vector<int32_t> shape(n), up(n), setting(n), rattler(n), nsub(n, 0);
    std::vector<double> orad(n), rad(n), asp(n), x(n), y(n), vx(n), vy(n), rot(n), w(n),
        vol(n), mass(n), im(n), I(n), iI(n), bx(n, 0.0), by(n, 0.0), s1x(n, 0.0), s1y(n, 0.0),
        s2x(n, 0.0), s2y(n, 0.0);
    bool any_seg = false;
    for (int i = 0; i < n; ++i) {
      BaseParticle* p = ps[i];
      if (p->getID() != i) {
        std::printf("[xdem_gpu] particle %d has id %d: ids must equal indices\n", i, p->getID());
        std::exit(-1);
      }
      up[i] = p->getUpLevel();
      setting[i] = static_cast<int32_t>(p->getSettings());
      rattler[i] = ParticleAccess::rattler(p) ? 1 : 0;
      orad[i] = p->getOuterRadius();
      x[i] = p->getPosX();
      y[i] = p->getPosY();
      vx[i] = p->getVelX();
      vy[i] = p->getVelY();
      rot[i] = p->getRot();
      w[i] = p->getRotVel();
      vol[i] = p->getVolume();
      mass[i] = p->getMass();
      im[i] = p->getInvMass();
      I[i] = p->getInertia();
      iI[i] = p->getInvInertia();
      asp[i] = 1.0;
      if (GluedParticle* g = dynamic_cast<GluedParticle*>(p)) {
        shape[i] = XDEM_SHAPE_CLUMP;
        rad[i] = -1.0;
        const std::vector<BaseParticle*>& subs = GluedAccess::subs(g);
        const std::vector<vector2d>& br = GluedAccess::branches(g);
        nsub[i] = static_cast<int32_t>(subs.size());
        for (size_t k = 0; k < subs.size(); ++k) {
          const int sid = subs[k]->getID();
          if (sid != i + 1 + static_cast<int>(k)) {
            std::printf("[xdem_gpu] clump %d: sub-particle ids must follow the clump's\n", i);
            std::exit(-1);
          }
          bx[sid] = br[k].x();
          by[sid] = br[k].y();
        }
      } else if (EllipticParticle* e = dynamic_cast<EllipticParticle*>(p)) {
        shape[i] = XDEM_SHAPE_ELLIPSE;
        rad[i] = e->getRadius();
        asp[i] = e->getAspectRatio();
      } else if (CircularParticle* c = dynamic_cast<CircularParticle*>(p)) {
        shape[i] = XDEM_SHAPE_CIRCLE;
        rad[i] = c->getRadius();
      } else if (SegmentObject* s = dynamic_cast<SegmentObject*>(p)) {
        shape[i] = XDEM_SHAPE_SEGMENT;
        rad[i] = s->getRadius();
        s1x[i] = s->getVertex1().x();
        s1y[i] = s->getVertex1().y();
        s2x[i] = s->getVertex2().x();
        s2y[i] = s->getVertex2().y();
        any_seg = true;
      } else {
        std::printf("[xdem_gpu] particle %d: shape without a GPU contact law\n", i);
        std::exit(-1);
      }
    }
    xdem_particles P{};
    P.n = n;
    P.shape = shape.data();
    P.up_level = up.data();
    P.setting = setting.data();
    P.is_rattler = rattler.data();
    P.outer_radius = orad.data();
    P.radius = rad.data();
    P.aspect_ratio = asp.data();
    P.x = x.data();
    P.y = y.data();
    P.vx = vx.data();
    P.vy = vy.data();
    P.rot = rot.data();
    P.rot_vel = w.data();
    P.volume = vol.data();
    P.mass = mass.data();
    P.inv_mass = im.data();
    P.inertia = I.data();
    P.inv_inertia = iI.data();
    P.num_sub = nsub.data();
    P.branch_x = bx.data();
    P.branch_y = by.data();
    if (any_seg) {
      P.seg_x1 = s1x.data();
      P.seg_y1 = s1y.data();
      P.seg_x2 = s2x.data();
      P.seg_y2 = s2y.data();
    }
    check(xdem_set_particles(h_, &P), "set_particles");
    upload_contacts();
  }

  // every particle's contact map, keyed (owner id, partner id)
  void upload_contacts() {
    const std::vector<BaseParticle*>& ps = this->_particleHandlers;
    std::vector<int32_t> ci, cj;
    std::vector<double> f[19];
    for (size_t i = 0; i < ps.size(); ++i)
      for (const auto& kv : ParticleAccess::contacts(ps[i])) {
        const ContactInformation& c = kv.second;
        ci.push_back(static_cast<int32_t>(i));
        cj.push_back(kv.first);
        const double v[19] = {c._contactNormal.x(),      c._contactNormal.y(),
                              c._contactPoint.x(),       c._contactPoint.y(),
                              c._branchVector.x(),       c._branchVector.y(),
                              c._branchVectorFromP1.x(), c._branchVectorFromP1.y(),
                              c._branchVectorFromP2.x(), c._branchVectorFromP2.y(),
                              c._shearOverlap.x(),       c._shearOverlap.y(),
                              c._normalForce.x(),        c._normalForce.y(),
                              c._shearForce.x(),         c._shearForce.y(),
                              c._torqueOnP1,             c._torqueOnP2,
                              c._dampingConstant};
        for (int k = 0; k < 19; ++k) f[k].push_back(v[k]);
      }
    xdem_contacts C{};
    C.count = static_cast<int64_t>(ci.size());
    C.capacity = C.count;
    C.id_i = ci.data();
    C.id_j = cj.data();
    double** dst[19] = {&C.normal_x, &C.normal_y, &C.point_x, &C.point_y, &C.branch_x,
                        &C.branch_y, &C.bv1_x,    &C.bv1_y,   &C.bv2_x,   &C.bv2_y,
                        &C.shear_x,  &C.shear_y,  &C.fn_x,    &C.fn_y,    &C.ft_x,
                        &C.ft_y,     &C.torque_i, &C.torque_j, &C.damping};
    for (int k = 0; k < 19; ++k) *dst[k] = f[k].data();
    check(xdem_set_contacts(h_, &C), "set_contacts");
  }

  void pull_scalars() {
    double box[4], s[4];
    check(xdem_get_boundary(h_, box), "get_boundary");
    this->_xmin = box[0];
    this->_xmax = box[1];
    this->_ymin = box[2];
    this->_ymax = box[3];
    this->_xlen = box[1] - box[0];
    this->_ylen = box[3] - box[2];
    check(xdem_get_stress(h_, s), "get_stress");
    this->_totalStress = matrix2d(s[0], s[1], s[2], s[3]);
    if constexpr (Kind == XDEM_WORLD_LEES_EDWARDS) {
      double le[4];
      check(xdem_get_lees_edwards(h_, le), "get_lees_edwards");
      this->_totalShift = le[0];
      this->_shiftVel = le[1];
      this->_totalStrain = le[2];
      this->_shiftStrainRate = le[3];
    }
  }

  void pull_particles() {
    const std::vector<BaseParticle*>& ps = this->_particleHandlers;
    const int n = static_cast<int>(ps.size());
    std::vector<int32_t> rattler(n), nc(n);
    std::vector<double> x(n), y(n), vx(n), vy(n), rot(n), w(n), bx(n), by(n), fx(n), fy(n), t(n);
    xdem_particles P{};
    P.n = n;
    P.is_rattler = rattler.data();
    P.x = x.data();
    P.y = y.data();
    P.vx = vx.data();
    P.vy = vy.data();
    P.rot = rot.data();
    P.rot_vel = w.data();
    P.branch_x = bx.data();
    P.branch_y = by.data();
    check(xdem_get_particles(h_, &P), "get_particles");
    check(xdem_get_force_and_torque(h_, fx.data(), fy.data(), t.data(), nc.data()),
          "get_force_and_torque");
    this->_totalForce.resize(n);
    this->_totalTorque.resize(n);
    this->_numContactPerParticle.resize(n);
    for (int i = 0; i < n; ++i) {
      BaseParticle* p = ps[i];
      p->setPos(vector2d(x[i], y[i]));
      p->setVel(vector2d(vx[i], vy[i]));
      p->setRot(rot[i]);
      p->setRotVel(w[i]);
      ParticleAccess::rattler(p) = rattler[i] != 0;
      this->_totalForce[i] = vector2d(fx[i], fy[i]);
      this->_totalTorque[i] = t[i];
      this->_numContactPerParticle[i] = nc[i];
      ParticleAccess::contacts(p).clear();
      if (GluedParticle* g = dynamic_cast<GluedParticle*>(p)) {
        std::vector<vector2d>& br = GluedAccess::branches(g);
        for (size_t k = 0; k < br.size(); ++k) br[k] = vector2d(bx[i + 1 + k], by[i + 1 + k]);
      }
    }
    // the contact maps
    xdem_contacts C{};
    C.capacity = 0;
    int32_t st = xdem_get_contacts(h_, &C);
    if (st && st != XDEM_ERR_CAPACITY) check(st, "get_contacts");
    const int64_t m = C.count;
    std::vector<int32_t> ci(m), cj(m);
    std::vector<double> f[19];
    for (auto& v : f) v.resize(m);
    C.capacity = m;
    C.id_i = ci.data();
    C.id_j = cj.data();
    double** dst[19] = {&C.normal_x, &C.normal_y, &C.point_x, &C.point_y, &C.branch_x,
                        &C.branch_y, &C.bv1_x,    &C.bv1_y,   &C.bv2_x,   &C.bv2_y,
                        &C.shear_x,  &C.shear_y,  &C.fn_x,    &C.fn_y,    &C.ft_x,
                        &C.ft_y,     &C.torque_i, &C.torque_j, &C.damping};
    for (int k = 0; k < 19; ++k) *dst[k] = f[k].data();
    if (m > 0) check(xdem_get_contacts(h_, &C), "get_contacts");
    for (int64_t c = 0; c < m; ++c) {
      ContactInformation info;
      info._otherID = cj[c];
      info._contactNormal = vector2d(f[0][c], f[1][c]);
      info._contactPoint = vector2d(f[2][c], f[3][c]);
      info._branchVector = vector2d(f[4][c], f[5][c]);
      info._branchVectorFromP1 = vector2d(f[6][c], f[7][c]);
      info._branchVectorFromP2 = vector2d(f[8][c], f[9][c]);
      info._shearOverlap = vector2d(f[10][c], f[11][c]);
      info._normalForce = vector2d(f[12][c], f[13][c]);
      info._shearForce = vector2d(f[14][c], f[15][c]);
      info._dampingConstant = f[18][c];
      // ContactInformation::calculateTotalForceAndTorque (ContactInformation.h:62-68)
      info._force = info._normalForce + info._shearForce;
      info._forceOnP1 = info._force;
      info._forceOnP2 = -info._force;
      info._torqueOnP1 = f[16][c];
      info._torqueOnP2 = f[17][c];
      ParticleAccess::contacts(ps[ci[c]])[cj[c]] = info;
    }
  }

  xdem_world h_ = nullptr;
  double consts_[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  bool host_sync_ = true;
  bool newton_reported_ = false;
  bool pending_x_ = false;
  double pending_stress_ = 0.0;
  int32_t method_ = XDEM_ELLIPSE_CLOSEST_APPROACH;
  int32_t precision_ = XDEM_PRECISION_FP64;
};

}  // namespace xdem_gpu

using GpuPeriodicBoundaryWorld = xdem_gpu::GpuWorld<PeriodicBoundaryWorld, XDEM_WORLD_PERIODIC>;
using GpuPeriodicControlWorld =
    xdem_gpu::GpuWorld<PeriodicControlWorld, XDEM_WORLD_PERIODIC_CONTROL>;
using GpuLeesEdwardsBoundaryWorld =
    xdem_gpu::GpuWorld<LeesEdwardsBoundaryWorld, XDEM_WORLD_LEES_EDWARDS>;
