/*
 * xdem_gpu.h — C-ABI of the B200 (sm_100a) implementation of xDEM's
 * per-timestep hot path.
 *
 * One opaque world handle owns the device copy of a particle system (SoA
 * arrays in HBM), its contact history (per-owner sorted slots) and its world
 * scalars (box, Lees-Edwards shift, control-law state).  Every entry point
 * below replaces one method of the reference's C++ class hierarchy; the cited
 * file:line is the reference method whose argument meaning, sequencing and
 * side effects the entry point reproduces.  Where the reference prints and
 * calls exit(), these entry points return an XDEM_ERR_* bit set instead and
 * leave the handle usable.
 *
 * Conventions
 *   - particle ids equal indices 0..n-1 (the reference relies on this in
 *     BaseWorld.cpp:72-74);
 *   - a contact is keyed by (id_i, id_j) with id_i < id_j and its history is
 *     owned by id_i (PeriodicBoundaryWorld.cpp:118, BaseParticle.cpp:36-95);
 *   - all arrays are host pointers unless a name says otherwise; every call is
 *     serialised on the handle's CUDA stream;
 *   - return value: 0 (XDEM_OK) or an OR of XDEM_ERR_* bits.
 */
#ifndef XDEM_GPU_H
#define XDEM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XDEM_ABI_VERSION 1

/* Status bits.  Device kernels OR them into a per-world status word. */
enum xdem_status_bits {
  XDEM_OK = 0,
  /* candidate list of one particle reached 200 entries
     (PeriodicBoundaryWorld.cpp:75-78 exits with -2), or a particle ran out of
     history slots (no reference counterpart: its hash map grows) */
  XDEM_ERR_CAPACITY = 1 << 0,
  /* a closest-approach Newton iteration did not terminate: it repeated an
     earlier iterate (it would cycle forever) or reached 1,000 iterations
     (EllipticParticle.cpp:621 has no cap and never returns there); the
     quartic's root between the analytic start and 1 was taken by bisection */
  XDEM_ERR_NEWTON = 1 << 1,
  /* a time integral produced a non-finite position, velocity or spin (the
     reference carries NaN on silently) */
  XDEM_ERR_NONFINITE = 1 << 2,
  /* pair of shapes without a contact law, e.g. circle-ellipse
     (CircularParticle.cpp:38, EllipticParticle.cpp:30 exit with -1) */
  XDEM_ERR_UNSUPPORTED_PAIR = 1 << 3,
  /* normalisation of a zero-length vector (MathVector.h:180-190 exits) */
  XDEM_ERR_ZERO_VECTOR = 1 << 4,
  /* a CUDA runtime call failed */
  XDEM_ERR_CUDA = 1 << 5,
  /* bad argument, unknown enum, or call not valid for this world kind */
  XDEM_ERR_ARGUMENT = 1 << 6,
  /* cell grid has fewer than 3 cells along an axis (the reference's 3x3
     neighbour scan would visit a cell twice) */
  XDEM_ERR_GRID = 1 << 7,
  /* a device-side wait (tensor-core completion barrier) ran out of its
     iteration limit; the kernel freed its resources and stopped */
  XDEM_ERR_TIMEOUT = 1 << 8
};

/* World kinds: PeriodicBoundaryWorld.h:8, PeriodicControlWorld.h:5,
   LeesEdwardsBoundaryWorld.h:5 */
enum xdem_world_kind {
  XDEM_WORLD_PERIODIC = 0,
  XDEM_WORLD_PERIODIC_CONTROL = 1,
  XDEM_WORLD_LEES_EDWARDS = 2
};

/* Particle shapes: CircularParticle.h:10, EllipticParticle.h:10,
   GluedParticle.h:5, SegmentObject.h:13.  A segment is a fixed wall between
   two vertices (xdem_particles.seg_*): radius = outer_radius = half its
   length, (x, y) = the vertices' midpoint, rot = the direction's angle, and
   SKIP_TIME_INTEGRAL set, as the reference constructor leaves them
   (SegmentObject.h:24-40).  Segments touch circles only; a segment meeting an
   ellipse raises XDEM_ERR_UNSUPPORTED_PAIR (the reference exits). */
enum xdem_shape {
  XDEM_SHAPE_CIRCLE = 0,
  XDEM_SHAPE_ELLIPSE = 1,
  XDEM_SHAPE_CLUMP = 2,
  XDEM_SHAPE_SEGMENT = 3
};

/* SETTING bit flags, same values as BaseParticle.h:19-24 */
enum xdem_setting {
  XDEM_SETTING_NONE = 0,
  XDEM_SKIP_TIME_INTEGRAL = 1 << 0,
  XDEM_SKIP_CONTACT_DETECTION = 1 << 1,
  XDEM_SKIP_MACRO_SUM = 1 << 2
};

/* Ellipse-ellipse contact law.  CLOSEST_APPROACH is the Zheng and
   Palffy-Muhoray quartic solved by Newton (EllipticParticle.cpp:34-285, the
   one the reference dispatches at :27); INTERSECTION is Strobach's fast
   quartic solver on the intersection quartic (EllipticParticle.cpp:288-484). */
enum xdem_ellipse_method {
  XDEM_ELLIPSE_CLOSEST_APPROACH = 0,
  XDEM_ELLIPSE_INTERSECTION = 1
};

/* Arithmetic of contact geometry and forces.  State, history and the
   Lees-Edwards shift are FP64 in both modes. */
enum xdem_precision {
  XDEM_PRECISION_FP64 = 0,
  XDEM_PRECISION_MIXED = 1
};

/* Box-control laws of PeriodicControlWorld (PeriodicControlWorld.cpp:124-237) */
enum xdem_box_law {
  XDEM_BOX_NONE = 0,
  XDEM_BOX_STRAIN = 1,                 /* updatePeriodicBoundary_strainControl(p0, p1) */
  XDEM_BOX_STRESS_XY = 2,              /* stressControlX(p0) then stressControlY(p0) */
  XDEM_BOX_STRESS_UNIFORM = 3,         /* updatePeriodicBoundary_stressControlUniform(p0) */
  XDEM_BOX_STRESS_UNIFORM_LIMIT = 4    /* ..._stressControlUniform_strainLimit(p0) */
};

/* Step sequences */
enum xdem_sequence {
  /* the world kind's own takeTimeStep(): PeriodicBoundaryWorld.cpp:119-127,
     PeriodicControlWorld.cpp:114-122, LeesEdwardsBoundaryWorld.cpp:21-31 */
  XDEM_SEQ_TAKE_TIME_STEP = 0,
  /* the driver-composed compression loop of mainIsoCircPack_WCCM.cpp:117-126:
     modifyParticlePosition, findPossibleContacts, updateContacts,
     collectForceAndTorque, takeTimeIntegral (no rattler reset) */
  XDEM_SEQ_SUBSTEPS = 1
};

/* Construction parameters: BaseWorld(dt, particles, model) (BaseWorld.h:44-56),
   setWorldBoundary (BaseWorld.cpp:3-11), the contact model constructor
   (ContactModel_LinearDissipativeFrictional.h:11-24), _GlobalDamping_
   (BaseParticle.cpp:9) and setShiftStrainRate (LeesEdwardsBoundaryWorld.cpp:485). */
typedef struct xdem_params {
  int32_t world_kind;        /* enum xdem_world_kind */
  int32_t ellipse_method;    /* enum xdem_ellipse_method */
  int32_t precision;         /* enum xdem_precision */
  int32_t max_contacts;      /* history slots per particle (<= 32), 0 = default (24) */
  double dt;
  double xmin, xmax, ymin, ymax;
  double normal_stiffness, shear_stiffness, restitution_coeff, frictional_coeff;
  double global_damping;
  double shift_strain_rate;  /* Lees-Edwards only */
  /* cell size; 0 = 2.01 * max outer radius (BaseWorld.cpp:201-219).  Any value
     >= 2 * max outer radius gives the same contact set. */
  double max_particle_size;
} xdem_params;

/* Per-step extras of xdem_run, matching what the reference drivers do around
   the step (mainIsoCircPack_WCCM.cpp:76-85,115-126,
   mainIsoElpsPackTestEntropy.cpp:171). */
typedef struct xdem_control {
  int32_t sequence;            /* enum xdem_sequence */
  int32_t scale_rattlers;      /* 1: scaleVelocityOfRattlers(rattler_scale) before the step */
  int32_t reset_rattlers;      /* 1: resetVelocityOfRattlers() after the step */
  int32_t update_stress;       /* 1: updateTotalStress() after the step */
  int32_t box_law;             /* enum xdem_box_law, applied after the stress update */
  int32_t stop_on_pressure;    /* 1: stop once trace(stress)/2 >= stop_pressure (checked on device) */
  double rattler_scale;
  double p0, p1;               /* box-law arguments */
  double stop_pressure;
} xdem_control;

/* Particle arrays (length n).  For xdem_set_particles every pointer must be
   non-NULL except num_sub/branch_x/branch_y (NULL = no clumps), seg_* (NULL =
   no segments) and
   is_rattler (NULL = all rattlers, as before the first collect).  For
   xdem_get_particles, NULL pointers are skipped. */
typedef struct xdem_particles {
  int32_t n;
  int32_t *shape, *up_level, *setting, *is_rattler;
  double *outer_radius;      /* BaseParticle::_outerRadius */
  double *radius;            /* circle radius / ellipse semi-major axis a */
  double *aspect_ratio;      /* a/b for ellipses, 1 otherwise */
  double *x, *y, *vx, *vy, *rot, *rot_vel;
  double *volume, *mass, *inv_mass, *inertia, *inv_inertia;
  int32_t *num_sub;          /* clump: number of sub-particles whose ids follow it */
  double *branch_x, *branch_y; /* sub-particle: GluedParticle::_branchVectors entry */
  /* segment: SegmentObject::_vertex1, _vertex2 (NULL when there are no
     segments; entries of other shapes are ignored) */
  double *seg_x1, *seg_y1, *seg_x2, *seg_y2;
} xdem_particles;

/* Contact records, sorted by (id_i, id_j); the fields of ContactInformation
   (ContactInformation.h:14-29).  branch = p_i - (p_j + offset)
   (BaseParticle.cpp:85); force = fn + ft; torque_i/j = torqueOnP1/P2. */
typedef struct xdem_contacts {
  int64_t count;             /* in: records to upload; out: records present */
  int64_t capacity;          /* out-calls: array length available */
  int32_t *id_i, *id_j;
  double *normal_x, *normal_y, *point_x, *point_y, *branch_x, *branch_y;
  double *bv1_x, *bv1_y, *bv2_x, *bv2_y;
  double *shear_x, *shear_y;
  double *fn_x, *fn_y, *ft_x, *ft_y;
  double *torque_i, *torque_j, *damping;
} xdem_contacts;

typedef struct xdem_world_s* xdem_world;
typedef struct xdem_mlp_s* xdem_mlp;

/* ---- library ---------------------------------------------------------- */
int32_t xdem_abi_version(void);
const char* xdem_status_string(int32_t status_bit);
/* sets *out to the number of CUDA devices; returns XDEM_ERR_CUDA if none */
int32_t xdem_device_count(int32_t* out);

/* ---- lifetime ---------------------------------------------------------- */
/* BaseWorld::BaseWorld (BaseWorld.h:44-56) + setWorldBoundary (BaseWorld.cpp:3-11).
   The world is created empty; xdem_set_particles sizes it. */
int32_t xdem_create(const xdem_params* params, xdem_world* out);
int32_t xdem_destroy(xdem_world w);
/* run this world's work on a caller-owned cudaStream_t (NULL = own stream) */
int32_t xdem_set_stream(xdem_world w, void* cuda_stream);
/* the cudaStream_t this world's work runs on */
int32_t xdem_get_stream(xdem_world w, void** cuda_stream);

/* ---- batched systems ----------------------------------------------------- */
/* No counterpart in the reference, which runs one world per process.  Puts
   nsys independent systems of this world's kind into one handle, so that each
   kernel of a step covers all of them and xdem_run replays one captured graph
   for the whole batch.  systems[s] holds system s with local ids 0..n_s-1
   (up_level local too); in the world its particles take the ids first_s + id,
   first_s = n_0 + ... + n_{s-1}, and every other entry point addresses that
   concatenation (contacts, state, particles).  boxes: xmin, xmax, ymin, ymax
   per system; dts: time step per system (NULL = the world's).  The contact
   model, precision, ellipse method and slot count are the world's.  Replaces
   xdem_set_particles.  Per-system results come from the xdem_batch_get_*
   calls; xdem_get_boundary, xdem_get_stress and xdem_get_lees_edwards report
   system 0; xdem_set_boundary, xdem_set_lees_edwards and
   xdem_scale_boundary_to_solid_fraction, and xdem_run with stop_on_pressure,
   return XDEM_ERR_ARGUMENT on a batch; the other setters apply to every
   system. */
int32_t xdem_batch_set_particles(xdem_world w, int32_t nsys, const xdem_particles* systems,
                                 const double* boxes, const double* dts);
/* *nsys = systems in the world; first (may be NULL): nsys + 1 entries, the
   first id of each system and then n */
int32_t xdem_batch_info(xdem_world w, int32_t* nsys, int32_t* first);
/* updateTotalStress result of each system (xx, xy, yx, yy per system) */
int32_t xdem_batch_get_stress(xdem_world w, double* stress);
/* box of each system (xmin, xmax, ymin, ymax per system) */
int32_t xdem_batch_get_boundaries(xdem_world w, double* boxes);
/* countActucalContacts of each system */
int32_t xdem_batch_count_contacts(xdem_world w, int64_t* counts);

/* ---- state exchange ----------------------------------------------------- */
/* upload: vector<BaseParticle*> handed to the world constructor (BaseWorld.h:44);
   also runs updateMaximumParticleSize (BaseWorld.cpp:201-219) and
   updateTotalParticleVolume (BaseWorld.cpp:188-199) */
int32_t xdem_set_particles(xdem_world w, const xdem_particles* p);
/* download: the BaseParticle getters (BaseParticle.h:109-127) */
int32_t xdem_get_particles(xdem_world w, xdem_particles* p);
/* upload a contact history: the per-particle _contactInfo maps
   (BaseParticle.h:46; read4File_particle BaseParticle.cpp:172-186) */
int32_t xdem_set_contacts(xdem_world w, const xdem_contacts* c);
/* download contacts: getContactInfo() of every particle (BaseParticle.h:125).
   With capacity < count only count is written (returns XDEM_ERR_CAPACITY). */
int32_t xdem_get_contacts(xdem_world w, xdem_contacts* c);
/* _totalForce/_totalTorque/_numContactPerParticle after collectForceAndTorque
   (BaseWorld.cpp:17-57) */
int32_t xdem_get_force_and_torque(xdem_world w, double* fx, double* fy, double* torque,
                                  int32_t* num_contacts);
/* countActucalContacts (BaseWorld.cpp:262-269) */
int32_t xdem_count_contacts(xdem_world w, int64_t* out);

/* Dynamic state only (positions, velocities, orientations, spins), the part a
   driver reads and writes every step through the BaseParticle getters and
   setters (BaseParticle.h:112-119, :140-153).  Host arrays may be pinned
   (cudaHostAlloc); the copies are then asynchronous on the world's stream and
   xdem_download_state returns after they complete. */
int32_t xdem_upload_state(xdem_world w, const double* x, const double* y, const double* vx,
                          const double* vy, const double* rot, const double* rot_vel);
int32_t xdem_download_state(xdem_world w, double* x, double* y, double* vx, double* vy,
                            double* rot, double* rot_vel);

/* ---- world scalars ------------------------------------------------------ */
/* getXmin/getXmax/getYmin/getYmax (BaseWorld.h:75-78) */
int32_t xdem_get_boundary(xdem_world w, double box[4]);
/* setWorldBoundary (BaseWorld.cpp:3-11) */
int32_t xdem_set_boundary(xdem_world w, const double box[4]);
/* getStress after updateTotalStress (BaseWorld.h:89): xx, xy, yx, yy */
int32_t xdem_get_stress(xdem_world w, double stress[4]);
/* getTotalShift, shift velocity, getTotalStrain, shift strain rate
   (LeesEdwardsBoundaryWorld.h:39-40) */
int32_t xdem_get_lees_edwards(xdem_world w, double out[4]);
int32_t xdem_set_lees_edwards(xdem_world w, const double in[4]);
/* setShiftStrainRate (LeesEdwardsBoundaryWorld.cpp:485-489) */
int32_t xdem_set_shift_strain_rate(xdem_world w, double rate);
/* setTimeIncrement (BaseWorld.cpp:178-181) */
int32_t xdem_set_time_increment(xdem_world w, double dt);
/* BaseParticle::_GlobalDamping_ (BaseParticle.cpp:9) */
int32_t xdem_set_global_damping(xdem_world w, double damping);
/* setFriction/setRestitutionCoeff/recalculateFactor
   (ContactModel_LinearDissipativeFrictional.cpp:56-71); the damping constant
   of an existing contact is kept, as in the reference */
int32_t xdem_set_contact_model(xdem_world w, double kn, double kt, double restitution,
                               double friction);
/* setVirtualBoundaryMass() / (mass) and setMaxStrainRate
   (PeriodicControlWorld.cpp:58-71) */
int32_t xdem_set_virtual_boundary_mass(xdem_world w, double mass /* <0: from particles */);
int32_t xdem_set_max_strain_rate(xdem_world w, double rate);
/* kinetic energy (BaseWorld.cpp:302-310) */
int32_t xdem_get_kinetic_energy(xdem_world w, double* out);
/* closest-approach Newton statistics since creation or the last reset:
   out = {solves, iterations, solves that did not terminate (a repeated iterate or the cap)}
   (NewtonRaphsonForQuartic, EllipticParticle.cpp:613-626) */
int32_t xdem_get_newton_stats(xdem_world w, int64_t out[3]);
int32_t xdem_reset_newton_stats(xdem_world w);
/* pairs that passed the last candidate scan's coarse test (the pairs whose
   geometry was evaluated) */
int32_t xdem_get_pair_count(xdem_world w, int64_t* out);

/* ---- binary snapshots ----------------------------------------------------- */
/* Checkpoint and resume (the reference writes text files,
   BaseParticle.cpp:158-186, ContactInformation.h:51-60, and reads particles
   back with read4File_particle): the whole world — every system's box, time
   step, contact model, Lees-Edwards and box-law state, every particle field
   and the full contact history — in one binary file, so that a loaded world
   continues exactly as the saved one would have.  Loading needs a world of
   the same kind (its precision, ellipse law and slot count stay its own) and
   replaces its particles, contacts and scalars; the file is tied to the
   library's build (native byte order, structure sizes checked). */
int32_t xdem_save_snapshot(xdem_world w, const char* path);
int32_t xdem_load_snapshot(xdem_world w, const char* path);
/* Host only (no device needed): reads and checks a snapshot file as
   xdem_load_snapshot does before it touches the device (sizes against the
   file length, systems covering ids [0, n) in order, the saved memory order a
   permutation within each system, contact ids in range); out = {n, systems,
   contacts, world kind}.  XDEM_ERR_ARGUMENT for a missing, truncated or
   inconsistent file. */
int32_t xdem_snapshot_info(const char* path, int64_t out[4]);
/* Byte layout of this build's snapshot files: {header size, size of one
   system's scalar record, offset of its first-id field, offset of its
   particle-count field}. */
int32_t xdem_snapshot_layout(int64_t out[4]);

/* ---- observables ---------------------------------------------------------- */
/* QuadronAnalysis's rattler-free coordination number and solid fraction
   (QuadronAnalysis.cpp:663-668,980-986,144-165,703-713,724-732) on the
   device, from the current contacts: particles without contacts leave, then
   repeatedly the particles left with one contact, with it; out = {Z = 2 x
   remaining contacts / remaining particles, remaining volume / box area}.
   The batch form writes two values per system. */
int32_t xdem_quadron_z_phi(xdem_world w, double out[2]);
int32_t xdem_batch_quadron_z_phi(xdem_world w, double* out);

/* ---- sub-steps (each one reference method) ----------------------------- */
/* PeriodicBoundaryWorld::modifyParticlePosition (PeriodicBoundaryWorld.cpp:129-142)
   or LeesEdwardsBoundaryWorld::modifyParticlePosition (LeesEdwardsBoundaryWorld.cpp:304-333) */
int32_t xdem_modify_particle_position(xdem_world w);
/* LeesEdwardsBoundaryWorld::apply/removeBackgroudVelocity (:508-530) */
int32_t xdem_apply_background_velocity(xdem_world w);
int32_t xdem_remove_background_velocity(xdem_world w);
/* findPossibleContacts: the cell grid (PeriodicBoundaryWorld.cpp:12-85,
   LeesEdwardsBoundaryWorld.cpp:34-205).  Candidates are generated from it
   inside xdem_update_contacts; the set is the same. */
int32_t xdem_find_possible_contacts(xdem_world w);
/* updateContacts: per candidate pair geometry, force and history
   (PeriodicBoundaryWorld.cpp:87-107, LeesEdwardsBoundaryWorld.cpp:207-283,
   BaseParticle.cpp:27-98) */
int32_t xdem_update_contacts(xdem_world w);
/* BaseWorld::collectForceAndTorque (BaseWorld.cpp:17-57) */
int32_t xdem_collect_force_and_torque(xdem_world w);
/* BaseWorld::takeTimeIntegral (BaseWorld.cpp:59-77, BaseParticle.cpp:107-118,
   GluedParticle.cpp:91-125) */
int32_t xdem_take_time_integral(xdem_world w);
/* BaseWorld::resetVelocityOfRattlers / scaleVelocityOfRattlers (BaseWorld.cpp:79-106) */
int32_t xdem_reset_velocity_of_rattlers(xdem_world w);
int32_t xdem_scale_velocity_of_rattlers(xdem_world w, double scale);
/* BaseWorld::updateTotalStress (BaseWorld.cpp:158-176); stress may be NULL */
int32_t xdem_update_total_stress(xdem_world w, double stress[4]);
/* PeriodicControlWorld box laws (PeriodicControlWorld.cpp:124-237) */
int32_t xdem_update_boundary(xdem_world w, int32_t box_law, double p0, double p1);
/* LeesEdwardsBoundaryWorld::updateLeesEdwardBoundary (:285-296) */
int32_t xdem_update_lees_edwards_boundary(xdem_world w);
/* scaleBoundarySizeToGivenSolidFraction (PeriodicBoundaryWorld.cpp:276-284) */
int32_t xdem_scale_boundary_to_solid_fraction(xdem_world w, double solid_fraction);

/* ---- whole steps -------------------------------------------------------- */
/* the world kind's takeTimeStep() */
int32_t xdem_take_time_step(xdem_world w);
/* nsteps iterations of ctl's sequence with fused kernels, captured in a CUDA
   graph; *steps_done (may be NULL) receives the number of steps executed.
   Returns the OR of all status bits raised (synchronises once at the end). */
int32_t xdem_run(xdem_world w, int32_t nsteps, const xdem_control* ctl, int32_t* steps_done);
/* wait for the handle's stream; returns and clears the device status word */
int32_t xdem_synchronize(xdem_world w);

/* ---- per-kernel timing (CUDA events on the world's stream) --------------- */
/* enable=1: every kernel launch of this world is bracketed by CUDA events and
   xdem_run launches without graph capture; enable=0 stops and clears. */
int32_t xdem_set_profiling(xdem_world w, int32_t enable);
/* Number of kernel kinds; name of kind k. */
int32_t xdem_profile_kinds(void);
const char* xdem_profile_name(int32_t kind);
/* Synchronises, then for every kernel kind k < nkinds writes the launches
   recorded since profiling was enabled and their summed device time (ms). */
int32_t xdem_get_profile(xdem_world w, int32_t nkinds, int64_t* launches, double* total_ms);
/* Kernel launches issued on this world's stream since creation (graph
   replays count every kernel node). */
int32_t xdem_launch_count(xdem_world w, int64_t* out);
/* Device-side interval on the world's stream: start records an event; stop
   records a second one, waits for it and returns the elapsed milliseconds. */
int32_t xdem_timer_start(xdem_world w);
int32_t xdem_timer_stop(xdem_world w, double* ms);
/* NVTX range around the calls in between (for profilers: ncu --nvtx
   --nvtx-include "<name>/"); no effect without a tool attached. */
int32_t xdem_range_push(const char* name);
int32_t xdem_range_pop(void);
/* Page-locked host memory for asynchronous state exchange. */
void* xdem_host_alloc(int64_t bytes);
void xdem_host_free(void* p);

/* ---- launch configuration and autotuning ---------------------------------- */
/* No counterpart in the reference.  Results do not depend on these (the
   contact set of any cell size >= 2 r_max is the same, and force sums run in
   id order), only the speed does.  pair_blocks_per_sm: blocks of 128 threads
   per SM of the pair kernels, whose grid-stride loop gives each thread
   npairs / (148 * blocks * 128) pairs (default 16); cell_factor: cell size as
   a multiple of 2.01 x the largest outer radius, in [1, 4] (default 1; a
   larger cell meets the 200-candidate cap sooner). */
int32_t xdem_set_launch_config(xdem_world w, int32_t pair_blocks_per_sm, double cell_factor);
int32_t xdem_get_launch_config(xdem_world w, int32_t* pair_blocks_per_sm, double* cell_factor);
/* Candidate lists kept across steps (no counterpart in the reference, which
   rescans the 3x3 cells every step, PeriodicBoundaryWorld.cpp:47-84): each
   particle keeps the partners within its screening distance plus a skin
   (skin_fraction x the cell size) found by the last full scan, and only those
   are tested each step with the reference's tests; the lists are rebuilt when
   particles, the Lees-Edwards shift or the box have moved enough to use up the
   skin, after memory-order refreshes and after host changes.  The pairs found
   are the full scan's.  capacity: partners kept per particle (0 = full scan
   every step; default 48; a particle with more is scanned in full until the next
   build); skin_fraction in
   (0, 1] (default 0.1).  Call before xdem_set_particles. */
int32_t xdem_set_candidate_lists(xdem_world w, int32_t capacity, double skin_fraction);
/* Steps between refreshes of the particles' memory order on the device (no
   counterpart in the reference, whose particles stay in id order).  The
   arrays are re-sorted by cell every `interval` steps so that neighbours sit
   at nearby addresses; results do not depend on it.  interval: odd, or 0 =
   never re-sort; default 63. */
int32_t xdem_set_memory_order_refresh(xdem_world w, int32_t interval);
/* out = {list rebuilds since the last xdem_reset_newton_stats, longest list,
   total entries, capacity} */
int32_t xdem_get_candidate_list_stats(xdem_world w, int64_t out[4]);
/* Times steps_per_trial steps of ctl for each of 12 configurations
   (blocks 4, 8, 16, 32 x cell factors 1, 1.2, 1.5; CUDA events on the
   world's stream), keeps the fastest and returns the OR of the status bits of
   the trials.  The trials are real steps: the world advances by
   12 * (steps_per_trial + 1) steps.  trial_ms (may be NULL): 12 times,
   factor-major. */
int32_t xdem_autotune(xdem_world w, const xdem_control* ctl, int32_t steps_per_trial,
                      double* trial_ms);

/* ---- single-pair geometry (known-answer tests) ------------------------- */
/* BaseParticle::calculateContactGeometry for one pair on the device.
   pi/pj: {shape, radius, aspect_ratio, x, y, vx, vy, rot, rot_vel};
   out: {contacted, nx, ny, cpx, cpy, bv1x, bv1y, bv2x, bv2y, overlap,
         rvx, rvy, nrvx, nrvy, srvx, srvy, newton_iterations} per pair. */
int32_t xdem_pair_geometry(int32_t npairs, int32_t ellipse_method, int32_t precision,
                           const double* pi /* npairs*9 */, const double* pj /* npairs*9 */,
                           const double* offset /* npairs*4: ox, oy, ovx, ovy */,
                           double* out /* npairs*17 */);

/* ---- learned warm start of the closest-approach Newton iteration ---------- */
/* No counterpart in the reference.  A network (7 inputs: the centre offset in
   ellipse i's frame over b_i, cos and sin of θ_j - θ_i, a_i/b_i, a_j/b_i,
   b_j/b_i; three hidden layers of 64 with SiLU; outputs: the root of the
   reference's quartic (EllipticParticle.cpp:92-100, 163) as a fraction of
   Newton's analytic start sqrt(δ+1), and a contact logit), BF16 weights with
   FP32 accumulation on the tensor cores, trained on pairs harvested from a
   world.  With xdem_set_warm_start a closest-approach world starts Newton
   from the prediction when its first step is small, keeps the plain start
   otherwise, and iterates to the reference's tolerance either way, so the
   result is the plain solver's wherever the plain iteration's root lies in
   [min(1, sqrt(δ+1)), max(1, sqrt(δ+1))] (after a long wander it can end
   outside, where the warm-started solve returns the interval's root);
   xdem_get_warm_stats counts what happened. */
int32_t xdem_mlp_create(uint64_t seed, xdem_mlp* out);
int32_t xdem_mlp_destroy(xdem_mlp m);
/* number of FP32 parameters: W1[64][16], b1[64], W2[64][64], b2[64],
   W3[64][64], b3[64], W4[8][64], b4[8] (input columns 7..15 of W1 and
   output rows 2..7 of W4 are padding and stay zero) */
int32_t xdem_mlp_param_count(void);
/* parameters (host arrays of xdem_mlp_param_count floats) and the 7 input
   scales (each feature is multiplied by its scale); either may be NULL */
int32_t xdem_mlp_get_params(xdem_mlp m, float* theta, float* scale);
int32_t xdem_mlp_set_params(xdem_mlp m, const float* theta, const float* scale);
/* forward pass of n rows of 7 features (host arrays; y: 2 per row) */
int32_t xdem_mlp_forward(xdem_mlp m, int64_t n, const float* x, float* y);
/* Self-test of the tensor-core kernels' bounded waits (no reference
   counterpart): one CTA waits on a completion barrier that nothing arrives
   on; returns XDEM_ERR_TIMEOUT once the wait limit has passed, with the
   kernel's elapsed milliseconds in *ms. */
int32_t xdem_selftest_bounded_wait(double* ms);
/* gradient of the mean loss over n samples (host arrays: x 7 per row,
   target root fraction or NaN where no root exists, contact 0/1):
   (y0 - target)^2 where the target exists + 0.1 * BCE(y1, contact) */
int32_t xdem_mlp_gradient(xdem_mlp m, int64_t n, const float* x, const float* target,
                          const float* contact, float* grad, float* loss);
/* the network's training set: append host samples, read it back (arrays
   may be NULL; *size receives the count), clear it */
int32_t xdem_mlp_add_samples(xdem_mlp m, int64_t n, const float* x, const float* target,
                             const float* contact);
int32_t xdem_mlp_dataset(xdem_mlp m, int64_t* size, float* x, float* target, float* contact);
int32_t xdem_mlp_clear_dataset(xdem_mlp m);
/* Adam over the training set (first max_samples, 0 = all): epochs passes of
   shuffled mini-batches (batch >= 64); epoch_loss (may be NULL) receives the
   mean loss of each epoch */
int32_t xdem_mlp_train(xdem_mlp m, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                       int64_t max_samples, float* epoch_loss);
/* appends to m's training set every stride-th ellipse pair of the world's
   last candidate list (features, the plain Newton root as a fraction of its
   start or NaN, contact flag); at most max_new, *added receives the count */
int32_t xdem_harvest_pairs(xdem_world w, xdem_mlp m, int32_t stride, int64_t max_new,
                           int64_t* added);
/* m (NULL: off) gives the closest-approach Newton iteration of this world its
   warm start from the next step on; m must outlive the setting */
int32_t xdem_set_warm_start(xdem_world w, xdem_mlp m);
/* since the last xdem_reset_newton_stats: {starts offered, used, rejected by
   the residual test, used but overruled by the plain start, contact logits
   that matched the outcome} */
int32_t xdem_get_warm_stats(xdem_world w, int64_t out[5]);

/* ---- allocation-free stress ---------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
   memory (code inside a CUDA graph being captured, hosts that own a fixed
   device budget, real-time loops that must not take allocator locks): the box
   stress sum_c F_c (x) b_c / area (the sum of BaseWorld::updateTotalStress)
   from per-contact force (fx, fy) and branch vector (bx, by) arrays the caller
   holds on the device; stress receives xx, xy, yx, yy on the device.  All
   pointers are device pointers; work is queued on cuda_stream (NULL = the
   default stream) and is not waited for.  Uses no cudaMalloc: its partial sums
   live in a fixed array of the library (128 KiB on every GPU that loads it,
   held until exit), so at most xdem_total_stress_noalloc_max_contacts()
   contacts per call (4,194,304; more returns XDEM_ERR_CAPACITY), and calls
   that may overlap on the GPU race on that array and must be ordered by the
   caller.  The first call on a device looks the array up for that device:
   make it with the device current and before any stream capture begins.  The
   address is kept for the life of the process, so the entry point must not be
   used on a device after a cudaDeviceReset there. */
int32_t xdem_total_stress_noalloc(int64_t ncontacts, const double* fx, const double* fy,
                                  const double* bx, const double* by, double area,
                                  double* stress, void* cuda_stream);
int64_t xdem_total_stress_noalloc_max_contacts(void);

/* ---- packing generation (host only, no GPU) ------------------------------ */
/* Random sequential addition of discs of the given bounding radii into the
   box [xmin,xmax]x[ymin,ymax] without overlap; seeded, deterministic.
   Returns XDEM_ERR_CAPACITY if max_attempts proposals for one disc fail. */
int32_t xdem_rsa_positions(int32_t n, const double* radius, const double box[4], uint64_t seed,
                           int64_t max_attempts, double* x, double* y);

/* CircularParticle/EllipticParticle/SegmentObject::calculateParticleProperties
   (density) (CircularParticle.cpp:16-23, EllipticParticle.cpp:7-14,
   SegmentObject.cpp:4-10; a segment's radius is half its length) */
int32_t xdem_particle_properties(int32_t n, const int32_t* shape, const double* radius,
                                 const double* aspect_ratio, double density, double* volume,
                                 double* mass, double* inv_mass, double* inertia,
                                 double* inv_inertia);
/* GluedParticle::calculateParticleProperties(density) (GluedParticle.cpp:7-80)
   for one clump of nsub sub-particles; out_clump = {x, y, volume, mass,
   inv_mass, inertia, inv_inertia}; branch_x/y receive each sub-particle's
   branch vector.  The sub-particles take the clump's mass and inertia. */
int32_t xdem_clump_properties(int32_t nsub, const int32_t* sub_shape, const double* sub_radius,
                              const double* sub_aspect_ratio, const double* sub_x,
                              const double* sub_y, const double* sub_rot, double density,
                              double* out_clump, double* branch_x, double* branch_y);

#ifdef __cplusplus
}
#endif

#endif /* XDEM_GPU_H */
