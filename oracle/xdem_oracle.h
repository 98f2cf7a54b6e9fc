/* xdem_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * C restatement of the reference xDEM per-timestep path, used as the CPU
 * checker of the CUDA implementation (tests/, __graft_entry__.smoke(),
 * bench.py's CPU-baseline leg).  It is pinned against the compiled reference
 * (oracle/_ref) by tests/test_oracle_vs_reference.py.
 *
 * Differences from the reference, all deliberate and shared with the CUDA
 * path:
 *   - per-particle force sums run in a fixed order: contacts owned by lower
 *     ids (ascending owner), then own contacts (ascending partner); the
 *     reference's single-thread order is the same except that own contacts
 *     follow unordered_map iteration order (BaseWorld.cpp:26-56);
 *   - the closest-approach Newton loop stops when it repeats an earlier
 *     iterate (it would cycle forever) or after XO_NEWTON_CAP iterations,
 *     takes the quartic's root on [min(1, s), max(1, s)] by bisection, and
 *     raises XDEM_ERR_NEWTON (EllipticParticle.cpp:621 has no cap and does
 *     not return there);
 *   - errors that exit() in the reference raise status bits instead.
 */
#ifndef XDEM_ORACLE_H
#define XDEM_ORACLE_H
#include <stdint.h>
#include "../include/xdem_gpu.h"

#define XO_NEWTON_CAP 1000
#define XO_CANDIDATE_CAP 200

typedef struct xo_world xo_world;

xo_world* xo_create(const xdem_params* prm, int32_t num_threads);
void xo_destroy(xo_world* w);
int32_t xo_set_particles(xo_world* w, const xdem_particles* p);
int32_t xo_get_particles(xo_world* w, xdem_particles* p);
int32_t xo_set_contacts(xo_world* w, const xdem_contacts* c);
int32_t xo_get_contacts(xo_world* w, xdem_contacts* c);
int32_t xo_get_force_and_torque(xo_world* w, double* fx, double* fy, double* t, int32_t* nc);
void xo_get_boundary(xo_world* w, double* box);
void xo_get_stress(xo_world* w, double* s);
void xo_get_lees_edwards(xo_world* w, double* out);
void xo_set_lees_edwards(xo_world* w, const double* in);
void xo_set_virtual_boundary_mass(xo_world* w, double mass);
void xo_set_max_strain_rate(xo_world* w, double r);
double xo_kinetic_energy(xo_world* w);
int64_t xo_count_contacts(xo_world* w);
int32_t xo_call(xo_world* w, int32_t which, double a, double b, double c);
int32_t xo_run(xo_world* w, int32_t nsteps, const xdem_control* ctl, int32_t* steps_done);
uint32_t xo_status(xo_world* w);
void xo_quadron_z_phi(xo_world* w, double* out);

int32_t xo_pair_geometry(int32_t npairs, int32_t method, const double* pi, const double* pj,
                         const double* off, double* out);
/* Newton on A r^4 + B r^3 + C r^2 + D r + E from init; *iters gets the count,
   *stuck 1 when the iteration repeated an earlier iterate or reached
   XO_NEWTON_CAP (either may be NULL). */
double xo_newton_quartic(double A, double B, double C, double D, double E, double init,
                         int32_t* iters, int32_t* stuck);
/* the root on [min(1, s), max(1, s)] by bisection (q if no sign change) */
double xo_bisect_quartic(double A, double B, double C, double D, double E, double s, double q);
/* Closest approach of ellipse pairs (layout of xo_pair_geometry's inputs): per
   pair A, B, C, D, E of the quartic, the analytic start s = sqrt(delta+1), the
   root q, Newton's iterations, 1 where Newton did not terminate, contacted.
   Pairs rejected before the quartic is formed carry zeros. */
int32_t xo_closest_quartic(int32_t npairs, const double* pi, const double* pj, const double* off,
                           double* out);

#endif
