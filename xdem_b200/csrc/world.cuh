// world.cuh — device-side layout of one DEM world.
//
// Particles are SoA in id order (ids equal indices, as the reference assumes).
// Contact history lives in per-owner slots: slot s of particle i is element
// s*n + i of each slot array (slot-major, so consecutive particles touch
// consecutive addresses), owner = lower id as in the reference's per-particle
// maps.  Two slot sets alternate between steps: one holds the previous step's
// history, the other receives this step's contacts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xdem {

constexpr int kMaxSlots = 32;  // upper bound of history slots per particle

struct Slots {
  int32_t* count;    // [n] contacts owned by particle i
  int32_t* partner;  // [K*n] partner id j (> i)
  double2* n;        // contact normal
  double2* s;        // tangential spring (shear overlap)
  double* damp;      // damping constant, fixed at creation
  double2* f;        // total contact force on the owner (forceOnP1)
  double* t1;        // torqueOnP1
  double* t2;        // torqueOnP2
  double2* b;        // branch vector p_i - (p_j + offset)
  double2* cp;       // contact point            (recorded fields)
  double2* bv1;      // branch vector from P1
  double2* bv2;      // branch vector from P2
  double2* fn;       // normal force
  double2* ft;       // shear force
};

// World scalars kept on the device so that box laws and the Lees-Edwards
// update run inside a captured step without host round trips.
struct WorldScalars {
  double xmin, xmax, ymin, ymax, xlen, ylen;
  double shift, shift_vel, strain, shift_rate;
  double velX, velY, vmass, max_strain_rate;
  double stress[4];
  double scale_x, scale_y;  // affine position scale set by the last box law
  double dt, g, kn, kt, mu, factor;
  double maxsize;
  double ke;
  int32_t stop;        // set once a run's stop condition is met
  int32_t steps_done;  // steps completed in the current run
};

struct DevWorld {
  int n;
  int K;  // slots per particle
  int kind;
  int method;
  int precision;
  int nx_cap, ny_cap;  // cell-grid capacity
  // static particle data
  const int32_t* shape;
  const int32_t* up;
  const int32_t* setting;
  const int32_t* num_sub;
  const double* orad;
  const double* rad;
  const double* asp;
  const double* mass;
  const double* im;
  const double* I;
  const double* iI;
  const double* vol;
  // dynamic particle data
  double2* pos;
  double2* vel;
  double* rot;
  double* w;
  double2* branch;
  int32_t* rattler;
  double2* force;
  double* torque;
  int32_t* ncp;
  // cell grid: regular cells, then two ghost rows of nx (Lees-Edwards images)
  int32_t* cell_count;
  int32_t* cell_start;
  int32_t* cell_mem;
  int32_t* pcell;  // [n] regular cell of particle
  int32_t* prank;  // [n] rank within the cell
  int32_t* gcell;  // [n] ghost cell or -1
  int32_t* grank;
  // contacts
  Slots slots[2];
  int32_t* incnt;   // [n] contacts owned by lower ids
  uint32_t* inref;  // [K*n] owner*K + slot of those contacts
  // scalars, status, scratch
  WorldScalars* ws;
  uint32_t* status;
  double* partials;  // block partial sums
};

}  // namespace xdem
