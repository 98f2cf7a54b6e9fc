// world.cuh — device-side layout of one DEM world.
//
// Memory order.  Every per-particle array is stored in a memory order m that
// follows the cell grid: particles of one cell are contiguous, cells in
// row-major order, ties broken by particle id.  The order is refreshed every
// few steps (resort.cuh), so that the 3x3 neighbourhood of a warp's particles
// is a handful of contiguous address ranges.  id_of[m] is the reference's
// particle id at position m and mpos[id] its inverse; everything the reference
// orders by id (contact ownership, force-sum order, clump sub-particles) is
// ordered by id here too, so results do not depend on the memory order.
//
// Contact history lives in records kept in pair-list order: the contacts of
// the particle at m (the owner is the lower id, as in the reference's
// per-particle maps) are the `count[m]` consecutive records from `base[m]`,
// slot s being record base[m] + s.  Each step the candidate kernel reserves
// the owner's records in the pair list (its listed pairs, then the old
// contacts it carries over), so the pair kernels read last step's record of
// a pair and write this step's in pair order.  Two record sets alternate: one
// holds the previous history while the other receives the new contacts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xdem {

constexpr int kMaxSlots = 32;  // upper bound of history slots per particle

struct Slots {
  int32_t* count;    // [n] records owned by the particle at m
  int32_t* base;     // [n] its first record
  // records [K*n], indexed by record (pair-list) index
  int32_t* partner;  // partner id j (> owner id), -1 for a listed pair without contact
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
  double vl_travel;  // relative displacement budget used since the candidate lists were built
                     // (Lees-Edwards shift travelled, affine box scaling)
  int32_t stop;        // set once a run's stop condition is met
  int32_t steps_done;  // steps completed in the current run
  int32_t flips;       // slot-set swaps executed in the current run
  int32_t last_pairs;  // pairs listed by the last candidate scan
  // cell grid of this system: capacity per axis and first cell in the cell
  // arrays; particles (ids and memory positions) [first, first + count)
  int32_t nx_cap, ny_cap, cell_base, first, count;
  // candidate lists (verlet.cuh), system 0: 0 once they must be rebuilt;
  // 1 while the step's build kernel rebuilds them; 1 when a list of the last
  // build overflowed (its owner is scanned in full every step)
  int32_t vl_valid, vl_build, vl_overflow;
  // closest-approach Newton statistics since the last reset: solves,
  // iterations, solves stopped by the iteration cap
  unsigned long long newton_solves, newton_iters, newton_capped;
  // learned warm start since the last reset: starts offered, used, rejected by
  // the residual test, used but overruled by the plain start; contact logits
  // that matched the outcome
  unsigned long long warm_offered, warm_used, warm_rejected, warm_restarted, logit_right;
  unsigned long long vl_builds;  // candidate-list rebuilds since the last reset
};

// One body as the pair kernels read it: every field of a contact
// construction in one 96-byte record (three 32-byte sectors per gather,
// against eight scattered arrays).  The candidate kernels rewrite it each
// step, after the last position move of the step's first half.
struct alignas(32) BodyRec {
  double2 pos, vel;
  double rot, w, r, asp;
  double2 cs;  // (cos, sin) of rot for an ellipse, zero otherwise
  int32_t shape, id, setting, pad;
};
static_assert(sizeof(BodyRec) == 96, "BodyRec is three sectors");

// one entry of the pair list (and the index of its history record): owner
// position, partner position, last step's record of the pair (-1 when the
// pair is new), and packed in `code` the image kind (bits 0-7), the owner's
// slot (bits 8-15), its slot in the old set, 255 when the pair is new (bits
// 16-23), and the flags kDeepFlag and kCarryFlag
struct PairEntry {
  int32_t m, mj, code, old;
};
constexpr int kNoOldSlot = 255;
// a listed pair that the centre-line screen classed deep (mixed precision)
constexpr int kDeepFlag = 1 << 24;
// an old contact carried over without a candidate pair: its record is copied
// by the candidate kernel and the pair kernels skip the entry
constexpr int kCarryFlag = 1 << 25;


// A world holds one system or, batched, nsys independent systems of the same
// world kind side by side: system s owns the particles (ids and memory
// positions) [ws[s].first, ws[s].first + ws[s].count), its own block of
// cells, and its own scalars ws[s]; ids are global, so contacts, slots and
// the pair list need no system index.  The run-level counters and the stop
// flag live in ws[0].
struct DevWorld {
  int n;
  int K;  // slots per particle
  int kind;
  int method;
  int precision;
  int nsys;         // systems in this world
  int ncell_total;  // cells of all systems (regular + Lees-Edwards ghost rows, at capacity)
  int32_t* sys_of;  // [n] system of the particle at m (NULL when nsys == 1)
  int32_t* sys_cell_base;  // [nsys + 1] first cell of each system, then ncell_total
  // particle arrays, memory order
  int32_t* id_of;  // id at position m
  int32_t* mpos;   // [id] position of id
  int32_t* shape;
  int32_t* up;
  int32_t* setting;
  int32_t* num_sub;
  double* orad;
  double* rad;
  double* asp;
  double* mass;
  double* im;
  double* I;
  double* iI;
  double* vol;
  double2* pos;
  double2* vel;
  double* rot;
  double* w;
  double2* branch;
  double4* seg;  // [id] wall segment vertices (x1, y1, x2, y2); NULL without segments
  int32_t* rattler;
  double2* force;
  double* torque;
  int32_t* ncp;
  // cell grid: regular cells, then two ghost rows of nx (Lees-Edwards images);
  // cell_mem holds memory positions
  int32_t* cell_count;
  int32_t* cell_max;  // largest cell count of this step's binning (all systems)
  int32_t* cell_start;
  int32_t* tile_sum;  // scan tile sums
  // [4] blocks finished of the list check, of the scan's tile pass and of the
  // launch that ends the pair phase (the fourth is unused): the last block of
  // each finishes the pass's work, then resets its counter
  uint32_t* done;
  int32_t* cell_mem;
  double2* cell_pos;      // [2n] position of each cell entry, cell order
  // [2n] screening record of each cell entry, cell order: position relative
  // to its cell's corner (FP32; magnitudes below a cell size), the radius of
  // the coarse test, and the id as int bits (negative when the particle skips
  // contact detection, so that one comparison applies both filters)
  float4* cell_scr;
  int32_t* cell_up;       // [2n] upLevel of each cell entry
  BodyRec* body;          // [n] this step's pair-kernel record of each body
  // [n] FP32 (cos, sin) of each ellipse's orientation and its semi-axes (a, b),
  // for the centre-line screen of the mixed-precision candidate kernels;
  // written by k_scatter, moved by a re-sort (NULL in FP64 worlds)
  float4* axis;
  const double* screen_r; // rad for an all-circle world, orad otherwise (segments: screen_radius)
  int32_t* pcell;  // [n] regular cell of the particle at m
  int32_t* prank;  // [n] rank within the cell
  int32_t* gcell;  // [n] ghost cell or -1
  int32_t* grank;
  int32_t* newpos;  // [n] destination of m in a re-sort
  // contacts
  Slots slots[2];
  int32_t* incnt;   // [n] contacts owned by lower ids
  // [K*n] those contacts: owner id << 32 | record (the force sum orders them
  // by owner id without looking it up)
  uint64_t* inref;
  PairEntry* pairs; // [K*n] pairs that passed the candidate scan
  int32_t* npairs;  // number of listed pairs (low half of pair_counts)
  int32_t* fallback;   // [K*n] mixed precision: listed pairs deferred to the FP64 construction
  int32_t* nfallback;  // number of deferred pairs
  // mixed precision, closest approach: listed pairs classed deep by the
  // centre-line screen (indices into pairs), evaluated beside the others
  int32_t* deep;   // [K*n]
  int32_t* ndeep;  // number of deep pairs (high half of pair_counts)
  unsigned long long* pair_counts;  // the two counts, reserved together
  float2* warm;        // [K*n] learned warm start of each listed pair: (root fraction, contact logit)
  // candidate lists kept across steps (verlet.cuh); V == 0: full scan each step
  int V;
  double skin;
  int32_t* vl;       // [V*n] entries (partner memory position << 2 | image kind), slot-major
  int32_t* vl_cnt;   // [n]
  double* vl_disp;   // [n] path length since the lists were built
  double* vl_part;   // block maxima of vl_disp
  // scalars (one per system), status, scratch
  WorldScalars* ws;
  uint32_t* status;
  double* partials;  // block partial sums
  char* scratch;     // re-sort staging, one slab per particle array
  double* stage;     // [6n] id-ordered staging of the dynamic state
};

}  // namespace xdem
