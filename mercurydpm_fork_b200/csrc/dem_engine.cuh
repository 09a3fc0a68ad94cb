// dem_engine.cuh -- device data layout shared by the DEM kernels.
//
// Layout in HBM (all arrays indexed by the engine's sorted particle order,
// which is (instance, level, cell, id) after every neighbour-list rebuild):
//   pr[b][i]   double4 (x, y, z, radius)         b = state buffer 0/1
//   vm[b][i]   double4 (vx, vy, vz, invMass)
//   wi[b][i]   double4 (wx, wy, wz, invInertia)
//   qo[b][i]   double4 orientation quaternion (q0..q3)
//   info[b][i] int4    (id, species, instance, flags)
//   caller[b][i] int   index of the particle in the caller's upload order
// The 32-byte records let a neighbour's position+radius, velocity+mass and
// angular velocity+inertia each arrive in one 32-byte sector.
// Neighbour lists are fixed-capacity rows, one per particle: nbr[l][i*cap + k]
// (k < count[l][i]); l = Control::lbuf flips at every rebuild. The force
// kernel walks a warp's entries particle by particle, so a particle's entries
// are contiguous. Contact history is stored per contact, not per entry: the
// springs of an evaluation's contacts sit in a pool indexed by the contact's
// item number in that evaluation, pool[p][j*stride + c] (3 or 9 components
// per spring, padded), and every list entry keeps the pool index of its
// contact of the last evaluation, hidx[b][k*ncap + i], valid where its active
// bit, act[b][w*ncap + i] (bit k%32 of word k/32), is set. hidx and act follow
// the state buffer b = Control::cur (a rebuild carries them to the new order);
// the pool flips with every force evaluation (p = Control::pcur: read p,
// write p^1), and a rebuild leaves it in place. A thread may therefore read its
// partner's spring of the previous step (needed for periodic pairs) while
// the partner writes the next one.
#pragma once
#include <cstdint>
#include "dem_math.cuh"
#include "dem_walls.cuh"
#include "../../include/dem_b200.h"

namespace dem {

constexpr int FLAG_FIXED = 1;
// deleted by a DeletionBoundary: also FLAG_FIXED, parked at DELETED_COORD,
// sorted into the graveyard cell (the last cell) at the next rebuild
constexpr int FLAG_DELETED = 2;
// a free row of an insertion boundary: parked like a deleted particle (also
// FLAG_DELETED and FLAG_FIXED) until a placement fills it
constexpr int FLAG_DORMANT = 4;
// the last drift moved the particle across a periodic boundary (set and
// cleared by every drift): the reference's HGrid still files it under its
// cell before the shift until the grid is next updated, which the insertion
// check reproduces
constexpr int FLAG_WRAPPED = 8;
constexpr double DELETED_COORD = 1e300;
constexpr int LEVEL_SHIFT = 8;

struct InstanceDev {
    double origin[3];
    double gravity[3];
    double per_lo[3];
    double per_hi[3];
    double per_L[3];
    double per_half[3];
    uint32_t per_mask;
    int species_offset;
    int n_species;
    int wall_begin;
    int wall_end;
    int n_levels;
    int cell_base[DEM_MAX_LEVELS];
    int dims[DEM_MAX_LEVELS][3];
    double inv_cell[DEM_MAX_LEVELS][3];
    double level_rmax[DEM_MAX_LEVELS];
    // the banding that assigned the levels (radius r: binary exponent of
    // r / level_rmin, clamped to level_bands - 1, through level_remap), for
    // particles placed by insertion boundaries
    double level_rmin;
    int level_bands;
    int level_remap[DEM_MAX_LEVELS];
    double max_interaction_distance;
    // DeletionBoundary planes: a particle is deleted when del_d - x . del_n < 0
    int n_del;
    uint32_t tri_mask;     // walls (bit w = wall_begin + w) that are triangle walls
    // walls (same bits) whose distance field stays put while the simulation
    // runs: no translation, and no rotation or one about the wall's own
    // normal / symmetry axis (infinite and axisymmetric walls). The list
    // rebuild records which of them are within reach + skin of a particle
    // (wcand); k_detect tests the others not at all until the next rebuild
    uint32_t wall_still_mask;
    // walls (same bits) taken out during the run (WallHandler::removeObject):
    // no contacts with them from the next time step on
    uint32_t wall_off_mask;
    int tri_static;        // every triangle wall of the instance stands still: tri_lo/hi hold
    double tri_lo[3], tri_hi[3]; // the bounding box of all their vertices
    double del_n[DEM_MAX_DELETION_PER_INSTANCE][3];
    double del_d[DEM_MAX_DELETION_PER_INSTANCE];
};

// Contact record written at the last force evaluation of a dem_step call:
// one row per contact (particle pairs once, from P's side; wall contacts).
struct ContactRecord {
    int id_p, id_i;
    int is_wall, periodic;
    int slot_p, slot_i;         // sorted indices (slot_i = wall index for walls)
    double overlap;
    double elastic_energy;
    double force[3];
    double contact_point[3];
    double branch[3];           // x_P - x_I (image position for periodic pairs); wall: 0
    double normal[3];           // unit normal of the contact (from I towards P)
    double tangential[3];       // the friction force (part of force)
    double springs[9];
};

struct Control {
    int cur;               // state buffer holding the current state
    int lbuf;              // neighbour-list buffer in use
    int pending_flip;      // the last force kernel wrote the other state buffer
    int rebuild;           // this step rebuilds the neighbour list
    int final_step;        // this step is the last of the dem_step call
    int force_rebuild;     // rebuild at the next control point regardless of displacement
    int record;            // record contacts at final/initial evaluations
    int pad0;
    long long steps_left;
    long long n_rebuilds;
    long long steps_done;  // time steps since the upload
    int first_step;        // this step is the first after the initial evaluation
    int pad1;
    double disp_acc;       // sum of per-step maximum displacements since the last rebuild
    double skin;
    unsigned long long step_disp2_bits; // max |dx|^2 this step (bits of a non-negative double)
    unsigned int status;   // OR of (1u << DEM_ERR_*)
    unsigned int n_records;
    unsigned int record_capacity;
    unsigned int lost_history;
    unsigned int n_items;  // contact items of the current evaluation
    unsigned int n_tri;    // triangle-wall items of the current evaluation (tri_list)
    int pcur;              // spring pool holding the springs of the last evaluation
    unsigned int n_carry;  // first time step: springs kept without a contact (pool top)
};

// Entry-major layouts: entry k of every particle is contiguous, so threads
// of consecutive particles touch consecutive words; the spring components of
// one entry are contiguous (one sector for a contact's history).
__host__ __device__ __forceinline__ size_t nbr_at(int ncap, int i, int k) { return (size_t)k * ncap + i; }
// A spring record holds ncomp doubles padded to an even count (3 -> 4,
// 9 -> 10), so every record starts on 16 bytes and moves as 16-byte vectors.
__host__ __device__ __forceinline__ int hist_stride(int ncomp) { return ncomp + (ncomp & 1); }
__host__ __device__ __forceinline__ size_t pool_at(int ncomp, int j) { return (size_t)j * hist_stride(ncomp); }
__host__ __device__ __forceinline__ size_t whist_at(int ncap, int ncomp, int i, int w)
{
    return ((size_t)w * ncap + i) * hist_stride(ncomp);
}

struct DevPtrs {
    // particle state, two buffers
    double4 *pr[2], *vm[2], *wi[2], *qo[2];
    int4 *info[2];
    int *caller[2];
    // forces of the last force evaluation (3 per particle, sorted order)
    double *force, *torque;
    // neighbour lists, two buffers
    int *nbr[2];
    int *cnt[2];
    // ownership bits of list buffer l, laid out like act: bit k%32 of word
    // own[l][(k/32)*ncap + i] is set when particle i has the lower id of its
    // entry k's pair (it is P unless the pair meets across a periodic boundary)
    unsigned int *own[2];
    // per particle of list buffer l: bit w set when still wall w (above) was
    // within reach + skin at the rebuild (particles move less than skin / 2
    // between rebuilds, so the other still walls cannot be touched)
    unsigned int *wcand[2];
    double *pool[2];        // springs per contact (item_cap records each)
    int *hidx[2];           // per entry: pool index of its contact's spring
    unsigned int *act[2];
    double *whist[2];
    unsigned int *wact[2];
    // broad phase scratch
    int *key, *perm, *newidx, *cell_count, *cell_start, *cell_cursor, *block_sums;
    unsigned long long *rb_barrier; // arrivals at the rebuild's grid barriers (only grows)
    float4 *pf;              // (x, y, z, r) in FP32 of the gathered state: the list build's prefilter
    int *row_slot;           // caller row -> slot of the current order (insertion boundaries only, else null)
    int *rows;               // neighbour lists particle-major (rows[s * cap + k]), for the reverse index
    // tables
    const InstanceDev *inst;
    const dem_species_pair *species;
    dem_wall *walls;         // moved by k_control every step
    const WallGeom *wgeom;   // per wall; faces, edges and corners of intersection walls
    int n_walls;
    int n_instances;
    // compact contact list of one evaluation (dem_pipeline.cuh)
    int *rev;                // reverse index of the neighbour lists, n * cap
    int *slot;               // per entry: item index, or SLOT_NONE / SLOT_IS_I
    int *slotw;              // per (particle, wall): item index or SLOT_NONE
    int4 *items;             // (particle, entry or ITEM_WALL + wall, partner slot, 0);
                             // (particle, ITEM_TRI, triangle-wall hit bits, 0)
    int *tri_list;           // item index of each triangle-wall item (n_tri of them)
    int *slott;              // per particle: its triangle-wall item or SLOT_NONE
    double *tri_first;       // triangle contacts of the initial evaluation, TRI_REC doubles each,
                             // DEM_MAX_TRIANGLE_CONTACTS per particle in caller order (k_tri)
    int *tri_first_n;        // their number per particle (caller order)
    double *shares;          // 12 doubles per item
    int item_cap;
    Control *ctl;
    ContactRecord *records;
    // sizes
    int n;            // particles
    int ncap;         // allocated particle slots (ELL stride)
    int cap;          // neighbour capacity per particle (multiple of 32)
    int nwords;       // cap / 32
    int ncomp;        // history components per contact (3 or 9)
    int wmax;         // max walls per instance
    int ncells;
    int rotation;
    int single_instance;   // one instance: k_contacts stages its record in shared memory
    int n_species_table;   // entries of the species table
    int zero_idist;        // every species pair has interaction distance 0
    int has_tri;           // some wall is a triangle wall (k_tri runs)
    double dt;
    double drag;
};

} // namespace dem
