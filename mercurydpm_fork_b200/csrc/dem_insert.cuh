// dem_insert.cuh -- insertion boundaries (CubeInsertionBoundary and
// ChuteInsertionBoundary) and the chute's compact inflow fill
// (Chute::addFlowParticlesCompactly) on the device.
//
// InsertionBoundary::checkBoundaryBeforeTimeStep (Kernel/Boundaries/
// InsertionBoundary.cc:184-296) is sequential by nature: every draw of the
// random number generators depends on whether the placements before it
// succeeded, and every placement is tested against the particles placed
// before it. k_insert therefore runs one block per instance that has
// insertion boundaries: thread 0 draws and decides, exactly in the
// reference's order, and the whole block tests each candidate (walls, the
// particles of the cells around the candidate and its periodic images, the
// particles placed earlier in the same launch). It runs in every time step
// after k_control (walls moved, state buffers flipped) and before the
// rebuild, which it requests when it placed a particle: that is the
// reference's place in DPMBase::computeOneTimeStep (after the drift, before
// the forces, DPMBase.cc:4348-4352).
//
// The cell table is the one of the last rebuild. A particle has moved less
// than Control::disp_acc (the accumulated per-step maximum displacement)
// since then, so a cell search widened by it finds every particle a
// candidate can touch; the test itself is the exact one on the current
// positions. Particles placed in this launch are not in the cell table yet:
// each is filed in a per-cell list of its own (ovf_head / ovf_next, the cell
// its position and radius give, as keys_one would), which the search walks
// with the cell; the next launch empties the lists it filled (the rebuild of
// the step has put those particles into the table).
//
// One trait of the reference's search is kept: Mercury3D::hGridHasParticleContacts
// (Mercury3D.cc:485-542) looks particles up in the HGrid cells filed at the
// previous step (hGridActionsBeforeTimeStep runs after the insertion), so a
// particle that the drift of this step shifted across a periodic boundary
// sits in a cell on the far side of the period and is not found, until a
// placed particle larger than any the grid was built for makes the grid
// rebuild from the current positions (HGrid::insertParticleToHgrid,
// HGrid.cc:88-118). Such particles (FLAG_WRAPPED) are left out of the test
// in the same way. (A particle that crossed an ordinary cell boundary in the
// step is filed one cell off as well; the reference then misses it only when
// it also lies at the edge of the searched cells, which is left out.)
#pragma once
#include "dem_kernels.cuh"

namespace dem {

constexpr int INS_THREADS = 256;
constexpr double INS_PI = 3.1415926535897932384626433832795; // constants::pi (Kernel/Math/ExtendedMath.h)
// status bit of an insertion that found no free row (not a DEM_ERR_* code)
constexpr int INS_STATUS_NO_ROW = 16;

// ---- Kernel/Math/RNG.cc ----------------------------------------------------
// The reference's default generator: a lagged Fibonacci generator
// x_n = (x_{n-607} + x_{n-273}) mod 1 (RNG::getRandomNumberFromLaggedFibonacciGenerator),
// its 607 lags filled by the linear congruential generator
// s <- (1103515245 s + 12345) mod 2^30, x = s / (2^30 + 1)
// (RNG::seedLaggedFibonacciGenerator after RNG::setRandomSeed). The lags
// live in a ring: `head` is the oldest value, lag 607 - 273 is
// head + 334.
constexpr int LFG_P = 607;
constexpr int LFG_Q = 273;

struct Lfg {
    double v[LFG_P];
    int head;
    int pad;
};

__host__ inline void lfg_seed(uint64_t seed, Lfg& g)
{
    uint64_t s = seed; // unsigned long in the reference (64 bits here)
    const uint64_t a = 1103515245ull, c = 12345ull, m = 1024ull * 1024ull * 1024ull;
    for (int i = 0; i < LFG_P; ++i) {
        s = (a * s + c) % m;
        // min + range * s / (m + 1.0) with min = 0, range = 1
        g.v[i] = 0.0 + 1.0 * (double)s / ((double)m + 1.0);
    }
    g.head = 0;
    g.pad = 0;
}

// RNG::getRandomNumber(lo, hi) = lo + (hi - lo) * x_n.
__host__ __device__ __forceinline__ double lfg_uniform(double* v, int& head, double lo, double hi)
{
    int lag = head + (LFG_P - LFG_Q);
    if (lag >= LFG_P) lag -= LFG_P;
    const double x = fmod(v[head] + v[lag], 1.0);
    v[head] = x;
    head = (head + 1 == LFG_P) ? 0 : head + 1;
    const double range = hi - lo;
    return lo + range * x;
}

// ---- device state ----------------------------------------------------------
struct InsBoundaryDev {
    dem_insertion_boundary b;
    Lfg psd;                  // PSD::random_
    double p0_radius;         // the particle generated and not yet placed (InsertionBoundary::p0)
    double volume_inserted;   // volumeInserted_
    long long n_inserted;     // numberOfParticlesInserted_
    int has_p0;
    int pad;
};

struct InsInstanceDev {
    Lfg rng;                  // DPMBase::random
    double time;              // DPMBase::time_ at the current step
    // the largest radius the reference's HGrid was last rebuilt for: placing a
    // larger particle makes it rebuild (HGrid::insertParticleToHgrid against
    // the top cell nextafter(2 r_max), MercuryBase::hGridRebuild)
    double grid_rmax;
    int instance;
    int first, count;         // its boundaries in InsBoundaryDev order
    int rows_begin, rows_end; // its free rows in the row list
    int next_row;             // the next free row to fill
    int filed_from;           // rows filed in the per-cell lists by the last launch: filed_from .. next_row - 1
};

struct InsPtrs {
    InsInstanceDev* inst;
    InsBoundaryDev* bnd;
    const int* rows;          // free rows (caller order), grouped by instance
    int* ovf_head;            // per cell: a particle placed in this launch, -1: none
    int* ovf_next;            // per slot: the next placed particle of its cell
    int* filed_key;           // per free-row index: the cell its particle was filed in
};

// The cell key keys_one gives a particle of radius r at x (level by radius).
__device__ __forceinline__ int ins_cell_key(const InstanceDev& I, double x, double y, double z, int lvl)
{
    const int cx = cell_coord(x, I.origin[0], I.inv_cell[lvl][0], I.dims[lvl][0], I.per_mask & 1u);
    const int cy = cell_coord(y, I.origin[1], I.inv_cell[lvl][1], I.dims[lvl][1], (I.per_mask >> 1) & 1u);
    const int cz = cell_coord(z, I.origin[2], I.inv_cell[lvl][2], I.dims[lvl][2], (I.per_mask >> 2) & 1u);
    return I.cell_base[lvl] + (cz * I.dims[lvl][1] + cy) * I.dims[lvl][0] + cx;
}

// PSD::drawSample (Kernel/Math/PSD.cc:114-128): std::lower_bound over the
// cumulative probabilities, then a*r_low + (1 - a)*r_high.
__host__ __device__ __forceinline__ double psd_draw(const dem_insertion_boundary& b, double* v, int& head)
{
    const double prob = lfg_uniform(v, head, 0.0, 1.0);
    int hi = 0;
    while (hi < b.n_psd - 1 && b.psd_probability[hi] < prob) ++hi;
    const int lo = hi > 0 ? hi - 1 : 0;
    const double rmin = b.psd_radius[lo], rmax = b.psd_radius[hi];
    const double pmin = b.psd_probability[lo], pmax = b.psd_probability[hi];
    const double a = (prob - pmin) / (pmax - pmin);
    return a * rmin + (1.0 - a) * rmax;
}

// BaseParticle::isInContactWith / getSumOfInteractionRadii (BaseParticle.cc:
// 863-871, BaseParticle.h:383-385): candidate c against particle t.
__device__ __forceinline__ bool ins_overlaps(V3 c, double rc, double4 pt, double idist)
{
    const double X = c.x - pt.x, Y = c.y - pt.y, Z = c.z - pt.z;
    const double sum = rc + pt.w + idist;
    return X * X + Y * Y + Z * Z < sum * sum;
}

// One candidate: its position, its periodic images (the copies
// DPMBase::checkParticleForInteractionLocalPeriodic tests, DPMBase.cc:
// 4868-4904: shifted by the period towards the far side, in every periodic
// direction whose boundary is within reach, and all their combinations).
struct InsCandidate {
    double x[8][3];
    double v[3];
    double r;
    int n_img;
};

// The candidate's periodic images (cand.x[0] set): a copy the reference would
// not make lies farther than reach = r_c + r_max + distance outside the
// period and touches nothing, so making it anyway leaves the test unchanged.
__device__ __forceinline__ void make_images(const InstanceDev& I, double reach, InsCandidate& cand)
{
    int n = 1;
    for (int k = 0; k < 3; ++k) {
        if (!((I.per_mask >> k) & 1u)) continue;
        const double x = cand.x[0][k];
        const double left = I.per_lo[k], right = I.per_hi[k];
        const double dist = fmin(x - left, right - x); // PeriodicBoundary::getDistance
        if (!(dist < reach)) continue;
        // PeriodicBoundary::shiftPosition: towards the far side
        const double shifted = (right - x > x - left) ? x + I.per_L[k] : x - I.per_L[k];
        for (int j = 0; j < n; ++j) {
            for (int a = 0; a < 3; ++a) cand.x[n + j][a] = cand.x[j][a];
            cand.x[n + j][k] = shifted;
        }
        n *= 2;
    }
    cand.n_img = n;
}

// BaseWall::getDistanceAndNormal against every wall of the instance still in
// place, for the candidate and its images (walls split over the threads).
__device__ __forceinline__ bool ins_wall_hit(const DevPtrs& d, const InstanceDev& I, int species,
                                             const InsCandidate& cand)
{
    bool hit = false;
    const int nw = I.wall_end - I.wall_begin;
    for (int w = threadIdx.x; w < nw && !hit; w += blockDim.x) {
        if ((I.wall_off_mask >> w) & 1u) continue;
        const int wg = I.wall_begin + w;
        const dem_wall& wall = d.walls[wg];
        const double idist = d.species[I.species_offset + species * I.n_species + wall.species].interaction_distance;
        const double R = cand.r + idist; // BaseParticle::getWallInteractionRadius
        for (int m = 0; m < cand.n_img && !hit; ++m) {
            const V3 xm = v3(cand.x[m][0], cand.x[m][1], cand.x[m][2]);
            double dist;
            V3 nrm;
            hit = (wall.type == DEM_WALL_TRIANGLE) ? triangle_distance(d.wgeom[wg], xm, R, dist, nrm)
                                                   : wall_distance(wall, d.wgeom + wg, xm, R, dist, nrm);
        }
    }
    return hit;
}

// BaseParticle::computeMass (BaseParticle.cc:874-883) and getVolume
// (:147-166), 3D: the new particle's record in slot t of state buffer c.
__device__ __forceinline__ void ins_place(const DevPtrs& d, const InstanceDev& I, int c, int t, int inst, int species,
                                          double density, const double x[3], const double v[3], double r)
{
    const double im = 1.0 / (4.0 / 3.0 * INS_PI * r * r * r * density);
    const double ii = 1.0 / (.4 * (1.0 / im) * (r * r));
    const int4 old = d.info[c][t];
    d.pr[c][t] = make_double4(x[0], x[1], x[2], r);
    d.vm[c][t] = make_double4(v[0], v[1], v[2], im);
    d.wi[c][t] = make_double4(0.0, 0.0, 0.0, ii);
    d.qo[c][t] = make_double4(1.0, 0.0, 0.0, 0.0);
    d.info[c][t] = make_int4(old.x, species, inst, level_of_radius(I, r) << LEVEL_SHIFT);
    for (int k = 0; k < 3; ++k) {
        d.force[3 * t + k] = 0.0;
        d.torque[3 * t + k] = 0.0;
    }
}

__global__ void __launch_bounds__(INS_THREADS) k_insert(DevPtrs d, InsPtrs ip)
{
    InsInstanceDev& S = ip.inst[blockIdx.x];
    const int inst = S.instance;
    const InstanceDev& I = d.inst[inst];
    Control* ctl = d.ctl;
    const int c = ctl->cur;
    const int tid = threadIdx.x;
    const int ns = I.n_species;

    __shared__ double rng_v[LFG_P];
    __shared__ double psd_v[LFG_P];
    __shared__ int rng_head, psd_head;
    __shared__ InsCandidate cand;
    __shared__ int s_go, s_stop, s_placed, s_next_row, s_fresh;
    for (int k = tid; k < LFG_P; k += blockDim.x) rng_v[k] = S.rng.v[k];
    // empty the per-cell lists the last launch filled
    for (int k = S.filed_from + tid; k < S.next_row; k += blockDim.x) ip.ovf_head[ip.filed_key[k]] = -1;
    if (tid == 0) {
        rng_head = S.rng.head;
        s_placed = 0;
        s_next_row = S.next_row;
        s_fresh = 0; // the reference's grid holds the cells of the previous step
    }
    const int first_row = S.next_row; // rows filled in this launch: first_row .. s_next_row - 1
    const double next_time = S.time + d.dt; // DPMBase::getNextTime
    // reach of the cell search beyond r_c + r_t + interaction distance: the
    // largest displacement since the rebuild (with room for its rounding)
    const double disp = ctl->disp_acc * (1.0 + 1e-9);
    double rmax = 0.0;
    for (int l = 0; l < I.n_levels; ++l) rmax = fmax(rmax, I.level_rmax[l]);
    __syncthreads();

    for (int bi = S.first; bi < S.first + S.count; ++bi) {
        InsBoundaryDev& B = ip.bnd[bi];
        const dem_insertion_boundary& b = B.b;
        for (int k = tid; k < LFG_P; k += blockDim.x) psd_v[k] = B.psd.v[k];
        // thread 0's loop state (InsertionBoundary::checkBoundaryBeforeTimeStep)
        int failed = 0;
        double p0_r = B.p0_radius;
        int has_p0 = B.has_p0;
        double vol = B.volume_inserted;
        long long n_ins = B.n_inserted;
        if (tid == 0) psd_head = B.psd.head;
        __syncthreads();
        auto generate = [&]() { // InsertionBoundary::generateParticle: species draw, then the PSD's
            (void)lfg_uniform(rng_v, rng_head, 0.0, 1.0);
            p0_r = psd_draw(b, psd_v, psd_head);
            has_p0 = 1;
        };
        while (true) {
            if (tid == 0) {
                const bool go = failed <= b.max_failed && vol < b.volume_flow_rate * next_time + b.initial_volume;
                if (go) {
                    if (!has_p0) generate();
                    double x[3];
                    if (b.kind == DEM_INSERTION_CHUTE) { // ChuteInsertionBoundary::placeParticle
                        const double r = p0_r, u = b.inflow_velocity, var = b.inflow_velocity_variance;
                        x[0] = b.pos_min[0] + r;
                        x[1] = lfg_uniform(rng_v, rng_head, b.pos_min[1] - r, b.pos_max[1] + r);
                        x[2] = lfg_uniform(rng_v, rng_head, b.pos_min[2] - r, b.pos_max[2] + r + b.fixed_particle_radius);
                        cand.v[0] = u * lfg_uniform(rng_v, rng_head, -var, var) + u;
                        cand.v[1] = u * lfg_uniform(rng_v, rng_head, -var, var);
                        cand.v[2] = u * lfg_uniform(rng_v, rng_head, -var, var);
                    } else { // CubeInsertionBoundary::placeParticle
                        for (int k = 0; k < 3; ++k) x[k] = lfg_uniform(rng_v, rng_head, b.pos_min[k], b.pos_max[k]);
                        for (int k = 0; k < 3; ++k) cand.v[k] = lfg_uniform(rng_v, rng_head, b.vel_min[k], b.vel_max[k]);
                    }
                    cand.r = p0_r;
                    for (int k = 0; k < 3; ++k) cand.x[0][k] = x[k];
                    make_images(I, p0_r + rmax + I.max_interaction_distance, cand);
                }
                s_go = go ? 1 : 0;
            }
            __syncthreads();
            if (!s_go) break;

            // ---- the test (DPMBase::checkParticleForInteractionLocal): walls,
            // then particles, for the candidate and each image
            const double rc = cand.r;
            const int nimg = cand.n_img;
            bool hit = ins_wall_hit(d, I, b.species, cand);
            // particles of the cells around the candidate and its images
            for (int m = 0; m < nimg && !__syncthreads_or(hit); ++m) {
                const V3 xm = v3(cand.x[m][0], cand.x[m][1], cand.x[m][2]);
                for (int lvl = 0; lvl < I.n_levels; ++lvl) {
                    const double reach = rc + I.level_rmax[lvl] + I.max_interaction_distance + disp;
                    int lo[3], hi[3], nn[3];
                    cell_range(I, lvl, 0, xm.x, reach, lo[0], hi[0]);
                    cell_range(I, lvl, 1, xm.y, reach, lo[1], hi[1]);
                    cell_range(I, lvl, 2, xm.z, reach, lo[2], hi[2]);
                    for (int k = 0; k < 3; ++k) nn[k] = hi[k] - lo[k] + 1;
                    const int ncell = (nn[0] > 0 && nn[1] > 0 && nn[2] > 0) ? nn[0] * nn[1] * nn[2] : 0;
                    for (int q = tid; q < ncell && !hit; q += blockDim.x) {
                        int cc[3] = {lo[0] + q % nn[0], lo[1] + (q / nn[0]) % nn[1], lo[2] + q / (nn[0] * nn[1])};
                        for (int k = 0; k < 3; ++k)
                            if ((I.per_mask >> k) & 1u) cc[k] = wrap_cell(cc[k], I.dims[lvl][k]);
                        const int key = I.cell_base[lvl] + (cc[2] * I.dims[lvl][1] + cc[1]) * I.dims[lvl][0] + cc[0];
                        const int e = d.cell_start[key + 1];
                        for (int t = d.cell_start[key]; t < e && !hit; ++t) {
                            const int4 it = d.info[c][t];
                            if (it.w & FLAG_DELETED) continue;
                            if ((it.w & FLAG_WRAPPED) && !s_fresh) continue; // filed on the far side
                            const double idist =
                                d.species[I.species_offset + b.species * ns + it.y].interaction_distance;
                            hit = ins_overlaps(xm, rc, d.pr[c][t], idist);
                        }
                        for (int t = ip.ovf_head[key]; t >= 0 && !hit; t = ip.ovf_next[t]) { // placed in this launch
                            const double idist =
                                d.species[I.species_offset + b.species * ns + d.info[c][t].y].interaction_distance;
                            hit = ins_overlaps(xm, rc, d.pr[c][t], idist);
                        }
                    }
                }
            }
            hit = __syncthreads_or(hit);

            if (tid == 0) {
                s_stop = 0;
                if (!hit) {
                    if (s_next_row < S.rows_end) {
                        const int t = d.row_slot[ip.rows[s_next_row]];
                        const double r = cand.r;
                        ins_place(d, I, c, t, inst, b.species, b.density, cand.x[0], cand.v, r);
                        const int key = ins_cell_key(I, cand.x[0][0], cand.x[0][1], cand.x[0][2], level_of_radius(I, r));
                        ip.ovf_next[t] = ip.ovf_head[key];
                        ip.ovf_head[key] = t;
                        ip.filed_key[s_next_row] = key;
                        if (r > S.grid_rmax) { // the next test finds the grid rebuilt
                            S.grid_rmax = r;
                            s_fresh = 1;
                        }
                        ++s_next_row;
                        s_placed = 1;
                        failed = 0;
                        ++n_ins;
                        vol += 4.0 / 3.0 * INS_PI * r * r * r;
                        generate(); // the next particle is drawn at once
                    } else {
                        atomicOr(&ctl->status, 1u << INS_STATUS_NO_ROW);
                        s_stop = 1;
                    }
                } else {
                    ++failed;
                }
            }
            __syncthreads();
            if (s_stop) break;
        }
        // the boundary's state for the next step
        for (int k = tid; k < LFG_P; k += blockDim.x) B.psd.v[k] = psd_v[k];
        if (tid == 0) {
            B.psd.head = psd_head;
            B.p0_radius = p0_r;
            B.has_p0 = has_p0;
            B.volume_inserted = vol;
            B.n_inserted = n_ins;
        }
        __syncthreads();
    }
    for (int k = tid; k < LFG_P; k += blockDim.x) S.rng.v[k] = rng_v[k];
    if (tid == 0) {
        S.rng.head = rng_head;
        S.filed_from = first_row;
        S.next_row = s_next_row;
        S.time = next_time; // DPMBase::time_ += timeStep_ at the end of the step
        if (s_placed) ctl->rebuild = 1; // the new particles need cells and lists
    }
}

// ---------------------------------------------------------------------------
// Chute::addFlowParticlesCompactly (Kernel/Chute.cc:1083-1102), run once by
// the upload. Particles do not move during the fill, so a plain linked-list
// grid of the instance (cells of at least the largest reach) holds every
// particle, the placed ones added as they come, like the reference's HGrid.
// ---------------------------------------------------------------------------
struct FillGrid {
    int* head;           // per cell: the first particle (slot), -1: empty
    int* next;           // per slot: the next particle of its cell
    double origin[3];
    double inv[3];       // cells per unit length
    int dims[3];
};

struct FillDev {
    dem_chute_fill f;
    long long target;    // particles to place: N minus the particles in the instance
    double height;       // Chute::inflowHeight_, grown by failed candidates
    long long added;
    long long tries_left;// bound on the candidates (a fill that cannot finish stops)
    int status;          // 0 done, 1 no free row left, 2 gave up
    int instance_slot;   // its InsInstanceDev (the instance's generator)
};

__device__ __forceinline__ int fill_coord(const FillGrid& g, int k, double x, bool periodic)
{
    const double f = floor((x - g.origin[k]) * g.inv[k]);
    if (periodic) {
        if (!(fabs(f) < 1e9)) return 0;
        return wrap_cell((int)f, g.dims[k]);
    }
    if (!(f >= 0.0)) return 0;
    if (f >= (double)(g.dims[k] - 1)) return g.dims[k] - 1;
    return (int)f;
}

__device__ __forceinline__ int fill_cell(const FillGrid& g, uint32_t pm, V3 x)
{
    const int cx = fill_coord(g, 0, x.x, pm & 1u), cy = fill_coord(g, 1, x.y, (pm >> 1) & 1u),
              cz = fill_coord(g, 2, x.z, (pm >> 2) & 1u);
    return (cz * g.dims[1] + cy) * g.dims[0] + cx;
}

// every particle of the instance already in the state (buffer c) into the grid
__global__ void __launch_bounds__(256) k_fill_grid(DevPtrs d, FillGrid g, int inst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int c = d.ctl->cur;
    const int4 f = d.info[c][i];
    if (f.z != inst || (f.w & FLAG_DELETED)) return;
    const int cell = fill_cell(g, d.inst[inst].per_mask, xyz(d.pr[c][i]));
    g.next[i] = atomicExch(&g.head[cell], i);
}

__global__ void __launch_bounds__(INS_THREADS) k_fill(DevPtrs d, InsPtrs ip, FillDev* F, FillGrid g)
{
    FillDev& fd = *F;
    const dem_chute_fill& f = fd.f;
    InsInstanceDev& S = ip.inst[fd.instance_slot];
    const int inst = f.instance;
    const InstanceDev& I = d.inst[inst];
    const int c = d.ctl->cur;
    const int tid = threadIdx.x;
    __shared__ double rng_v[LFG_P];
    __shared__ int rng_head, s_go;
    __shared__ InsCandidate cand;
    for (int k = tid; k < LFG_P; k += blockDim.x) rng_v[k] = S.rng.v[k];
    double rmax = 0.0;
    for (int l = 0; l < I.n_levels; ++l) rmax = fmax(rmax, I.level_rmax[l]);
    // thread 0's loop state
    double height = f.inflow_height;
    long long added = 0, tries = fd.tries_left;
    int next_row = S.next_row;
    int status = 0;
    if (tid == 0) rng_head = S.rng.head;
    __syncthreads();
    while (true) {
        if (tid == 0) {
            bool go = added < fd.target;
            if (go && next_row >= S.rows_end) { status = 1; go = false; }
            if (go && tries-- <= 0) { status = 2; go = false; }
            if (go) { // Chute::createFlowParticle: radius, then z, y, x (g++'s argument order)
                const double r = lfg_uniform(rng_v, rng_head, f.min_radius, f.max_radius);
                double x[3];
                x[2] = lfg_uniform(rng_v, rng_head, f.z_min + r + f.fixed_particle_radius, height);
                x[1] = lfg_uniform(rng_v, rng_head, f.y_min + r, f.y_max - r);
                x[0] = lfg_uniform(rng_v, rng_head, f.x_min + r, f.x_max - r);
                cand.r = r;
                for (int k = 0; k < 3; ++k) {
                    cand.x[0][k] = x[k];
                    cand.v[k] = 0.0;
                }
                make_images(I, r + rmax + I.max_interaction_distance, cand);
            }
            s_go = go ? 1 : 0;
        }
        __syncthreads();
        if (!s_go) break;
        bool hit = ins_wall_hit(d, I, f.species, cand);
        const double rc = cand.r;
        const double reach = rc + rmax + I.max_interaction_distance;
        for (int m = 0; m < cand.n_img && !__syncthreads_or(hit); ++m) {
            const V3 xm = v3(cand.x[m][0], cand.x[m][1], cand.x[m][2]);
            int lo[3], nn[3];
            const double xc[3] = {xm.x, xm.y, xm.z};
            for (int k = 0; k < 3; ++k) {
                const bool per = (I.per_mask >> k) & 1u;
                const double flo = floor((xc[k] - reach - g.origin[k]) * g.inv[k]);
                const double fhi = floor((xc[k] + reach - g.origin[k]) * g.inv[k]);
                if (per) {
                    if (!(fhi - flo + 1.0 <= (double)g.dims[k]) || !(fabs(flo) < 1e9)) {
                        lo[k] = 0;
                        nn[k] = g.dims[k];
                    } else {
                        lo[k] = (int)flo;
                        nn[k] = (int)(fhi - flo) + 1;
                    }
                } else {
                    const int a = !(flo >= 0.0) ? 0 : (flo > (double)(g.dims[k] - 1) ? g.dims[k] - 1 : (int)flo);
                    const int b = !(fhi >= 0.0) ? 0 : (fhi > (double)(g.dims[k] - 1) ? g.dims[k] - 1 : (int)fhi);
                    lo[k] = a;
                    nn[k] = b - a + 1;
                }
            }
            const int ncell = nn[0] * nn[1] * nn[2];
            for (int q = tid; q < ncell && !hit; q += blockDim.x) {
                int cc[3] = {lo[0] + q % nn[0], lo[1] + (q / nn[0]) % nn[1], lo[2] + q / (nn[0] * nn[1])};
                for (int k = 0; k < 3; ++k)
                    if ((I.per_mask >> k) & 1u) cc[k] = wrap_cell(cc[k], g.dims[k]);
                int t = g.head[(cc[2] * g.dims[1] + cc[1]) * g.dims[0] + cc[0]];
                while (t >= 0 && !hit) {
                    const int4 it = d.info[c][t];
                    const double idist =
                        d.species[I.species_offset + f.species * I.n_species + it.y].interaction_distance;
                    hit = ins_overlaps(xm, rc, d.pr[c][t], idist);
                    t = g.next[t];
                }
            }
        }
        hit = __syncthreads_or(hit);
        if (tid == 0) {
            if (!hit) {
                const int t = d.row_slot[ip.rows[next_row]];
                ins_place(d, I, c, t, inst, f.species, f.density, cand.x[0], cand.v, cand.r);
                S.grid_rmax = fmax(S.grid_rmax, cand.r);
                const int cell = fill_cell(g, I.per_mask, v3(cand.x[0][0], cand.x[0][1], cand.x[0][2]));
                g.next[t] = g.head[cell];
                g.head[cell] = t;
                ++next_row;
                ++added;
            } else {
                height = height + .0001 * f.max_radius; // Chute::setInflowHeight
            }
        }
        __syncthreads();
    }
    for (int k = tid; k < LFG_P; k += blockDim.x) S.rng.v[k] = rng_v[k];
    if (tid == 0) {
        S.rng.head = rng_head;
        S.next_row = next_row;
        S.filed_from = next_row; // the fill files in its own grid, not in the per-cell lists
        fd.height = height;
        fd.added = added;
        fd.tries_left = tries;
        fd.status = status;
    }
}

} // namespace dem
