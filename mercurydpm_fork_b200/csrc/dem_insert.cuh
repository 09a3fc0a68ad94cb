// dem_insert.cuh -- insertion boundaries (CubeInsertionBoundary) on the device.
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
// positions. Particles placed in this launch are not in any cell yet: they
// are the free rows used so far, tested one by one.
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
    int instance;
    int first, count;         // its boundaries in InsBoundaryDev order
    int rows_begin, rows_end; // its free rows in the row list
    int next_row;             // the next free row to fill
    int pad;
};

struct InsPtrs {
    InsInstanceDev* inst;
    InsBoundaryDev* bnd;
    const int* rows;          // free rows (caller order), grouped by instance
};

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

// The HGrid level of radius r under the instance's banding (the host's
// setup_instance_grid made sure every band the PSD reaches has a level).
__device__ __forceinline__ int level_of_radius(const InstanceDev& I, double r)
{
    const double x = r / I.level_rmin;
    int l = (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
    l = l < 0 ? 0 : (l > I.level_bands - 1 ? I.level_bands - 1 : l);
    const int m = I.level_remap[l];
    return m < 0 ? 0 : m;
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

__global__ void __launch_bounds__(INS_THREADS) k_insert(DevPtrs d, InsPtrs ip)
{
    InsInstanceDev& S = ip.inst[blockIdx.x];
    const int inst = S.instance;
    const InstanceDev& I = d.inst[inst];
    Control* ctl = d.ctl;
    const int c = ctl->cur;
    const int tid = threadIdx.x;
    const int ns = I.n_species;
    const int nw = I.wall_end - I.wall_begin;

    __shared__ double rng_v[LFG_P];
    __shared__ double psd_v[LFG_P];
    __shared__ int rng_head, psd_head;
    __shared__ InsCandidate cand;
    __shared__ int s_go, s_stop, s_placed, s_next_row;
    for (int k = tid; k < LFG_P; k += blockDim.x) rng_v[k] = S.rng.v[k];
    if (tid == 0) {
        rng_head = S.rng.head;
        s_placed = 0;
        s_next_row = S.next_row;
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
                    // CubeInsertionBoundary::placeParticle
                    double x[3];
                    for (int k = 0; k < 3; ++k) x[k] = lfg_uniform(rng_v, rng_head, b.pos_min[k], b.pos_max[k]);
                    for (int k = 0; k < 3; ++k) cand.v[k] = lfg_uniform(rng_v, rng_head, b.vel_min[k], b.vel_max[k]);
                    cand.r = p0_r;
                    for (int k = 0; k < 3; ++k) cand.x[0][k] = x[k];
                    int n = 1;
                    // periodic images; a copy the reference would not make lies
                    // farther than r_c + r_max + distance outside the period and
                    // touches nothing, so the wider test below is the same test
                    const double reach = p0_r + rmax + I.max_interaction_distance;
                    for (int k = 0; k < 3; ++k) {
                        if (!((I.per_mask >> k) & 1u)) continue;
                        const double left = I.per_lo[k], right = I.per_hi[k];
                        const double dist = fmin(x[k] - left, right - x[k]); // PeriodicBoundary::getDistance
                        if (!(dist < reach)) continue;
                        // PeriodicBoundary::shiftPosition: towards the far side
                        const double shifted = (right - x[k] > x[k] - left) ? x[k] + I.per_L[k] : x[k] - I.per_L[k];
                        for (int j = 0; j < n; ++j) {
                            for (int a = 0; a < 3; ++a) cand.x[n + j][a] = cand.x[j][a];
                            cand.x[n + j][k] = shifted;
                        }
                        n *= 2;
                    }
                    cand.n_img = n;
                }
                s_go = go ? 1 : 0;
            }
            __syncthreads();
            if (!s_go) break;

            // ---- the test (DPMBase::checkParticleForInteractionLocal): walls,
            // then particles, for the candidate and each image
            bool hit = false;
            const double rc = cand.r;
            const int nimg = cand.n_img;
            for (int w = tid; w < nw && !hit; w += blockDim.x) {
                if ((I.wall_off_mask >> w) & 1u) continue;
                const int wg = I.wall_begin + w;
                const dem_wall& wall = d.walls[wg];
                const double idist = d.species[I.species_offset + b.species * ns + wall.species].interaction_distance;
                const double R = rc + idist; // BaseParticle::getWallInteractionRadius
                for (int m = 0; m < nimg && !hit; ++m) {
                    const V3 xm = v3(cand.x[m][0], cand.x[m][1], cand.x[m][2]);
                    double dist;
                    V3 nrm;
                    hit = (wall.type == DEM_WALL_TRIANGLE) ? triangle_distance(d.wgeom[wg], xm, R, dist, nrm)
                                                           : wall_distance(wall, d.wgeom + wg, xm, R, dist, nrm);
                }
            }
            // particles placed earlier in this launch
            for (int k = first_row + tid; k < s_next_row && !hit; k += blockDim.x) {
                const int t = d.row_slot[ip.rows[k]];
                const double4 pt = d.pr[c][t];
                const int4 it = d.info[c][t];
                const double idist = d.species[I.species_offset + b.species * ns + it.y].interaction_distance;
                for (int m = 0; m < nimg && !hit; ++m)
                    hit = ins_overlaps(v3(cand.x[m][0], cand.x[m][1], cand.x[m][2]), rc, pt, idist);
            }
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
                            const double idist =
                                d.species[I.species_offset + b.species * ns + it.y].interaction_distance;
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
                        const int row = ip.rows[s_next_row];
                        const int t = d.row_slot[row];
                        const double r = cand.r;
                        // BaseParticle::computeMass (BaseParticle.cc:874-883), getVolume (:147-166)
                        const double im = 1.0 / (4.0 / 3.0 * INS_PI * r * r * r * b.density);
                        const double ii = 1.0 / (.4 * (1.0 / im) * (r * r));
                        const int4 old = d.info[c][t];
                        d.pr[c][t] = make_double4(cand.x[0][0], cand.x[0][1], cand.x[0][2], r);
                        d.vm[c][t] = make_double4(cand.v[0], cand.v[1], cand.v[2], im);
                        d.wi[c][t] = make_double4(0.0, 0.0, 0.0, ii);
                        d.qo[c][t] = make_double4(1.0, 0.0, 0.0, 0.0);
                        d.info[c][t] = make_int4(old.x, b.species, inst, level_of_radius(I, r) << LEVEL_SHIFT);
                        for (int k = 0; k < 3; ++k) {
                            d.force[3 * t + k] = 0.0;
                            d.torque[3 * t + k] = 0.0;
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
        S.next_row = s_next_row;
        S.time = next_time; // DPMBase::time_ += timeStep_ at the end of the step
        if (s_placed) ctl->rebuild = 1; // the new particles need cells and lists
    }
}

} // namespace dem
