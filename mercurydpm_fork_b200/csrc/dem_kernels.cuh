// dem_kernels.cuh -- the DEM time-step kernels.
//
// Per time step (captured in a CUDA graph):
//   k_control   moves the walls (one thread per wall); one thread applies
//               the pending state-buffer flip, adds the last step's maximum
//               displacement to the skin budget and sets the rebuild flag
//               (MercuryBase::hGridNeedsRebuilding, MercuryBase.cc:496-535,
//               turned into a Verlet-skin test).
//   k_rebuild   one cooperative kernel, launched every step and returning at
//               once unless the flag is set (dem_rebuild.cuh): cell keys per
//               HGrid level, counting sort, per-cell ordering by particle id,
//               permutation gather of the state, neighbour lists with
//               contact-history carry-over, their reverse index (replaces
//               HGrid buckets + InteractionHandler lookup, Mercury3D.cc:224-416,
//               InteractionHandler.cc:103-174). The per-item steps are below.
//   force       k_detect -> k_contacts -> k_sum (dem_pipeline.cuh): the exact
//               FP64 contact predicate (BaseParticle::getInteractionWith,
//               BaseParticle.cc:688-710) on the entries each particle owns,
//               the contact law once per contact with its spring history,
//               the ordered sums with body force and walls, and the
//               integration (second half-kick of this step, then first
//               half-kick and drift of the next one: BaseParticle.cc:718-776)
//               into the other state buffer.
#pragma once
#include "dem_engine.cuh"
#include "dem_laws.cuh"

namespace dem {

__device__ __forceinline__ V3 xyz(double4 a) { return V3{a.x, a.y, a.z}; }

// ---------------------------------------------------------------------------
// control
// ---------------------------------------------------------------------------
__global__ void k_control(Control* ctl, dem_wall* walls, WallGeom* wgeom, int n_walls, double dt)
{
    // Walls move before the force evaluation of every step, after the particles
    // (DPMBase::integrateBeforeForceComputation, DPMBase.cc:3228-3261, through
    // BaseInteractable::integrateBeforeForceComputation, BaseInteractable.cc:538-600:
    // move(v dt), then rotate(omega dt) = Quaternion::updateAngularDisplacement).
    // A triangle wall then recomputes its vertices and normals
    // (TriangleWall::move / rotate -> updateVertexAndNormal).
    for (int k = threadIdx.x; k < n_walls; k += blockDim.x) {
        dem_wall& w = walls[k];
        for (int a = 0; a < 3; ++a) w.position[a] += w.velocity[a] * dt;
        const Q4 q = quat_rotate(Q4{w.orientation[0], w.orientation[1], w.orientation[2], w.orientation[3]},
                                 v3(w.angular_velocity[0] * dt, w.angular_velocity[1] * dt, w.angular_velocity[2] * dt));
        w.orientation[0] = q.q0; w.orientation[1] = q.q1; w.orientation[2] = q.q2; w.orientation[3] = q.q3;
        const bool still = w.velocity[0] == 0.0 && w.velocity[1] == 0.0 && w.velocity[2] == 0.0 &&
                           w.angular_velocity[0] == 0.0 && w.angular_velocity[1] == 0.0 &&
                           w.angular_velocity[2] == 0.0; // nothing moved: the geometry stands
        if (w.type == DEM_WALL_TRIANGLE && !still) triangle_geometry(w, wgeom[k]);
    }
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (ctl->pending_flip) { // a force evaluation wrote the other state buffer and spring pool
        ctl->cur ^= 1;
        ctl->pcur ^= 1;
        ctl->pending_flip = 0;
    }
    const double d = sqrt(__longlong_as_double((long long)ctl->step_disp2_bits));
    ctl->step_disp2_bits = 0ull;
    ctl->disp_acc += d;
    const int rebuild = ctl->force_rebuild || (2.0 * ctl->disp_acc >= ctl->skin);
    ctl->rebuild = rebuild;
    ctl->force_rebuild = 0;
    ctl->final_step = (ctl->steps_left <= 1);
    ctl->steps_left -= 1;
    if (ctl->final_step) ctl->n_records = 0; // records describe the last evaluation only
    ctl->first_step = (ctl->steps_done == 0);
    ctl->steps_done += 1;
    ctl->pending_flip = 1; // the force kernel of this step writes the other buffer
}

__global__ void k_flip(Control* ctl)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (ctl->pending_flip) { // a force evaluation wrote the other state buffer and spring pool
        ctl->cur ^= 1;
        ctl->pcur ^= 1;
        ctl->pending_flip = 0;
    }
}

// ---------------------------------------------------------------------------
// broad phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ int cell_coord(double x, double origin, double inv, int dim, bool periodic)
{
    const double f = floor((x - origin) * inv);
    // periodic: a particle just outside the period (an insertion may place one
    // there; the next drift shifts it back) is filed in the cell the searches
    // reach it in, the wrapped one
    if (periodic && fabs(f) < 1e9) {
        const int c = (int)f % dim;
        return c < 0 ? c + dim : c;
    }
    // positions far outside the grid are clamped into the edge cells
    if (!(f >= 0.0)) return 0;
    if (f >= (double)(dim - 1)) return dim - 1;
    return (int)f;
}

// ---- the steps of a rebuild, one item each (run by k_rebuild, dem_rebuild.cuh) ----

// Cell key of particle i (state buffer c) and its count.
__device__ __forceinline__ void keys_one(const DevPtrs& d, int i, int c)
{
    const double4 p = d.pr[c][i];
    const int4 inf = d.info[c][i];
    if (inf.w & FLAG_DELETED) { // the graveyard: the last cell, never searched
        d.key[i] = d.ncells - 1;
        atomicAdd(&d.cell_count[d.ncells - 1], 1);
        return;
    }
    const InstanceDev& I = d.inst[inf.z];
    const int lvl = (inf.w >> LEVEL_SHIFT) & 0xff;
    const int cx = cell_coord(p.x, I.origin[0], I.inv_cell[lvl][0], I.dims[lvl][0], I.per_mask & 1u);
    const int cy = cell_coord(p.y, I.origin[1], I.inv_cell[lvl][1], I.dims[lvl][1], (I.per_mask >> 1) & 1u);
    const int cz = cell_coord(p.z, I.origin[2], I.inv_cell[lvl][2], I.dims[lvl][2], (I.per_mask >> 2) & 1u);
    const int key = I.cell_base[lvl] + (cz * I.dims[lvl][1] + cy) * I.dims[lvl][0] + cx;
    d.key[i] = key;
    atomicAdd(&d.cell_count[key], 1);
}

// Slot of particle i in the counting sort.
__device__ __forceinline__ void scatter_one(const DevPtrs& d, int i)
{
    const int key = d.key[i];
    const int slot = d.cell_start[key] + atomicAdd(&d.cell_cursor[key], 1);
    d.perm[slot] = i;
}

// Orders the members of every cell by particle id, so the sorted order (and
// with it every neighbour list and force sum) does not depend on the order in
// which the atomics above were served. Resets the counters for the next rebuild.
__device__ __forceinline__ void cell_sort_one(const DevPtrs& d, int cell, int c)
{
    const int b = d.cell_start[cell], e = d.cell_start[cell + 1];
    d.cell_count[cell] = 0;
    d.cell_cursor[cell] = 0;
    if (e - b < 2 || cell == d.ncells - 1) return; // the graveyard is not ordered
    if (e - b > 512) { // pathological pile-up (e.g. particles far outside the grid)
        atomicOr(&d.ctl->status, 1u << DEM_ERR_DOMAIN);
        return;
    }
    for (int a = b + 1; a < e; ++a) {
        const int v = d.perm[a];
        const int id = d.info[c][v].x;
        int k = a - 1;
        while (k >= b && d.info[c][d.perm[k]].x > id) {
            d.perm[k + 1] = d.perm[k];
            --k;
        }
        d.perm[k + 1] = v;
    }
}

// State of slot s gathered from buffer c into the other buffer.
__device__ __forceinline__ void gather_one(const DevPtrs& d, int s, int c)
{
    const int nb = c ^ 1;
    const int o = d.perm[s];
    const double4 p = d.pr[c][o];
    const int4 inf = d.info[c][o];
    d.pr[nb][s] = p;
    const double* g = d.inst[inf.z].origin; // relative to the grid origin: small magnitudes in FP32
    d.pf[s] = make_float4((float)(p.x - g[0]), (float)(p.y - g[1]), (float)(p.z - g[2]), (float)p.w);
    d.vm[nb][s] = d.vm[c][o];
    d.wi[nb][s] = d.wi[c][o];
    d.qo[nb][s] = d.qo[c][o];
    d.info[nb][s] = inf;
    d.caller[nb][s] = d.caller[c][o];
    if (d.row_slot) d.row_slot[d.caller[c][o]] = s;
    d.newidx[o] = s;
}

// Minimum-image position of particle t as seen from position xs, with the
// rounding of a periodic ghost: x_t +- L (PeriodicBoundary::shiftPosition,
// PeriodicBoundary.cc:219-229).
__device__ __forceinline__ V3 image_of(const InstanceDev& I, V3 xs, V3 xt, bool& periodic)
{
    periodic = false;
    if (I.per_mask) {
        double* c = &xt.x;
        const double* s = &xs.x;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if ((I.per_mask >> k) & 1u) {
                const double raw = s[k] - c[k];
                if (raw > I.per_half[k]) {
                    c[k] = c[k] + I.per_L[k];
                    periodic = true;
                } else if (raw < -I.per_half[k]) {
                    c[k] = c[k] - I.per_L[k];
                    periodic = true;
                }
            }
        }
    }
    return xt;
}

__device__ __forceinline__ void cell_range(const InstanceDev& I, int lvl, int k, double x, double reach, int& lo,
                                           int& hi)
{
    const int dim = I.dims[lvl][k];
    const double inv = I.inv_cell[lvl][k];
    const double flo = floor((x - reach - I.origin[k]) * inv);
    const double fhi = floor((x + reach - I.origin[k]) * inv);
    if ((I.per_mask >> k) & 1u) {
        // periodic: wrap, but visit each cell at most once; non-finite or far
        // away coordinates (a diverging run) fall back to the whole row, so
        // the loop bounds always stay small integers
        double span = fhi - flo + 1.0;
        if (!(span <= (double)dim) || !(fabs(flo) < 1e9) || !(fabs(fhi) < 1e9)) {
            lo = 0;
            hi = dim - 1;
        } else {
            lo = (int)flo;
            hi = (int)fhi;
        }
    } else {
        lo = (flo < 0.0) ? 0 : ((flo > (double)(dim - 1)) ? dim - 1 : (int)flo);
        hi = (fhi < 0.0) ? 0 : ((fhi > (double)(dim - 1)) ? dim - 1 : (int)fhi);
    }
}

__device__ __forceinline__ int wrap_cell(int c, int dim)
{
    if ((unsigned)c < (unsigned)dim) return c;
    const int once = c < 0 ? c + dim : c - dim; // a range one period beyond the grid
    if ((unsigned)once < (unsigned)dim) return once;
    c %= dim;
    return c < 0 ? c + dim : c;
}

// Sets bit m of a 4-word mask held in registers.
__device__ __forceinline__ void set_bit4(unsigned int& w0, unsigned int& w1, unsigned int& w2, unsigned int& w3, int m)
{
    const unsigned int bit = 1u << (m & 31);
    const int w = m >> 5;
    if (w == 0) w0 |= bit;
    else if (w == 1) w1 |= bit;
    else if (w == 2) w2 |= bit;
    else w3 |= bit;
}

// Slot ranges of one (z, y) row of cells between x cells lo..hi: one range,
// or two when a periodic row wraps (the second empty otherwise).
__device__ __forceinline__ void row_ranges(const DevPtrs& d, const InstanceDev& I, int lvl, int row, int lo, int hi,
                                           int& b0, int& e0, int& b1, int& e1)
{
    const int dx = I.dims[lvl][0];
    int l0 = lo, h0 = hi, l1 = 0, h1 = -1;
    if (I.per_mask & 1u) {
        if (lo < 0) {
            l0 = lo + dx; h0 = dx - 1;
            l1 = 0; h1 = hi;
        } else if (hi >= dx) {
            l0 = lo; h0 = dx - 1;
            l1 = 0; h1 = hi - dx;
        }
    }
    b0 = d.cell_start[row + l0];
    e0 = d.cell_start[row + h0 + 1];
    if (h1 >= l1) {
        b1 = d.cell_start[row + l1];
        e1 = d.cell_start[row + h1 + 1];
    } else {
        b1 = e1 = 0;
    }
}

// Neighbour list of one particle: every particle of the cells within reach
// whose distance is below r_s + r_t + interaction distance + skin, in
// cell-row order. The distance test runs in FP32 on the `pf` copy
// (coordinates relative to the grid origin) with a margin that bounds its
// rounding (16 units of FP32 rounding on the cut and on the magnitudes of the
// coordinates and the period), so the list is a superset of the FP64 test's
// list; pairs whose periodic image is ambiguous in FP32, or whose margin
// exceeds 1/16 of the cut (coordinates very large against the particles),
// take the FP64 test. Contacts themselves are always decided in FP64
// by the force evaluation, so the superset changes no result. The next row's
// slot ranges are read ahead and candidates are read BUILD_BATCH at a time.
constexpr int BUILD_BATCH = 2;
__device__ __forceinline__ void build_one(const DevPtrs& d, int s, int hc, int lo_)
{
    // hc: old state order and its history; lo_: old lists
    const int nb = hc ^ 1;             // gathered (new) state; new history
    const int ln = lo_ ^ 1;            // new lists
    const double4 ps = d.pr[nb][s];
    const int4 is = d.info[nb][s];
    const InstanceDev& I = d.inst[is.z];
    const V3 xs = xyz(ps);
    const bool fixed_s = (is.w & FLAG_FIXED) != 0;
    if (is.w & FLAG_DELETED) {
        d.cnt[ln][s] = 0;
        d.wcand[ln][s] = 0u;
        for (int w = 0; w < d.nwords; ++w) d.act[nb][(size_t)w * d.ncap + s] = 0u;
        d.wact[nb][s] = 0u;
        return;
    }
    const double extra = I.max_interaction_distance + d.ctl->skin;
    const float4 fs = d.pf[s];
    const float ms = fmaxf(fabsf(fs.x), fmaxf(fabsf(fs.y), fabsf(fs.z)));
    const float extra_f = (float)extra;
    const unsigned int pm = I.per_mask;
    float Lf[3], hf[3], lmax = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Lf[k] = (float)I.per_L[k];
        hf[k] = (float)I.per_half[k];
        if ((pm >> k) & 1u) lmax = fmaxf(lmax, fabsf(Lf[k]));
    }
    constexpr float U20 = 9.5367431640625e-07f; // 2^-20
    int count = 0;
    bool overflow = false;
    unsigned int ownw = 0u; // ownership bits of the list word being filled
    for (int lvl = 0; lvl < I.n_levels; ++lvl) {
        const double reach = ps.w + I.level_rmax[lvl] + extra;
        int lox, hix, loy, hiy, loz, hiz;
        cell_range(I, lvl, 0, xs.x, reach, lox, hix);
        cell_range(I, lvl, 1, xs.y, reach, loy, hiy);
        cell_range(I, lvl, 2, xs.z, reach, loz, hiz);
        const int dx = I.dims[lvl][0], dy = I.dims[lvl][1], dz = I.dims[lvl][2];
        const int ny = hiy - loy + 1, nz = hiz - loz + 1;
        const int nrows = (ny > 0 && nz > 0) ? ny * nz : 0;
        auto row_of = [&](int cz, int cy) {
            const int wz = ((pm >> 2) & 1u) ? wrap_cell(cz, dz) : cz;
            const int wy = ((pm >> 1) & 1u) ? wrap_cell(cy, dy) : cy;
            return I.cell_base[lvl] + (wz * dy + wy) * dx;
        };
        int cz = loz, cy = loy;
        int nb0 = 0, ne0 = 0, nb1 = 0, ne1 = 0;
        if (nrows > 0) row_ranges(d, I, lvl, row_of(cz, cy), lox, hix, nb0, ne0, nb1, ne1);
        for (int r = 0; r < nrows; ++r) {
            const int b0 = nb0, e0 = ne0, b1 = nb1, e1 = ne1;
            int ncy = cy + 1, ncz = cz;
            if (ncy > hiy) {
                ncy = loy;
                ++ncz;
            }
            if (r + 1 < nrows) row_ranges(d, I, lvl, row_of(ncz, ncy), lox, hix, nb0, ne0, nb1, ne1);
            cy = ncy;
            cz = ncz;
            for (int g = 0; g < 2; ++g) {
                const int b = g ? b1 : b0, e = g ? e1 : e0;
                for (int t0 = b; t0 < e; t0 += BUILD_BATCH) {
                    float4 ftb[BUILD_BATCH];
#pragma unroll
                    for (int j = 0; j < BUILD_BATCH; ++j)
                        if (t0 + j < e) ftb[j] = d.pf[t0 + j];
#pragma unroll
                    for (int j = 0; j < BUILD_BATCH; ++j) {
                        const int t = t0 + j;
                        if (t >= e) break;
                        if (t == s) continue;
                        if (fixed_s && (d.info[nb][t].w & FLAG_FIXED)) continue; // DPMBase.cc:3116-3120
                        const float4 ft = ftb[j];
                        const float mt = fmaxf(fabsf(ft.x), fmaxf(fabsf(ft.y), fabsf(ft.z)));
                        const float err = U20 * ((ms + mt) + lmax);
                        float bq[3] = {fs.x - ft.x, fs.y - ft.y, fs.z - ft.z};
                        bool ambiguous = false;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            if ((pm >> k) & 1u) {
                                ambiguous = ambiguous || fabsf(fabsf(bq[k]) - hf[k]) <= 4.0f * err;
                                if (bq[k] > hf[k]) bq[k] = bq[k] - Lf[k];
                                else if (bq[k] < -hf[k]) bq[k] = bq[k] + Lf[k];
                            }
                        }
                        bool near;
                        const float cut = (fs.w + ft.w) + extra_f;
                        if (!ambiguous && err <= 0.0625f * cut) {
                            const float lim = cut * (1.0f + U20) + err;
                            near = (bq[0] * bq[0] + bq[1] * bq[1] + bq[2] * bq[2]) < lim * lim;
                        } else { // the FP64 test of the sequential scan
                            const double4 pt = d.pr[nb][t];
                            bool per;
                            const V3 xt = image_of(I, xs, xyz(pt), per);
                            const V3 br = xs - xt;
                            const double cut = ps.w + pt.w + extra;
                            near = len2(br) < cut * cut;
                        }
                        if (near) {
                            if (count < d.cap) {
                                d.nbr[ln][nbr_at(d.ncap, s, count)] = t;
                                d.rows[(size_t)s * d.cap + count] = t;
                                if (is.x < d.info[nb][t].x) ownw |= 1u << (count & 31);
                                if ((count & 31) == 31) {
                                    d.own[ln][(size_t)(count >> 5) * d.ncap + s] = ownw;
                                    ownw = 0u;
                                }
                            } else {
                                overflow = true;
                            }
                            ++count;
                        }
                    }
                }
            }
        }
    }
    if (overflow) {
        atomicOr(&d.ctl->status, 1u << DEM_ERR_CAPACITY);
        count = d.cap;
    }
    if (count & 31) d.own[ln][(size_t)(count >> 5) * d.ncap + s] = ownw; // the last, partial word
    d.cnt[ln][s] = count;

    // still walls within reach + skin (k_detect tests only these until the next rebuild)
    unsigned int wc = 0u;
    if (!fixed_s) {
        const int nwl = I.wall_end - I.wall_begin;
        for (int w = 0; w < nwl; ++w) {
            if (!((I.wall_still_mask >> w) & 1u)) continue;
            const int wg = I.wall_begin + w;
            const dem_wall& wall = d.walls[wg];
            const double R = ps.w + d.species[I.species_offset + is.y * I.n_species + wall.species].interaction_distance +
                             d.ctl->skin;
            double dist;
            V3 nrm;
            if (wall_distance(wall, d.wgeom + wg, xs, R, dist, nrm)) wc |= 1u << w;
        }
    }
    d.wcand[ln][s] = wc;

    // carry contact history from the old list (old order) to the new one, up
    // to 4 contacts per pass over the new list
    const int o = d.perm[s];
    const int ocnt = d.cnt[lo_][o];
    unsigned int n0 = 0u, n1 = 0u, n2 = 0u, n3 = 0u;
    for (int w = 0; w < d.nwords; ++w) {
        unsigned int bits = d.act[hc][(size_t)w * d.ncap + o];
        while (bits) {
            int kk[4], tn[4], m[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                kk[j] = -1;
                if (bits) {
                    const int k = w * 32 + __ffs(bits) - 1;
                    bits &= bits - 1;
                    if (k < ocnt) kk[j] = k; // bits past the old count are stale
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) tn[j] = kk[j] >= 0 ? d.nbr[lo_][nbr_at(d.ncap, o, kk[j])] : -1;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                tn[j] = tn[j] >= 0 ? d.newidx[tn[j]] : -1;
                m[j] = -1;
            }
            for (int q0 = 0; q0 < count; q0 += 4) {
                int v[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) v[i] = (q0 + i < count) ? d.nbr[ln][nbr_at(d.ncap, s, q0 + i)] : -2;
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (m[j] < 0 && tn[j] >= 0 && v[i] == tn[j]) m[j] = q0 + i;
                bool done = true;
#pragma unroll
                for (int j = 0; j < 4; ++j) done = done && (tn[j] < 0 || m[j] >= 0);
                if (done) break;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (kk[j] < 0) continue;
                if (m[j] < 0) {
                    atomicAdd(&d.ctl->lost_history, 1u);
                    continue;
                }
                // the spring stays where it is in the pool; the new entry points at it
                d.hidx[nb][nbr_at(d.ncap, s, m[j])] = d.hidx[hc][nbr_at(d.ncap, o, kk[j])];
                set_bit4(n0, n1, n2, n3, m[j]);
            }
        }
    }
    const unsigned int nw[4] = {n0, n1, n2, n3};
#pragma unroll
    for (int w = 0; w < 4; ++w)
        if (w < d.nwords) d.act[nb][(size_t)w * d.ncap + s] = nw[w];
    // wall history moves with the particle (with the pad word: a triangle
    // contact's creation key, k_tri)
    const unsigned int wbits = d.wact[hc][o];
    d.wact[nb][s] = wbits;
    unsigned int bits = wbits;
    while (bits) {
        const int w = __ffs(bits) - 1;
        bits &= bits - 1;
        for (int comp = 0; comp < d.ncomp; ++comp)
            d.whist[nb][whist_at(d.ncap, d.ncomp, s, w) + comp] = d.whist[hc][whist_at(d.ncap, d.ncomp, o, w) + comp];
        if (d.has_tri) d.whist[nb][whist_at(d.ncap, d.ncomp, s, w) + d.ncomp] = d.whist[hc][whist_at(d.ncap, d.ncomp, o, w) + d.ncomp];
    }
}

// ---------------------------------------------------------------------------
// force + integration
// ---------------------------------------------------------------------------
// One spring record (pool_at / whist_at: 16-byte aligned, padded to an even
// count) as 16-byte vectors.
__device__ __forceinline__ void load_springs(const double* h, size_t base, int ncomp, Springs& s)
{
    const double2* p = reinterpret_cast<const double2*>(h + base);
    const double2 a = p[0], b = p[1];
    s.slide = v3(a.x, a.y, b.x);
    if (ncomp > 3) {
        const double2 c = p[2], e = p[3], f = p[4];
        s.roll = v3(b.y, c.x, c.y);
        s.tors = v3(e.x, e.y, f.x);
    } else {
        s.roll = zero3();
        s.tors = zero3();
    }
}

__device__ __forceinline__ void store_springs(double* h, size_t base, int ncomp, const Springs& s)
{
    double2* p = reinterpret_cast<double2*>(h + base);
    if (ncomp > 3) {
        p[0] = make_double2(s.slide.x, s.slide.y);
        p[1] = make_double2(s.slide.z, s.roll.x);
        p[2] = make_double2(s.roll.y, s.roll.z);
        p[3] = make_double2(s.tors.x, s.tors.y);
        p[4] = make_double2(s.tors.z, 0.0);
    } else {
        p[0] = make_double2(s.slide.x, s.slide.y);
        p[1] = make_double2(s.slide.z, 0.0);
    }
}

__device__ __forceinline__ void write_record(const DevPtrs& d, int id_p, int id_i, int is_wall, int periodic,
                                             int slot_p, int slot_i, const ContactGeom& g, const ContactOut& out,
                                             const Springs& s, double spring_energy)
{
    const unsigned int idx = atomicAdd(&d.ctl->n_records, 1u);
    if (idx >= d.ctl->record_capacity) return;
    ContactRecord& r = d.records[idx];
    r.id_p = id_p;
    r.id_i = id_i;
    r.is_wall = is_wall;
    r.periodic = periodic;
    r.slot_p = slot_p;
    r.slot_i = slot_i;
    r.overlap = g.overlap;
    r.elastic_energy = out.normal_stiffness_energy + spring_energy;
    r.force[0] = out.force.x; r.force[1] = out.force.y; r.force[2] = out.force.z;
    r.contact_point[0] = g.c.x; r.contact_point[1] = g.c.y; r.contact_point[2] = g.c.z;
    const V3 br = is_wall ? zero3() : g.xp - g.xi;
    r.branch[0] = br.x; r.branch[1] = br.y; r.branch[2] = br.z;
    r.normal[0] = g.n.x; r.normal[1] = g.n.y; r.normal[2] = g.n.z;
    r.tangential[0] = out.tangential.x; r.tangential[1] = out.tangential.y; r.tangential[2] = out.tangential.z;
    r.springs[0] = s.slide.x; r.springs[1] = s.slide.y; r.springs[2] = s.slide.z;
    r.springs[3] = s.roll.x; r.springs[4] = s.roll.y; r.springs[5] = s.roll.z;
    r.springs[6] = s.tors.x; r.springs[7] = s.tors.y; r.springs[8] = s.tors.z;
}

// Elastic energy of the tangential springs (SlidingFrictionInteraction.cc:239-246,
// FrictionInteraction / Mindlin getElasticEnergy): used for the energy balance only.
__device__ __forceinline__ double spring_energy(const dem_species_pair& sp, const Springs& s, double meff)
{
    if (sp.friction_law == DEM_FRICTION_SLIDING || sp.friction_law == DEM_FRICTION_ROLLING_TORSION) {
        double e = sp.constant_restitution ? meff * sp.sliding_stiffness * len2(s.slide)
                                           : 0.5 * sp.sliding_stiffness * len2(s.slide);
        if (sp.friction_law == DEM_FRICTION_ROLLING_TORSION) {
            e += sp.constant_restitution ? meff * sp.rolling_stiffness * len2(s.roll)
                                         : 0.5 * sp.rolling_stiffness * len2(s.roll);
            e += sp.constant_restitution ? meff * sp.torsion_stiffness * len2(s.tors)
                                         : 0.5 * sp.torsion_stiffness * len2(s.tors);
        }
        return e;
    }
    return 0.0;
}

// DeletionBoundary::checkBoundaryAfterParticleMoved (DeletionBoundary.cc:109-126)
// after a drift: a deleted particle is parked far away as a fixed particle
// (no contact predicate can succeed against it) and a rebuild moves it to the
// graveyard cell.
__device__ __forceinline__ bool deletion_check(const InstanceDev& I, V3 x)
{
    for (int k = 0; k < I.n_del; ++k)
        if (I.del_d[k] - (x.x * I.del_n[k][0] + x.y * I.del_n[k][1] + x.z * I.del_n[k][2]) < 0) return true;
    return false;
}

__device__ __forceinline__ void park_deleted(Control* ctl, double4& p, double4& v, double4& w, int4& info)
{
    p = make_double4(DELETED_COORD, DELETED_COORD, DELETED_COORD, p.w);
    v = make_double4(0.0, 0.0, 0.0, 0.0);
    w = make_double4(0.0, 0.0, 0.0, 0.0);
    info.w |= FLAG_DELETED | FLAG_FIXED;
    ctl->force_rebuild = 1;
}

// First half-kick and drift from the stored forces: the
// integrateBeforeForceComputation that opens every dem_step call. It only
// touches each particle's own record, so it updates the current buffer in place.
__global__ void __launch_bounds__(256) k_kick_drift(DevPtrs d)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    Control* ctl = d.ctl;
    double disp2 = 0.0;
    if (s < d.n) {
        const int c = ctl->cur;
        const double4 ps = d.pr[c][s];
        const double4 vs = d.vm[c][s];
        const double4 ws = d.wi[c][s];
        const double4 qs = d.qo[c][s];
        const int4 is = d.info[c][s];
        const InstanceDev& I = d.inst[is.z];
        const double dt = d.dt;
        V3 x = xyz(ps), v = xyz(vs), w = xyz(ws);
        Q4 q{qs.x, qs.y, qs.z, qs.w};
        const V3 F = v3(d.force[3 * (size_t)s], d.force[3 * (size_t)s + 1], d.force[3 * (size_t)s + 2]);
        const V3 T = v3(d.torque[3 * (size_t)s], d.torque[3 * (size_t)s + 1], d.torque[3 * (size_t)s + 2]);
        if (vs.w != 0.0) {
            v += ((F * vs.w) * 0.5) * dt;
            const V3 disp = v * dt;
            x += disp;
            disp2 = len2(disp);
            if (d.rotation) {
                const S33 Ib{ws.w, 0.0, 0.0, ws.w, 0.0, ws.w};
                w += ((rotate_inverse_inertia(q, Ib) * T) * 0.5) * dt;
                q = quat_rotate(q, w * dt);
            }
        } else {
            const V3 disp = v * dt;
            x += disp;
            disp2 = len2(disp);
            q = quat_rotate(q, w * dt);
        }
        bool wrapped = false;
        if (I.per_mask) {
            double* xc = &x.x;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if ((I.per_mask >> k) & 1u) {
                    const double dl = xc[k] - I.per_lo[k], dr = I.per_hi[k] - xc[k];
                    if ((dl < dr ? dl : dr) < 0) {
                        wrapped = true;
                        if (I.per_hi[k] - xc[k] > xc[k] - I.per_lo[k])
                            xc[k] = xc[k] + I.per_L[k];
                        else
                            xc[k] = xc[k] - I.per_L[k];
                    }
                }
            }
        }
        double4 pn = make_double4(x.x, x.y, x.z, ps.w);
        double4 vn = make_double4(v.x, v.y, v.z, vs.w);
        double4 wn = make_double4(w.x, w.y, w.z, ws.w);
        int4 isn = is;
        isn.w = wrapped ? (is.w | FLAG_WRAPPED) : (is.w & ~FLAG_WRAPPED);
        if (I.n_del && !(is.w & FLAG_DELETED) && deletion_check(I, x)) {
            park_deleted(ctl, pn, vn, wn, isn);
            disp2 = 0.0;
        }
        if (isn.w != is.w) d.info[c][s] = isn;
        d.pr[c][s] = pn;
        d.vm[c][s] = vn;
        d.wi[c][s] = wn;
        d.qo[c][s] = make_double4(q.q0, q.q1, q.q2, q.q3);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) disp2 = fmax(disp2, __shfl_xor_sync(0xffffffffu, disp2, o));
    if ((threadIdx.x & 31) == 0 && disp2 > 0.0)
        atomicMax(&ctl->step_disp2_bits, (unsigned long long)__double_as_longlong(disp2));
}

} // namespace dem

namespace dem {

// ---------------------------------------------------------------------------
// global balances (DPMBase.cc:1528-1640); per-block partial sums, summed on
// the host in block order so the result does not depend on scheduling.
// slots: 0 kinetic, 1 rotational, 2 gravitational, 3 mass, 4-6 momentum,
//        7-9 mass*position, 10-12 angular momentum (I omega)
// ---------------------------------------------------------------------------
constexpr int RED_SLOTS = 13;

__global__ void __launch_bounds__(256) k_reduce_particles(DevPtrs d, int instance, double* partial)
{
    __shared__ double sh[RED_SLOTS][8];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double v[RED_SLOTS];
#pragma unroll
    for (int k = 0; k < RED_SLOTS; ++k) v[k] = 0.0;
    if (s < d.n) {
        const int c = d.ctl->cur;
        const int4 is = d.info[c][s];
        if (is.z == instance && !(is.w & FLAG_FIXED)) {
            const double4 p = d.pr[c][s];
            const double4 vm = d.vm[c][s];
            const double4 w = d.wi[c][s];
            const InstanceDev& I = d.inst[is.z];
            const double m = 1.0 / vm.w;
            const V3 vel = xyz(vm), om = xyz(w), x = xyz(p);
            v[0] = .5 * m * len2(vel);
            const double inertia = 1.0 / w.w; // isotropic sphere: getInertia() = 1/invInertia
            v[1] = .5 * dot(om, om * inertia);
            const V3 g = v3(-I.gravity[0], -I.gravity[1], -I.gravity[2]);
            v[2] = m * dot(g, x);
            v[3] = m;
            v[4] = m * vel.x; v[5] = m * vel.y; v[6] = m * vel.z;
            v[7] = m * x.x; v[8] = m * x.y; v[9] = m * x.z;
            v[10] = inertia * om.x; v[11] = inertia * om.y; v[12] = inertia * om.z;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < RED_SLOTS; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < RED_SLOTS) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x][w];
        partial[(size_t)blockIdx.x * RED_SLOTS + threadIdx.x] = x;
    }
}

// elastic energy and contact counts from the contact records of the last
// force evaluation; slots: 0 energy, 1 particle contacts, 2 wall contacts
__global__ void __launch_bounds__(256) k_reduce_records(DevPtrs d, int instance, unsigned n_records, double* partial)
{
    __shared__ double sh[3][8];
    const unsigned r = blockIdx.x * blockDim.x + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (r < n_records) {
        const ContactRecord& rec = d.records[r];
        const int c = d.ctl->cur;
        if (d.info[c][rec.slot_p].z == instance) {
            v[0] = rec.elastic_energy;
            if (rec.is_wall) v[2] = 1.0; else v[1] = 1.0;
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x][w];
        partial[(size_t)blockIdx.x * 3 + threadIdx.x] = x;
    }
}

// ---------------------------------------------------------------------------
// host <-> device particle exchange through a device staging area holding the
// caller's structure-of-arrays layout (dem_particles_soa), so that uploads and
// downloads are plain contiguous copies and the (un)permutation runs here
// ---------------------------------------------------------------------------
struct StagePtrs {
    double *pos, *vel, *ang, *ori, *rad, *im, *ii;
    int *sp, *id, *inst, *lvl;
};

// 18 words of 8 bytes per particle slot
__host__ __device__ inline StagePtrs stage_ptrs(double* base, size_t nc)
{
    StagePtrs s;
    s.pos = base;
    s.vel = base + 3 * nc;
    s.ang = base + 6 * nc;
    s.ori = base + 9 * nc;
    s.rad = base + 13 * nc;
    s.im = base + 14 * nc;
    s.ii = base + 15 * nc;
    int* ib = reinterpret_cast<int*>(base + 16 * nc);
    s.sp = ib;
    s.id = ib + nc;
    s.inst = ib + 2 * nc;
    s.lvl = ib + 3 * nc;
    return s;
}

// The HGrid level of radius r under the instance's banding: the binary
// exponent of r / level_rmin, clamped to the bands, through the remap of
// empty bands (setup_instance_grid; for insertion boundaries the host made
// every band the PSD reaches a level).
__device__ __forceinline__ int level_of_radius(const InstanceDev& I, double r)
{
    const double x = r / I.level_rmin;
    int l = (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
    l = l < 0 ? 0 : (l > I.level_bands - 1 ? I.level_bands - 1 : l);
    const int m = I.level_remap[l];
    return m < 0 ? 0 : m;
}

// Radii of a one-instance upload, before the cell grid is laid out: their
// extremes and whether any is not a positive finite number (stats[0], [1]:
// bits of the smallest and largest positive radius, which order like the
// values; stats[2]: nonzero if some radius is bad).
__global__ void __launch_bounds__(256) k_radius_extremes(const double* r, int n, unsigned long long* stats)
{
    double lo = DBL_MAX, hi = 0.0;
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = r[i];
        if (!(x > 0.0) || !(x <= DBL_MAX)) {
            bad = true;
            continue;
        }
        lo = fmin(lo, x);
        hi = fmax(hi, x);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&stats[0], (unsigned long long)__double_as_longlong(lo));
        atomicMax(&stats[1], (unsigned long long)__double_as_longlong(hi));
        if (bad) atomicOr(&stats[2], 1ull);
    }
}

// The largest radius of every band (setup_instance_grid's bands: binary
// exponent of r / rmin, clamped to nl - 1): band_max[l] gets its bits.
__global__ void __launch_bounds__(256) k_radius_bands(const double* r, int n, double rmin, int nl,
                                                      unsigned long long* band_max)
{
    unsigned long long m[DEM_MAX_LEVELS] = {0ull, 0ull, 0ull, 0ull};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = r[i] / rmin;
        int l = (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
        l = l < 0 ? 0 : (l > nl - 1 ? nl - 1 : l);
        const unsigned long long b = (unsigned long long)__double_as_longlong(r[i]);
#pragma unroll
        for (int k = 0; k < DEM_MAX_LEVELS; ++k)
            if (k == l && b > m[k]) m[k] = b;
    }
#pragma unroll
    for (int k = 0; k < DEM_MAX_LEVELS; ++k) {
        unsigned long long v = m[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if ((threadIdx.x & 31) == 0 && v) atomicMax(&band_max[k], v);
    }
}

// caller order -> state buffer 0 (identity permutation until the first rebuild).
// It also checks what it packs (finite positions and velocities, radius > 0,
// species below nsp, inverse mass >= 0, instance 0 where one_instance) and
// reports a violation as DEM_ERR_BAD_INPUT in the control status. Rows the
// host gave level -1 are free rows of insertion boundaries: packed dormant.
__global__ void __launch_bounds__(256) k_pack(DevPtrs d, StagePtrs s, int has_ang, int has_ori, int has_ii,
                                              int has_inst, int nsp, int one_instance, int levels_here)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    if (d.row_slot) d.row_slot[i] = i;
    // levels_here: a one-instance upload without free rows, whose levels are
    // computed here from the banding instead of sent by the host
    const int lvl = levels_here ? level_of_radius(d.inst[0], s.rad[i]) : s.lvl[i];
    if (lvl < 0) { // a free row of an insertion boundary (radius 0): dormant until filled
        d.pr[0][i] = make_double4(DELETED_COORD, DELETED_COORD, DELETED_COORD, 0.0);
        d.vm[0][i] = make_double4(0.0, 0.0, 0.0, 0.0);
        d.wi[0][i] = make_double4(0.0, 0.0, 0.0, 0.0);
        d.qo[0][i] = make_double4(1.0, 0.0, 0.0, 0.0);
        d.info[0][i] = make_int4(s.id[i], 0, has_inst ? s.inst[i] : 0, FLAG_FIXED | FLAG_DELETED | FLAG_DORMANT);
        d.caller[0][i] = i;
        return;
    }
    const double im = s.im[i];
    {
        bool bad = !(s.rad[i] > 0.0) || !(s.rad[i] <= DBL_MAX) || !(im >= 0.0) || s.sp[i] < 0 || s.sp[i] >= nsp ||
                   (one_instance && has_inst && s.inst[i] != 0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            bad = bad || !(fabs(s.pos[3 * i + k]) <= DBL_MAX) || !(fabs(s.vel[3 * i + k]) <= DBL_MAX);
        if (bad) atomicOr(&d.ctl->status, 1u << DEM_ERR_BAD_INPUT);
    }
    d.pr[0][i] = make_double4(s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2], s.rad[i]);
    d.vm[0][i] = make_double4(s.vel[3 * i], s.vel[3 * i + 1], s.vel[3 * i + 2], im);
    d.wi[0][i] = make_double4(has_ang ? s.ang[3 * i] : 0.0, has_ang ? s.ang[3 * i + 1] : 0.0,
                              has_ang ? s.ang[3 * i + 2] : 0.0, has_ii ? s.ii[i] : 0.0);
    d.qo[0][i] = has_ori ? make_double4(s.ori[4 * i], s.ori[4 * i + 1], s.ori[4 * i + 2], s.ori[4 * i + 3])
                         : make_double4(1.0, 0.0, 0.0, 0.0);
    const int flags = (im == 0.0 ? FLAG_FIXED : 0) | (lvl << LEVEL_SHIFT);
    d.info[0][i] = make_int4(s.id[i], s.sp[i], has_inst ? s.inst[i] : 0, flags);
    d.caller[0][i] = i;
}

// state buffer b (engine order) -> caller order
__global__ void __launch_bounds__(256) k_unpack(DevPtrs d, int b, StagePtrs s)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const int i = d.caller[b][k];
    const double4 p = d.pr[b][k], v = d.vm[b][k], w = d.wi[b][k], q = d.qo[b][k];
    const int4 f = d.info[b][k];
    s.pos[3 * i] = p.x; s.pos[3 * i + 1] = p.y; s.pos[3 * i + 2] = p.z;
    s.vel[3 * i] = v.x; s.vel[3 * i + 1] = v.y; s.vel[3 * i + 2] = v.z;
    s.ang[3 * i] = w.x; s.ang[3 * i + 1] = w.y; s.ang[3 * i + 2] = w.z;
    s.ori[4 * i] = q.x; s.ori[4 * i + 1] = q.y; s.ori[4 * i + 2] = q.z; s.ori[4 * i + 3] = q.w;
    s.rad[i] = p.w;
    s.im[i] = v.w;
    s.ii[i] = w.w;
    s.sp[i] = f.y;
    s.id[i] = f.x;
    s.inst[i] = (f.w & FLAG_DELETED) ? -1 : f.z;
}

// ---------------------------------------------------------------------------
// balances of many instances at once: instances are contiguous in the sorted
// order, so block k sums instance first+k over its slot range (from the cell
// table of the last rebuild) in a fixed order; contact records add their
// elastic energy and counts with atomics
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_reduce_instances(DevPtrs d, int first, double* out)
{
    __shared__ double sh[RED_SLOTS][8];
    const int k = first + blockIdx.x;
    const int c = d.ctl->cur;
    const int cb = d.inst[k].cell_base[0];
    const int ce = (k + 1 < d.n_instances) ? d.inst[k + 1].cell_base[0] : d.ncells - 1;
    const int b = d.cell_start[cb], e = d.cell_start[ce];
    double v[RED_SLOTS];
#pragma unroll
    for (int q = 0; q < RED_SLOTS; ++q) v[q] = 0.0;
    const InstanceDev& I = d.inst[k];
    for (int s = b + threadIdx.x; s < e; s += blockDim.x) {
        const int4 is = d.info[c][s];
        if (is.w & FLAG_FIXED) continue;
        const double4 p = d.pr[c][s];
        const double4 vm = d.vm[c][s];
        const double4 w = d.wi[c][s];
        const double m = 1.0 / vm.w;
        const V3 vel = xyz(vm), om = xyz(w), x = xyz(p);
        const double inertia = 1.0 / w.w;
        const V3 g = v3(-I.gravity[0], -I.gravity[1], -I.gravity[2]);
        v[0] += .5 * m * len2(vel);
        v[1] += .5 * dot(om, om * inertia);
        v[2] += m * dot(g, x);
        v[3] += m;
        v[4] += m * vel.x; v[5] += m * vel.y; v[6] += m * vel.z;
        v[7] += m * x.x; v[8] += m * x.y; v[9] += m * x.z;
        v[10] += inertia * om.x; v[11] += inertia * om.y; v[12] += inertia * om.z;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < RED_SLOTS; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < RED_SLOTS) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x][w];
        out[(size_t)blockIdx.x * (RED_SLOTS + 3) + threadIdx.x] = x;
    }
    if (threadIdx.x >= RED_SLOTS && threadIdx.x < RED_SLOTS + 3)
        out[(size_t)blockIdx.x * (RED_SLOTS + 3) + threadIdx.x] = 0.0;
}

__global__ void __launch_bounds__(256) k_reduce_records_instances(DevPtrs d, int first, int count,
                                                                  unsigned n_records, double* out)
{
    const unsigned r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_records) return;
    const ContactRecord& rec = d.records[r];
    const int k = d.info[d.ctl->cur][rec.slot_p].z - first;
    if (k < 0 || k >= count) return;
    double* o = out + (size_t)k * (RED_SLOTS + 3) + RED_SLOTS;
    atomicAdd(o, rec.elastic_energy);
    atomicAdd(o + (rec.is_wall ? 2 : 1), 1.0);
}

} // namespace dem
