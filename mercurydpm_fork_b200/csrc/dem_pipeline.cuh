// dem_pipeline.cuh -- one force evaluation as three kernels over a compact
// contact list, each contact's law evaluated once:
//
//   k_detect   one thread per particle: the exact contact predicate
//              (BaseParticle::getInteractionWith, BaseParticle.cc:688-710) on
//              the neighbour entries the particle owns as P -- the lower id,
//              or its own view of a periodic pair (DPMBase.cc:3124-3139) --
//              and on its walls; contacts are appended to a compact item list
//              (one atomic per block) and every entry gets its item index or a
//              role mark; history bits of the next buffer are written here.
//   k_contacts one thread per contact item: the contact law with the spring
//              history (DPMBase::computeInternalForce, DPMBase.cc:3113-3162;
//              walls: DPMBase.cc:3188-3215), the force/torque share of P and,
//              for an ordinary pair, of I, into the item's 12 doubles.
//   k_tri      (only with triangle walls) one thread per particle with
//              triangle-wall candidates: the reference's wall loop for them
//              with group merging and overlap weighting, into one item.
//   k_sum      one thread per particle: the shares in neighbour-list order
//              (P entries from its own items, I entries from the partner's
//              item, which k_contacts announces in I's entry through the
//              reverse index), the body force
//              (DPMBase.cc:3168-3179), then the wall shares -- the order the
//              sequential code adds them -- then the integration tail.
//
// The entry and item orders do not change any sum: each particle adds its
// shares in its own list order, so results are independent of the atomics.
#pragma once
#include "dem_kernels.cuh"

namespace dem {

constexpr int ITEM_WALL = 1 << 20;   // item entry field >= this: wall contact (ITEM_WALL + wall)
constexpr int ITEM_TRI = ITEM_WALL + (1 << 10); // all triangle-wall contacts of a particle (k_tri)
// One triangle contact of the initial evaluation (k_tri): wall, creation key,
// overlap, normal, force, torque, contact point, species, normal elastic
// energy, springs.
constexpr int TRI_REC = 26;
constexpr int SLOT_NONE = -1;        // P entry without a contact this evaluation
constexpr int SLOT_IS_I = -2;        // entry whose partner owns the pair, no contact this evaluation
constexpr int SLOT_I_BASE = -3;      // SLOT_I_BASE - q: I's share of the partner's item q
constexpr int SHARE = 12;            // doubles per item: P force, P torque, I force, I torque
// Launch shapes. k_detect and k_sum are compiled for blocks of 64, 128 and
// 256 threads and k_contacts' grid size is a run-time value; the handle keeps
// the choice (dem_autotune measures the variants on the live state).
constexpr int DETECT_BLOCK = 128;        // the default k_detect block
constexpr int CONTACT_BLOCK = 128;
constexpr int SUM_BLOCK = 128;           // the default k_sum block
constexpr int SUM_THREADS_PER_SM = 640;  // k_sum's launch bounds: 640 / block resident blocks per SM

// Shared-memory copies of the instance record (when there is one instance)
// and of the species-pair table (when it has at most SP_STAGE_MAX entries),
// staged by k_contacts' blocks before their first item: the contact law's
// parameters are then no dependent global loads (measured: 51.6 -> 49.1 us per
// evaluation on the 200k chute; k_detect and k_sum gained nothing from it).
constexpr int SP_STAGE_MAX = 16;
struct TableStage {
    __align__(16) unsigned char inst[sizeof(InstanceDev)];
    __align__(16) unsigned char sp[SP_STAGE_MAX * sizeof(dem_species_pair)];
};
static_assert(sizeof(InstanceDev) % 4 == 0 && sizeof(dem_species_pair) % 4 == 0, "staged as 32-bit words");

// Called by every thread of the block (it synchronises the block).
__device__ __forceinline__ void stage_tables(const DevPtrs& d, TableStage& st)
{
    if (d.single_instance) {
        const int* src = reinterpret_cast<const int*>(d.inst);
        int* dst = reinterpret_cast<int*>(st.inst);
        for (int k = threadIdx.x; k < (int)(sizeof(InstanceDev) / 4); k += blockDim.x) dst[k] = src[k];
    }
    if (d.n_species_table <= SP_STAGE_MAX) {
        const int* src = reinterpret_cast<const int*>(d.species);
        int* dst = reinterpret_cast<int*>(st.sp);
        const int words = d.n_species_table * (int)(sizeof(dem_species_pair) / 4);
        for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
}

__device__ __forceinline__ const InstanceDev& staged_inst(const DevPtrs& d, const TableStage& st, int z)
{
    return d.single_instance ? *reinterpret_cast<const InstanceDev*>(st.inst) : d.inst[z];
}

__device__ __forceinline__ const dem_species_pair* staged_species(const DevPtrs& d, const TableStage& st)
{
    return d.n_species_table <= SP_STAGE_MAX ? reinterpret_cast<const dem_species_pair*>(st.sp) : d.species;
}

// Position of s in the particle-major row of t (the first 16 entries come
// from `head`, read ahead by the caller); -1 if absent.
__device__ __forceinline__ int find_in_row(const DevPtrs& d, int s, int t, int ct, const int4 (&head)[4])
{
    const int4* row = reinterpret_cast<const int4*>(d.rows + (size_t)t * d.cap); // cap is a multiple of 32
    for (int m0 = 0; m0 < ct; m0 += 16) {
        int4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = m0 == 0 ? head[j] : ((m0 + 4 * j < ct) ? row[(m0 >> 2) + j] : make_int4(-1, -1, -1, -1));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int q = m0 + 4 * j;
            if (q + 0 < ct && v[j].x == s) return q + 0;
            if (q + 1 < ct && v[j].y == s) return q + 1;
            if (q + 2 < ct && v[j].z == s) return q + 2;
            if (q + 3 < ct && v[j].w == s) return q + 3;
        }
    }
    return -1;
}

// Reverse index of one particle's list (after a rebuild, lists buffer l):
// rev[s][k] = m with nbr[t][m] == s for t = nbr[s][k] (the lists are
// symmetric). Two entries at a time; the partners' rows are read from the
// particle-major copy that build_one writes (the first 16 entries of both
// rows in flight together). Run by k_rebuild.
__device__ __forceinline__ void rev_one(const DevPtrs& d, int s, int l)
{
    const int cnt = min(d.cnt[l][s], d.cap);
    for (int k0 = 0; k0 < cnt; k0 += 2) {
        int t[2], ct[2];
        int4 head[2][4];
#pragma unroll
        for (int j = 0; j < 2; ++j) t[j] = (k0 + j < cnt) ? d.nbr[l][nbr_at(d.ncap, s, k0 + j)] : -1;
#pragma unroll
        for (int j = 0; j < 2; ++j)
            if (t[j] >= 0) {
                ct[j] = d.cnt[l][t[j]];
                const int4* row = reinterpret_cast<const int4*>(d.rows + (size_t)t[j] * d.cap);
#pragma unroll
                for (int q = 0; q < 4; ++q) head[j][q] = row[q]; // 16 <= cap entries: inside the row
            }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (t[j] < 0) continue;
            int m = find_in_row(d, s, t[j], min(ct[j], d.cap), head[j]);
            if (m < 0) {
                atomicOr(&d.ctl->status, 1u << DEM_ERR_CAPACITY); // an asymmetric pair: the partner's row overflowed
                m = 0;
            }
            d.rev[nbr_at(d.ncap, s, k0 + j)] = m;
        }
    }
}

// Exclusive block scan of one int per thread (any block of whole warps); returns
// this thread's offset and the block total through `total`.
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    int before = 0;
    total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        if (w < wid) before += warp_sums[w];
        total += warp_sums[w];
    }
    return before + x - v;
}

template <int MODE, int NCOMP, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_detect(DevPtrs d)
{
    constexpr int HIT_KEEP = 16; // partner slots of the first hits, kept for the item pass
    __shared__ int warp_sums[BLOCK / 32];
    __shared__ int block_base;
    __shared__ int kept_t[HIT_KEEP][BLOCK];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    Control* ctl = d.ctl;
    const int c = ctl->cur, l = ctl->lbuf, nb = c ^ 1, pc = ctl->pcur;
    const bool first = (MODE == 1) && ctl->first_step;
    const bool active = s < d.n;
    // hit bits of the (at most 4) list words, in registers: each word is
    // finished before the next starts, so no dynamically indexed array
    unsigned int hit0 = 0u, hit1 = 0u, hit2 = 0u, hit3 = 0u;
    int nkept = 0;
    unsigned int whit = 0u, wnew = 0u, thit = 0u;
    int count = 0, nwalls = 0;
    if (active) {
        const double4 ps = d.pr[c][s];
        const int4 is = d.info[c][s];
        const InstanceDev& I = d.inst[is.z];
        const V3 xs = xyz(ps);
        count = min(d.cnt[l][s], d.cap);
        const int ns = I.n_species;
        constexpr int B = 2; // entries whose gathers are in flight together (2 keeps 80 registers)
        const int2* info2 = reinterpret_cast<const int2*>(d.info[c]); // (id, species) of each info record
        // Without periodic boundaries a pair's owner (the lower id) is fixed
        // for the life of a list, and the rebuild stored it (own bits): the
        // partner-owned entries are marked without gathering the partner, and
        // the owned ones are visited in list order, B at a time. With periodic
        // boundaries every entry is visited (its image decides the owner).
        const bool owner_known = I.per_mask == 0u;
        for (int w = 0; w < d.nwords; ++w) {
            unsigned int hitw = 0u, neww = 0u;
            const int kbeg = 32 * w, kend = min(count, kbeg + 32);
            const unsigned int valid = kend <= kbeg ? 0u : (kend - kbeg == 32 ? 0xffffffffu : (1u << (kend - kbeg)) - 1u);
            unsigned int todo = valid;
            if (owner_known && valid) {
                const unsigned int ow = d.own[l][(size_t)w * d.ncap + s];
                unsigned int other = valid & ~ow;
                while (other) {
                    const int k = kbeg + __ffs(other) - 1;
                    other &= other - 1;
                    d.slot[nbr_at(d.ncap, s, k)] = SLOT_IS_I;
                }
                todo = valid & ow;
            }
            const unsigned int aw = (first && valid) ? d.act[c][(size_t)w * d.ncap + s] : 0u;
            while (todo) {
                int kb[B], tb[B];
                double4 ptb[B];
                int2 itb[B];
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    kb[j] = -1;
                    if (todo) {
                        kb[j] = kbeg + __ffs(todo) - 1;
                        todo &= todo - 1;
                    }
                }
#pragma unroll
                for (int j = 0; j < B; ++j) tb[j] = kb[j] >= 0 ? d.nbr[l][nbr_at(d.ncap, s, kb[j])] : -1;
#pragma unroll
                for (int j = 0; j < B; ++j)
                    if (tb[j] >= 0) {
                        ptb[j] = d.pr[c][tb[j]];
                        itb[j] = info2[2 * (size_t)tb[j]];
                    }
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    const int k = kb[j];
                    if (k < 0) break;
                    const size_t e = nbr_at(d.ncap, s, k);
                    const double4 pt = ptb[j];
                    const int2 it = itb[j];
                    bool periodic;
                    const V3 xt = image_of(I, xs, xyz(pt), periodic);
                    if (!periodic && !(is.x < it.x)) { // the partner (lower id) owns this pair
                        d.slot[e] = SLOT_IS_I;
                        continue;
                    }
                    d.slot[e] = SLOT_NONE;
                    const V3 branch = xs - xt;
                    const double d2 = len2(branch);
                    double idist = 0.0; // x + 0.0 == x: skipping the lookup keeps the predicate exact
                    if (!d.zero_idist) idist = d.species[I.species_offset + is.y * ns + it.y].interaction_distance;
                    const double sum = pt.w + ps.w + idist; // rI + rP + distance (BaseParticle.cc:695-697)
                    const unsigned int bit = 1u << (k & 31);
                    if (!(d2 >= sum * sum)) {
                        hitw |= bit;
                        if (nkept < HIT_KEEP) kept_t[nkept++][threadIdx.x] = tb[j];
                        neww |= bit;
                    } else if (first && (aw & bit) && !(periodic && is.x > it.x)) {
                        // an interaction of the initial evaluation outlives step 0
                        // (InteractionHandler::eraseOldInteractions erases stamps <= 0 only):
                        // its spring moves to the top of the next pool, below which the
                        // items of this evaluation stay (k_sum checks that they met no carry)
                        const int top = d.item_cap - 1 - (int)atomicAdd(&ctl->n_carry, 1u);
                        if (top >= 0) {
                            const double2* from = reinterpret_cast<const double2*>(d.pool[pc] + pool_at(NCOMP, d.hidx[c][e]));
                            double2* to = reinterpret_cast<double2*>(d.pool[pc ^ 1] + pool_at(NCOMP, top));
#pragma unroll
                            for (int q = 0; q < hist_stride(NCOMP) / 2; ++q) to[q] = from[q];
                            d.hidx[nb][e] = top;
                            neww |= bit;
                        } else {
                            atomicOr(&ctl->status, 1u << DEM_ERR_CAPACITY);
                        }
                    }
                }
            }
            d.act[nb][(size_t)w * d.ncap + s] = neww;
            if (w == 0) hit0 = hitw;
            else if (w == 1) hit1 = hitw;
            else if (w == 2) hit2 = hitw;
            else hit3 = hitw;
        }
        if (!(is.w & FLAG_FIXED)) {
            const unsigned int wa = d.wact[c][s];
            nwalls = I.wall_end - I.wall_begin;
            bool near_tri = false; // within reach of the instance's triangles (all of them, if they move)
            if (d.has_tri && I.tri_mask) {
                d.slott[s] = SLOT_NONE;
                // widened by a relative 1e-12 so that rounding of tri_lo - R cannot
                // skip a particle at exactly the reach
                const double R = (ps.w + I.max_interaction_distance) * (1.0 + 1e-12);
                near_tri = !I.tri_static ||
                           (xs.x > I.tri_lo[0] - R && xs.x < I.tri_hi[0] + R && xs.y > I.tri_lo[1] - R &&
                            xs.y < I.tri_hi[1] + R && xs.z > I.tri_lo[2] - R && xs.z < I.tri_hi[2] + R);
            }
            // farther than reach + skin at the last rebuild, or taken out
            const unsigned int far_still = (I.wall_still_mask & ~d.wcand[l][s]) | I.wall_off_mask;
            for (int w = 0; w < nwalls; ++w) {
                const int wg = I.wall_begin + w;
                const unsigned int bit = 1u << w;
                bool hit;
                if (d.has_tri && (I.tri_mask & bit)) {
                    // within R of the vertices' bounding box (the region the reference
                    // searches, Mercury3D::computeWallForces with TriangleWall::isLocal)
                    // and the face-plane test that opens TriangleWall::getDistanceAndNormal,
                    // R with the instance's largest interaction distance; k_tri finishes
                    // it and settles the history bits of these walls
                    hit = false;
                    if (near_tri) {
                        const WallGeom& tg = d.wgeom[wg];
                        const double R = ps.w + I.max_interaction_distance;
                        hit = xs.x > tg.tlo[0] - R && xs.x < tg.thi[0] + R && xs.y > tg.tlo[1] - R &&
                              xs.y < tg.thi[1] + R && xs.z > tg.tlo[2] - R && xs.z < tg.thi[2] + R &&
                              fabs(dot(xs - row3(tg.tv[0]), row3(tg.tfn))) < R;
                        if (hit) thit |= bit;
                    }
                } else {
                    d.slotw[(size_t)w * d.ncap + s] = SLOT_NONE;
                    if (far_still & bit) {
                        hit = false;
                    } else {
                        const dem_wall& wall = d.walls[wg];
                        const dem_species_pair& sp = d.species[I.species_offset + is.y * ns + wall.species];
                        double dist;
                        V3 nrm;
                        hit = wall_distance(wall, d.wgeom + wg, xs, ps.w + sp.interaction_distance, dist, nrm);
                        if (hit) whit |= bit;
                    }
                }
                if (hit) {
                    wnew |= bit;
                } else if (first && (wa & bit) && !(I.wall_off_mask & bit)) {
                    for (int q = 0; q < hist_stride(NCOMP); ++q) // with a triangle contact's creation key
                        d.whist[nb][whist_at(d.ncap, NCOMP, s, w) + q] = d.whist[c][whist_at(d.ncap, NCOMP, s, w) + q];
                    wnew |= bit;
                }
            }
        }
        d.wact[nb][s] = wnew;
    }
    // ---- compact the contacts of the block into the item list ----
    const unsigned int hits[4] = {hit0, hit1, hit2, hit3};
    int nh = __popc(whit) + (thit ? 1 : 0);
#pragma unroll
    for (int w = 0; w < 4; ++w) nh += __popc(hits[w]);
    int total;
    const int off = block_exclusive_scan(nh, warp_sums, total);
    if (threadIdx.x == 0) block_base = total ? (int)atomicAdd(&ctl->n_items, (unsigned)total) : 0;
    __syncthreads();
    int q = block_base + off;
    if (nh == 0) return;
    if (q + nh > d.item_cap) {
        atomicOr(&ctl->status, 1u << DEM_ERR_CAPACITY);
        return;
    }
    int nh_seen = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        unsigned int b = hits[w];
        // the entry's spring of the last evaluation, where it had one, goes into
        // the item (its pool index; -1: a new contact), and its spring of this
        // evaluation will sit at the item's own index
        const unsigned int aw = b ? d.act[c][(size_t)w * d.ncap + s] : 0u;
        while (b) {
            const int k = w * 32 + __ffs(b) - 1;
            b &= b - 1;
            const size_t e = nbr_at(d.ncap, s, k);
            const int t = (nh_seen < HIT_KEEP) ? kept_t[nh_seen][threadIdx.x] : d.nbr[l][e];
            ++nh_seen;
            const int prev = ((aw >> (k & 31)) & 1u) ? d.hidx[c][e] : -1;
            d.items[q] = make_int4(s, k, t, prev);
            d.slot[e] = q;
            d.hidx[nb][e] = q;
            ++q;
        }
    }
    unsigned int b = whit;
    while (b) {
        const int w = __ffs(b) - 1;
        b &= b - 1;
        d.items[q] = make_int4(s, ITEM_WALL + w, -1, 0);
        d.slotw[(size_t)w * d.ncap + s] = q;
        ++q;
    }
    if (thit) { // its net share is summed after the other walls' shares
        d.items[q] = make_int4(s, ITEM_TRI, (int)thit, 0);
        d.slott[s] = q;
        d.tri_list[atomicAdd(&ctl->n_tri, 1u)] = q;
    }
}

// RECORD: this launch may be the last force evaluation of a dem_step call,
// which writes the contact records; the steps before it are launched with
// RECORD = false, a variant without the record path (fewer registers).
// MINB: resident blocks per SM the registers are budgeted for (4: 128
// registers a thread; 5: 102; 6: 85; 3: 168), i.e. warps in flight against
// spills; the time-step variant is compiled for 3 to 6 (dem_autotune).
template <int MODE, int NLAW, int FLAW, int NCOMP, bool RECORD, int MINB = 4>
__global__ void __launch_bounds__(CONTACT_BLOCK, MINB) k_contacts(DevPtrs d)
{
    Control* ctl = d.ctl;
    const int c = ctl->cur, nb = c ^ 1, pc = ctl->pcur;
    const bool final_step = (MODE == 0) ? true : (ctl->final_step != 0);
    const bool record = RECORD && final_step && ctl->record;
    const bool first = (MODE == 1) && ctl->first_step;
    const int n_items = min((int)ctl->n_items, d.item_cap);
    const double dt = d.dt;
    __shared__ TableStage tables;
    stage_tables(d, tables);
    const dem_species_pair* species = staged_species(d, tables);
    const int stride = gridDim.x * blockDim.x;
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    int4 next = q < n_items ? d.items[q] : make_int4(0, 0, 0, 0);
    for (; q < n_items; q += stride) {
        const int4 item = next; // the next item is read while this one is evaluated
        if (q + stride < n_items) next = d.items[q + stride];
        const int s = item.x, kq = item.y;
        if (d.has_tri && kq == ITEM_TRI) continue; // k_tri
        const double4 ps = d.pr[c][s];
        const double4 vs = d.vm[c][s];
        const double4 ws = d.wi[c][s];
        const int4 is = d.info[c][s];
        const InstanceDev& I = staged_inst(d, tables, is.z);
        const int ns = I.n_species;
        const V3 xq = xyz(ps), vq = xyz(vs), wq = xyz(ws);
        const double rq = ps.w, mq = vs.w;
        ContactGeom g;
        Springs spr;
        spr.slide = zero3(); spr.roll = zero3(); spr.tors = zero3();
        const dem_species_pair* spp;
        bool periodic = false, was_active = false;
        int tq = 0, pid_i = 0;
        const bool is_wall = kq >= ITEM_WALL;
        double* hdst;
        size_t hb;
        V3 xt = zero3();
        int rv = 0; // I's entry for this pair (reverse index), read with the other gathers
        if (is_wall) {
            // DPMBase::computeForcesDueToWalls / BaseWall::getInteractionWith
            // (DPMBase.cc:3188-3215, BaseWall.cc:367-437)
            const int wl = kq - ITEM_WALL;
            const int wg = I.wall_begin + wl;
            const dem_wall& wall = d.walls[wg];
            spp = &species[I.species_offset + is.y * ns + wall.species];
            double dist;
            V3 nrm;
            wall_distance(wall, d.wgeom + wg, xq, rq + spp->interaction_distance, dist, nrm);
            g.n = -nrm;
            g.distance = dist;
            g.overlap = rq - dist;
            g.c = xq - (rq - 0.5 * g.overlap) * g.n;
            g.xp = xq; g.vp = vq; g.wp = wq; g.inv_mass_p = mq; g.curv_p = 1.0 / rq;
            g.xi = v3(wall.position[0], wall.position[1], wall.position[2]);
            g.vi = v3(wall.velocity[0], wall.velocity[1], wall.velocity[2]);
            g.wi = v3(wall.angular_velocity[0], wall.angular_velocity[1], wall.angular_velocity[2]);
            g.inv_mass_i = 0.0;
            g.curv_i = 0.0;
            g.i_is_wall = true;
            hb = whist_at(d.ncap, NCOMP, s, wl);
            hdst = d.whist[nb];
            was_active = (d.wact[c][s] >> wl) & 1u;
            if (was_active) load_springs(d.whist[c], hb, NCOMP, spr);
            pid_i = wg;
        } else {
            const size_t e = nbr_at(d.ncap, s, kq);
            tq = item.z;
            rv = d.rev[e];
            hb = pool_at(NCOMP, q); // this evaluation's spring sits at the item's index
            // the spring of the last evaluation (item.w; -1 for a new contact, whose
            // record 0 is read and not used): read before anything else needs it
            Springs own;
            load_springs(d.pool[pc], pool_at(NCOMP, max(item.w, 0)), NCOMP, own);
            const double4 pt = d.pr[c][tq];
            const int4 it = d.info[c][tq];
            const double4 vt4 = d.vm[c][tq];
            const double4 wt4 = d.wi[c][tq];
            xt = image_of(I, xq, xyz(pt), periodic);
            // this particle is P: the lower id, or the real particle against
            // the partner's periodic ghost (DPMBase.cc:3129-3139)
            const V3 branch = xq - xt;
            const double d2 = len2(branch);
            spp = &species[I.species_offset + is.y * ns + it.y];
            g.distance = sqrt(d2);
            g.n = branch / g.distance;
            g.overlap = rq + pt.w - g.distance;
            g.xp = xq; g.vp = vq; g.wp = wq; g.inv_mass_p = mq;
            g.xi = xt; g.vi = xyz(vt4); g.wi = xyz(wt4); g.inv_mass_i = vt4.w;
            g.c = g.xp - (rq - 0.5 * g.overlap) * g.n;
            g.curv_p = 1.0 / rq;
            g.curv_i = 1.0 / pt.w;
            g.i_is_wall = false;
            hdst = d.pool[pc ^ 1];
            was_active = item.w >= 0;
            // the higher-id side of a periodic pair restarts every step from the
            // reversed spring of the lower-id side (InteractionHandler.cc:316-368,
            // BaseInteraction::copySwitchPointer / reverseHistory)
            const bool derived = periodic && (is.x > it.x);
            if (derived) {
                const int m = rv;
                if ((d.act[c][(size_t)(m >> 5) * d.ncap + tq] >> (m & 31)) & 1u) {
                    load_springs(d.pool[pc], pool_at(NCOMP, d.hidx[c][nbr_at(d.ncap, tq, m)]), NCOMP, spr);
                    spr.slide = -spr.slide; spr.roll = -spr.roll; spr.tors = -spr.tors;
                }
            } else if (was_active) {
                spr = own;
            }
            pid_i = it.x;
        }
        ContactOut out;
        evaluate_contact<NLAW, FLAW>(*spp, g, spr, dt, out);
        // step 0 keeps the lower-id side's old spring of a periodic pair that
        // existed at the initial evaluation (equal stamps, InteractionHandler.cc:339-352);
        // that side is not derived and was active, so its old spring is its own
        // stored one, read again here instead of kept in registers
        Springs kept = spr;
        if (first && periodic && !(is.x > pid_i) && was_active) load_springs(d.pool[pc], pool_at(NCOMP, item.w), NCOMP, kept);
        store_springs(hdst, hb, NCOMP, kept);
        // shares as 16-byte stores (96-byte items: every item and half is 16-byte aligned)
        double2* sh = reinterpret_cast<double2*>(d.shares + (size_t)q * SHARE);
        const V3 tp = out.torque - cross(xq - g.c, out.force);
        sh[0] = make_double2(out.force.x, out.force.y);
        sh[1] = make_double2(out.force.z, tp.x);
        sh[2] = make_double2(tp.y, tp.z);
        if (!is_wall && !periodic) { // I's share of an ordinary pair, announced in I's own entry
            const V3 fi = -out.force;
            const V3 ti = -out.torque + cross(xt - g.c, out.force);
            sh[3] = make_double2(fi.x, fi.y);
            sh[4] = make_double2(fi.z, ti.x);
            sh[5] = make_double2(ti.y, ti.z);
            d.slot[nbr_at(d.ncap, tq, rv)] = SLOT_I_BASE - q;
        }
        if (record && (is_wall || !periodic || is.x < pid_i)) {
            const double meff = 1.0 / (g.inv_mass_p + g.inv_mass_i);
            write_record(d, is.x, pid_i, is_wall ? 1 : 0, periodic ? 1 : 0, s, is_wall ? pid_i : tq, g, out, kept,
                         spring_energy(*spp, kept, meff));
        }
    }
}

// All triangle-wall contacts of one particle, in wall order, as the
// reference's sequential wall loop makes them with the triangle-wall
// correction on (its default build; DPMBase::computeForcesDueToWalls,
// DPMBase.cc:3188-3215):
//  * BaseWall::getInteractionWith (BaseWall.cc:375-409): a triangle of group
//    g > 0 meets every contact already made this step with a triangle of the
//    same group; unless both are face contacts, the larger overlap wins -- a
//    larger new overlap takes the earlier contact over (its force is taken
//    back, it moves to the new triangle with its spring), a smaller one drops
//    the new contact; otherwise the contact with this triangle from the last
//    step (InteractionHandler::getInteraction) or a new one is used.
//  * DPMBase::computeAllForces (DPMBase.cc:3443-3486): with two or more
//    triangle contacts, each force and torque is taken back and applied again
//    weighted by overlap / (sum of overlaps), at the contact point moved by
//    the same weight.
// The particle's net force and torque from these steps go into the item's P
// share; the springs of the contacts left go to their triangles' history rows.
// The contacts are visited in the particle's interaction-list order, which
// is creation order (BaseInteractable::addInteraction appends,
// removeInteraction erases in place): each triangle contact carries a
// creation key (the time step it was made x 16 + its rank within that
// step) in the pad word of its history row.
// The first time step shares its time stamp with the initial evaluation
// (both numberOfTimeSteps + 1 = 1), so there every contact of the initial
// evaluation counts as made this step: the group rule compares against all
// of them from the start, a triangle takes its own contact over from that
// list, and the weighting includes those not touched again. The initial
// evaluation keeps its contacts' state in tri_first for this.
constexpr int TRI_BLOCK = 64;
template <int MODE, int NLAW, int FLAW, int NCOMP>
__global__ void __launch_bounds__(TRI_BLOCK) k_tri(DevPtrs d)
{
    constexpr int MAXT = DEM_MAX_TRIANGLE_CONTACTS;
    static_assert(NCOMP % 2 == 1, "the pad word of a history row holds the creation key");
    Control* ctl = d.ctl;
    const int c = ctl->cur, nb = c ^ 1;
    const bool final_step = (MODE == 0) ? true : (ctl->final_step != 0);
    const bool record = final_step && ctl->record;
    const bool first = (MODE == 1) && ctl->first_step;
    const int n_tri = min((int)ctl->n_tri, d.n);
    const double dt = d.dt;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_tri; t += gridDim.x * blockDim.x) {
        const int q = d.tri_list[t];
        const int4 item = d.items[q];
        const int s = item.x;
        const unsigned int mask = (unsigned int)item.z;
        const double4 ps = d.pr[c][s];
        const double4 vs = d.vm[c][s];
        const double4 ws = d.wi[c][s];
        const int4 is = d.info[c][s];
        const InstanceDev& I = d.inst[is.z];
        const int ns = I.n_species;
        const V3 xq = xyz(ps), vq = xyz(vs), wq = xyz(ws);
        const double rq = ps.w, mq = vs.w;
        const unsigned int was = d.wact[c][s];
        int ew[MAXT], esw[MAXT], ord[MAXT]; // ord: entries in interaction-list order
        double eov[MAXT], eel[MAXT], ek[MAXT];
        const double step_key = 16.0 * (double)ctl->steps_done;
        int made = 0; // contacts made this step
        V3 en[MAXT], ec[MAXT], ef[MAXT], et[MAXT], etan[MAXT];
        Springs es[MAXT];
        int ne = 0;
        V3 F = zero3(), T = zero3();
        const int ci = d.caller[c][s];
        if (first) { // the initial evaluation's contacts, in list order
            const int n0 = min(d.tri_first_n[ci], MAXT);
            const double* rec = d.tri_first + (size_t)ci * MAXT * TRI_REC;
            for (int o = 0; o < n0; ++o, rec += TRI_REC) {
                ew[o] = (int)rec[0]; ek[o] = rec[1]; eov[o] = rec[2];
                en[o] = v3(rec[3], rec[4], rec[5]);
                ef[o] = v3(rec[6], rec[7], rec[8]);
                et[o] = v3(rec[9], rec[10], rec[11]);
                ec[o] = v3(rec[12], rec[13], rec[14]);
                esw[o] = (int)rec[15]; eel[o] = rec[16];
                es[o].slide = v3(rec[17], rec[18], rec[19]);
                es[o].roll = v3(rec[20], rec[21], rec[22]);
                es[o].tors = v3(rec[23], rec[24], rec[25]);
                etan[o] = zero3();
                ord[o] = o;
            }
            ne = n0;
        }
        for (unsigned int b = mask; b; b &= b - 1) {
            const int w = __ffs(b) - 1;
            const int wg = I.wall_begin + w;
            const dem_wall& wall = d.walls[wg];
            const dem_species_pair* spw = &d.species[I.species_offset + is.y * ns + wall.species];
            double dist;
            V3 nrm;
            if (!triangle_distance(d.wgeom[wg], xq, rq + spw->interaction_distance, dist, nrm)) continue;
            const double overlap = rq - dist;
            int k = -1;
            bool dropped = false;
            if (wall.group > 0) {
                const bool face = triangle_face_contact(d.wgeom[wg], nrm);
                for (int o = 0; o < ne; ++o) {
                    const int e = ord[o];
                    const int eg = I.wall_begin + ew[e];
                    if (d.walls[eg].group != wall.group) continue;
                    if (face && triangle_face_contact(d.wgeom[eg], en[e])) continue;
                    if (overlap > eov[e]) { // take e's force back; e moves to this triangle
                        F += -ef[e];
                        T += -et[e] + cross(xq - ec[e], ef[e]);
                        ew[e] = w;
                        k = e;
                    } else {
                        dropped = true;
                        break;
                    }
                }
            }
            if (dropped) continue;
            if (k < 0 && first) // InteractionHandler::getExistingInteraction: first in list order
                for (int o = 0; o < ne; ++o)
                    if (ew[ord[o]] == w) {
                        k = ord[o];
                        break;
                    }
            if (k < 0) {
                if (ne == MAXT) {
                    atomicOr(&ctl->status, 1u << DEM_ERR_CAPACITY);
                    continue;
                }
                k = ne;
                ew[k] = w;
                esw[k] = wall.species;
                es[k].slide = zero3(); es[k].roll = zero3(); es[k].tors = zero3();
                if (!first && ((was >> w) & 1u)) { // the contact with this triangle from the last step
                    const size_t hb = whist_at(d.ncap, NCOMP, s, w);
                    load_springs(d.whist[c], hb, NCOMP, es[k]);
                    ek[k] = d.whist[c][hb + NCOMP];
                } else {
                    ek[k] = step_key + (double)(made++);
                }
                int o = ne++; // insert by creation key
                while (o > 0 && ek[ord[o - 1]] > ek[k]) {
                    ord[o] = ord[o - 1];
                    --o;
                }
                ord[o] = k;
            }
            ContactGeom g;
            g.n = -nrm;
            g.distance = dist;
            g.overlap = overlap;
            g.c = xq - (rq - 0.5 * g.overlap) * g.n;
            g.xp = xq; g.vp = vq; g.wp = wq; g.inv_mass_p = mq; g.curv_p = 1.0 / rq;
            g.xi = v3(wall.position[0], wall.position[1], wall.position[2]);
            g.vi = v3(wall.velocity[0], wall.velocity[1], wall.velocity[2]);
            g.wi = v3(wall.angular_velocity[0], wall.angular_velocity[1], wall.angular_velocity[2]);
            g.inv_mass_i = 0.0;
            g.curv_i = 0.0;
            g.i_is_wall = true;
            ContactOut out;
            evaluate_contact<NLAW, FLAW>(d.species[I.species_offset + is.y * ns + esw[k]], g, es[k], dt, out);
            en[k] = g.n; eov[k] = g.overlap; ec[k] = g.c;
            ef[k] = out.force; et[k] = out.torque; etan[k] = out.tangential; eel[k] = out.normal_stiffness_energy;
            F += ef[k];
            T += et[k] - cross(xq - ec[k], ef[k]);
        }
        if (ne > 1) {
            double osum = 0.0;
            for (int o = 0; o < ne; ++o) osum += eov[ord[o]];
            for (int o = 0; o < ne; ++o) {
                const int e = ord[o];
                F += -ef[e];
                T += -et[e] + cross(xq - ec[e], ef[e]);
                const double wgt = eov[e] / osum;
                ec[e] = xq - (rq - 0.5 * eov[e]) * wgt * en[e];
                ef[e] = ef[e] * wgt;
                et[e] = et[e] * wgt;
                F += ef[e];
                T += et[e] - cross(xq - ec[e], ef[e]);
            }
        }
        double2* sh = reinterpret_cast<double2*>(d.shares + (size_t)q * SHARE);
        sh[0] = make_double2(F.x, F.y);
        sh[1] = make_double2(F.z, T.x);
        sh[2] = make_double2(T.y, T.z);
        // history: each triangle keeps the first contact (in order) now attached
        // to it; at the first step after the initial evaluation a contact of that
        // evaluation that no entry took outlives the step (as k_detect carries them)
        unsigned int kept_bits = 0u;
        for (int o = 0; o < ne; ++o) {
            const int e = ord[o];
            const unsigned int bit = 1u << ew[e];
            if (kept_bits & bit) continue;
            kept_bits |= bit;
            const size_t hb = whist_at(d.ncap, NCOMP, s, ew[e]);
            store_springs(d.whist[nb], hb, NCOMP, es[e]);
            d.whist[nb][hb + NCOMP] = ek[e];
        }
        d.wact[nb][s] = (d.wact[nb][s] & ~mask) | kept_bits;
        if (MODE == 0) { // kept for the first time step
            double* rec = d.tri_first + (size_t)ci * MAXT * TRI_REC;
            for (int o = 0; o < ne; ++o, rec += TRI_REC) {
                const int e = ord[o];
                rec[0] = (double)ew[e]; rec[1] = ek[e]; rec[2] = eov[e];
                rec[3] = en[e].x; rec[4] = en[e].y; rec[5] = en[e].z;
                rec[6] = ef[e].x; rec[7] = ef[e].y; rec[8] = ef[e].z;
                rec[9] = et[e].x; rec[10] = et[e].y; rec[11] = et[e].z;
                rec[12] = ec[e].x; rec[13] = ec[e].y; rec[14] = ec[e].z;
                rec[15] = (double)esw[e]; rec[16] = eel[e];
                rec[17] = es[e].slide.x; rec[18] = es[e].slide.y; rec[19] = es[e].slide.z;
                rec[20] = es[e].roll.x; rec[21] = es[e].roll.y; rec[22] = es[e].roll.z;
                rec[23] = es[e].tors.x; rec[24] = es[e].tors.y; rec[25] = es[e].tors.z;
            }
            d.tri_first_n[ci] = ne;
        }
        if (record) {
            for (int e = 0; e < ne; ++e) {
                const int wg = I.wall_begin + ew[e];
                ContactGeom g;
                g.n = en[e]; g.overlap = eov[e]; g.c = ec[e]; g.xp = xq; g.xi = zero3();
                ContactOut out;
                out.force = ef[e]; out.torque = et[e]; out.tangential = etan[e];
                out.abs_normal_force = 0.0; out.normal_stiffness_energy = eel[e];
                const dem_species_pair& sp = d.species[I.species_offset + is.y * ns + esw[e]];
                write_record(d, is.x, wg, 1, 0, s, wg, g, out, es[e], spring_energy(sp, es[e], 1.0 / mq));
            }
        }
    }
}

template <int MODE, int BLOCK>
__global__ void __launch_bounds__(BLOCK, SUM_THREADS_PER_SM / BLOCK) k_sum(DevPtrs d)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    Control* ctl = d.ctl;
    const int c = ctl->cur, l = ctl->lbuf, nb = c ^ 1;
    const bool final_step = (MODE == 0) ? true : (ctl->final_step != 0);
    const double dt = d.dt;
    if (s == 0) { // k_contacts and k_tri are done: the next evaluation starts new lists
        // the springs kept at the pool top in the first time step must not have
        // met this evaluation's items
        if (ctl->n_carry && (unsigned long long)ctl->n_items + ctl->n_carry > (unsigned long long)d.item_cap)
            atomicOr(&ctl->status, 1u << DEM_ERR_CAPACITY);
        ctl->n_carry = 0u;
        ctl->n_items = 0u;
        ctl->n_tri = 0u;
    }
    double disp2 = 0.0;
    if (s < d.n) {
        const double4 ps = d.pr[c][s];
        const double4 vs = d.vm[c][s];
        const double4 ws = d.wi[c][s];
        double4 qs = d.qo[c][s];
        const int4 is = d.info[c][s];
        const InstanceDev& I = d.inst[is.z];
        // ---- the shares in list order, the body force, the wall shares ----
        V3 F = zero3(), T = zero3();
        const int count = min(d.cnt[l][s], d.cap);
        constexpr int B = 4; // slots read together, then their shares
        for (int k0 = 0; k0 < count; k0 += B) {
            int qs_[B];
#pragma unroll
            for (int j = 0; j < B; ++j) qs_[j] = (k0 + j < count) ? d.slot[nbr_at(d.ncap, s, k0 + j)] : SLOT_NONE;
            double sh6[B][6];
#pragma unroll
            for (int j = 0; j < B; ++j) {
                int q = qs_[j];
                int half = 0;
                if (q <= SLOT_I_BASE) {
                    q = SLOT_I_BASE - q;
                    half = 6;
                }
                if (q >= 0) {
                    const double2* sh = reinterpret_cast<const double2*>(d.shares + (size_t)q * SHARE + half);
                    const double2 a = sh[0], b = sh[1], e2 = sh[2];
                    sh6[j][0] = a.x; sh6[j][1] = a.y; sh6[j][2] = b.x;
                    sh6[j][3] = b.y; sh6[j][4] = e2.x; sh6[j][5] = e2.y;
                }
            }
#pragma unroll
            for (int j = 0; j < B; ++j) // in list order
                if (qs_[j] >= 0 || qs_[j] <= SLOT_I_BASE) {
                    F += v3(sh6[j][0], sh6[j][1], sh6[j][2]);
                    T += v3(sh6[j][3], sh6[j][4], sh6[j][5]);
                }
        }
        if (!(is.w & FLAG_FIXED)) { // DPMBase::computeExternalForces (DPMBase.cc:3168-3179)
            const double m = 1.0 / vs.w;
            F += v3(I.gravity[0], I.gravity[1], I.gravity[2]) * m - d.drag * xyz(vs);
            const int nw = I.wall_end - I.wall_begin;
            for (int w = 0; w < nw; ++w) {
                if (d.has_tri && ((I.tri_mask >> w) & 1u)) continue;
                const int q = d.slotw[(size_t)w * d.ncap + s];
                if (q < 0) continue;
                const double2* sh = reinterpret_cast<const double2*>(d.shares + (size_t)q * SHARE);
                const double2 a = sh[0], b = sh[1], e2 = sh[2];
                F += v3(a.x, a.y, b.x);
                T += v3(b.y, e2.x, e2.y);
            }
            if (d.has_tri && I.tri_mask) { // the net share of all triangle contacts (k_tri)
                const int q = d.slott[s];
                if (q >= 0) {
                    const double2* sh = reinterpret_cast<const double2*>(d.shares + (size_t)q * SHARE);
                    const double2 a = sh[0], b = sh[1], e2 = sh[2];
                    F += v3(a.x, a.y, b.x);
                    T += v3(b.y, e2.x, e2.y);
                }
            }
        }
        if (!(isfinite(F.x) && isfinite(F.y) && isfinite(F.z))) atomicOr(&ctl->status, 1u << DEM_ERR_NAN);

        // ---- integration ----
        double4 pn = ps, vn = vs, wn = ws;
        bool wrapped = false;
        if (final_step) {
            d.force[3 * (size_t)s + 0] = F.x;
            d.force[3 * (size_t)s + 1] = F.y;
            d.force[3 * (size_t)s + 2] = F.z;
            d.torque[3 * (size_t)s + 0] = T.x;
            d.torque[3 * (size_t)s + 1] = T.y;
            d.torque[3 * (size_t)s + 2] = T.z;
        }
        if (MODE == 1) {
            V3 x = xyz(ps), v = xyz(vs), w = xyz(ws);
            Q4 q{qs.x, qs.y, qs.z, qs.w};
            if (vs.w != 0.0) {
                const V3 a = ((F * vs.w) * 0.5) * dt;
                v += a; // BaseParticle::integrateAfterForceComputation
                V3 aw = zero3();
                if (d.rotation) {
                    const S33 Ib{ws.w, 0.0, 0.0, ws.w, 0.0, ws.w};
                    aw = ((rotate_inverse_inertia(q, Ib) * T) * 0.5) * dt;
                    w += aw;
                }
                if (!final_step) { // BaseParticle::integrateBeforeForceComputation of the next step
                    v += a;
                    const V3 disp = v * dt;
                    x += disp;
                    disp2 = len2(disp);
                    if (d.rotation) {
                        w += aw;
                        q = quat_rotate(q, w * dt);
                    }
                }
            } else if (!final_step) { // BaseInteractable::integrateBeforeForceComputation
                const V3 disp = v * dt;
                x += disp;
                disp2 = len2(disp);
                q = quat_rotate(q, w * dt);
            }
            if (!final_step && I.per_mask) { // PeriodicBoundary::checkBoundaryAfterParticlesMove
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
            pn = make_double4(x.x, x.y, x.z, ps.w);
            vn = make_double4(v.x, v.y, v.z, vs.w);
            wn = make_double4(w.x, w.y, w.z, ws.w);
            qs = make_double4(q.q0, q.q1, q.q2, q.q3);
        }
        int4 isn = is;
        isn.w = wrapped ? (is.w | FLAG_WRAPPED) : (is.w & ~FLAG_WRAPPED);
        if (MODE == 1 && !final_step && I.n_del && !(is.w & FLAG_DELETED) && deletion_check(I, xyz(pn))) {
            park_deleted(ctl, pn, vn, wn, isn);
            disp2 = 0.0;
        }
        d.pr[nb][s] = pn;
        d.vm[nb][s] = vn;
        d.wi[nb][s] = wn;
        d.qo[nb][s] = qs;
        d.info[nb][s] = isn;
        d.caller[nb][s] = d.caller[c][s];
    }
    if (MODE == 1) { // maximum displacement of this step (for the skin test)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) disp2 = fmax(disp2, __shfl_xor_sync(0xffffffffu, disp2, o));
        if ((threadIdx.x & 31) == 0 && disp2 > 0.0)
            atomicMax(&ctl->step_disp2_bits, (unsigned long long)__double_as_longlong(disp2));
    }
}

} // namespace dem
