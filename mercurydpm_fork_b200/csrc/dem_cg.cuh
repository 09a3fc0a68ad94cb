// dem_cg.cuh -- Gaussian coarse-graining, CG<Coordinates, Gauss, StandardFields>.
//
// Restates CG::evaluateParticle and CG::evaluateContact (Kernel/CG/CG.hcc:333-528)
// with the Gauss function (Kernel/CG/Functions/Gauss.hcc:61-270), the
// coordinate systems O, XZ and XYZ (Kernel/CG/Coordinates/{O,XZ,XYZ}.cc,
// Base_XY_XZ_YZ.cc:32-53) and StandardFields (Kernel/CG/Fields/StandardFields.cc:184-250):
//   particles: phi = prefactor exp(-|r - x|^2 / 2w^2) within the cutoff;
//   contacts:  psi = line integral of the Gauss function between the two
//              ends the reference's IntegralType selects (I to P, contact to P,
//              I to contact), contact stress += F (x) branch psi, and
//              interaction force density += (+-F) phi(contact point) for
//              contacts with a fixed partner or a wall.
// Every point gathers its sums in a fixed order, so an evaluation is
// bit-for-bit reproducible: each particle and contact is prepared once (its
// point range per dimension, CG.hcc:340-395 and 478-495, and its field values),
// filed in the bin of the first point of its range, and the bins are sorted
// by (bin, particle slot) and (bin, contact pair) with stable radix sorts
// (contact records arrive in launch order; the pair key makes their order
// canonical). One warp per point then walks the bins that can reach it in
// index order, each lane a fixed stride of every bin, and sums the lanes in a
// fixed butterfly. The host divides by the volume of the averaged dimensions
// (CG::volumeAverageVariables).
// The contact records are those of the last force evaluation, i.e. the
// interactions the reference holds when writeOutputFiles evaluates CG at the
// start of the next step. Positions are the particles' own (for a pair that
// meets across a periodic boundary the reference's kept interaction joins the
// two real particles, InteractionHandler.cc:316-368, and CG uses those).
#pragma once
#include <cub/device/device_radix_sort.cuh>

namespace dem {

constexpr double CG_PI = 3.1415926535897932384626433832795;
constexpr double CG_SQRT_PI = 1.7724538509055160272981674833411;
constexpr double CG_SQRT_2 = 1.4142135623730950488016887242097;

struct CGDev {
    int coord;           // DEM_CG_*
    int instance;
    int n[3];            // points per dimension (1 for unresolved dimensions)
    int resolved[3];
    double min[3], max[3];
    double start[3], delta[3];
    double width, cutoff;
    double prefactor;    // Coordinates::getGaussPrefactor
};

__device__ __forceinline__ int cg_dims(const CGDev& g) { return g.coord == DEM_CG_XYZ ? 3 : (g.coord == DEM_CG_XZ ? 2 : 0); }

// squared distance in the resolved dimensions (XZ::getDistanceSquared, XYZ::getDistanceSquared)
__device__ __forceinline__ double cg_dist2(const CGDev& g, V3 p, V3 r)
{
    if (g.coord == DEM_CG_XYZ) return len2(r - p);
    if (g.coord == DEM_CG_XZ) return (p.x - r.x) * (p.x - r.x) + (p.z - r.z) * (p.z - r.z);
    return 0.0;
}

// Gauss::evaluateCGFunction
__device__ __forceinline__ double cg_phi(const CGDev& g, V3 p, V3 r)
{
    if (g.coord == DEM_CG_O) return 1.0;
    const double d2 = cg_dist2(g, p, r);
    return (d2 > g.cutoff * g.cutoff) ? 0.0 : g.prefactor * exp(-d2 / (2.0 * g.width * g.width));
}

// Coordinates::getGaussIntegralPrefactor (Base_XY_XZ_YZ.cc:40-53, XYZ.cc:157-171)
__device__ __forceinline__ double cg_integral_prefactor(const CGDev& g, double distance)
{
    const double widthSqrt2 = g.width * CG_SQRT_2;
    const double a = -g.cutoff;
    const double b = g.cutoff + distance;
    double prefactor;
    if (g.coord == DEM_CG_XZ) {
        prefactor = 1.0 / (widthSqrt2 * CG_SQRT_PI);
        prefactor /= erf(g.cutoff / (widthSqrt2));
    } else {
        prefactor = 1.0 / (CG_SQRT_2 * CG_SQRT_PI * g.width);
        prefactor = prefactor * prefactor / (1.0 - exp(-0.5 * ((g.cutoff / g.width) * (g.cutoff / g.width))));
    }
    return prefactor * 0.5 /
           (+erf(b / widthSqrt2) * b + widthSqrt2 / CG_SQRT_PI * exp(-((b / widthSqrt2) * (b / widthSqrt2))) -
            erf(a / widthSqrt2) * a - widthSqrt2 / CG_SQRT_PI * exp(-((a / widthSqrt2) * (a / widthSqrt2))));
}

__device__ __forceinline__ V3 cg_point(const CGDev& g, int i, int j, int k)
{
    return v3(g.start[0] + g.delta[0] * i, g.start[1] + g.delta[1] * j, g.start[2] + g.delta[2] * k);
}

// index range of the points a support [lo, hi] (in index units) touches: CG.hcc:340-395, 478-495
__device__ __forceinline__ void cg_range(const CGDev& g, int d, double lo_idx, double hi_idx, int& lo, int& hi)
{
    if (!g.resolved[d]) {
        lo = 0;
        hi = 1;
        return;
    }
    const double a = lo_idx + 1.0;
    const double b = hi_idx + 1.0;
    lo = a > 0.0 ? (a < (double)g.n[d] ? (int)a : g.n[d]) : 0;
    hi = b > 0.0 ? (b < (double)g.n[d] ? (int)b : g.n[d]) : 0;
}

// A particle as the gather reads it: position, point range, and the values
// StandardFields::setFields(const BaseParticle&) multiplies by phi (fields 0-10
// and 23-28: volume, mass, momentum, momentum flux, radius powers 0-5).
struct CGParticle {
    double x[3];
    double val[17];
    int lo[3], hi[3];
};
// value f of a particle goes to field f (f < 11) or f + 12 (the radius powers)
__host__ __device__ constexpr int cg_pfield(int f) { return f < 11 ? f : f + 12; }

// IntegralType of CG::getIntegralType (CG.hcc:451-466)
enum CGIntegral { CG_NONE = 0, CG_I_TO_P, CG_CONTACT_TO_P, CG_I_TO_CONTACT };

// A contact record as the gather reads it: the ends of its line integral, force,
// normal, the two force vectors of StandardFields::setFields(const
// BaseInteraction&), the integral prefactor and its point range.
struct CGContact {
    double P[3], C[3], I[3];
    double F[3], n[3], nhat[3], branch[3], ifd[3];
    double nlen, prefactor;
    int type, pad;
    int lo[3], hi[3];
};

// bins: one per point; a particle or contact goes to the point its range starts at
__device__ __forceinline__ int cg_bin(const CGDev& g, const int lo[3]) { return (lo[0] * g.n[1] + lo[1]) * g.n[2] + lo[2]; }

__device__ __forceinline__ void cg_width_max(int* wmax, const int lo[3], const int hi[3])
{
    for (int k = 0; k < 3; ++k) atomicMax(wmax + k, hi[k] - lo[k]);
}

// Particle s: its record and bin (npts, the end marker, when it adds to no point).
__global__ void __launch_bounds__(128) k_cg_prep_particles(DevPtrs d, CGDev g, CGParticle* rec, unsigned* bin,
                                                            int* slot, int* wmax)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n) return;
    const int npts = g.n[0] * g.n[1] * g.n[2];
    slot[s] = s;
    bin[s] = npts;
    const int c = d.ctl->cur;
    const int4 is = d.info[c][s];
    if (is.z != g.instance || (is.w & FLAG_FIXED)) return; // StandardFields::evaluateFixedParticles() is false
    const double4 p4 = d.pr[c][s];
    const double4 v4 = d.vm[c][s];
    const V3 x = xyz(p4), v = xyz(v4);
    const double r = p4.w;
    const double m = 1.0 / v4.w;
    CGParticle q;
    for (int k = 0; k < 3; ++k) {
        const double pos = (&x.x)[k] - g.min[k];
        const double invDelta = g.n[k] / (g.max[k] - g.min[k]);
        const double idPos = pos * invDelta - 0.5;
        const double idCutoff = g.cutoff * invDelta;
        cg_range(g, k, idPos - idCutoff, idPos + idCutoff, q.lo[k], q.hi[k]);
        if (q.lo[k] >= q.hi[k]) return;
    }
    q.x[0] = x.x; q.x[1] = x.y; q.x[2] = x.z;
    // StandardFields::setFields(const BaseParticle&)
    q.val[0] = 4.0 / 3.0 * CG_PI * r * r * r; // BaseParticle::getVolume (3D)
    q.val[1] = m;
    q.val[2] = v.x * m; q.val[3] = v.y * m; q.val[4] = v.z * m;
    q.val[5] = v.x * v.x * m; q.val[6] = v.x * v.y * m; q.val[7] = v.x * v.z * m;
    q.val[8] = v.y * v.y * m; q.val[9] = v.y * v.z * m; q.val[10] = v.z * v.z * m;
    double ps = 1.0;
    for (int f = 0; f < 6; ++f) {
        q.val[11 + f] = ps;
        ps *= r;
    }
    rec[s] = q;
    bin[s] = (unsigned)cg_bin(g, q.lo);
    cg_width_max(wmax, q.lo, q.hi);
}

// Contact record rix: its canonical key (P's slot, wall flag, I's slot or wall).
__global__ void __launch_bounds__(128) k_cg_contact_keys(DevPtrs d, unsigned nrec, unsigned long long* key, int* idx)
{
    const unsigned rix = blockIdx.x * blockDim.x + threadIdx.x;
    if (rix >= nrec) return;
    const ContactRecord& r = d.records[rix];
    key[rix] = ((unsigned long long)(unsigned)r.slot_p << 32) | ((unsigned long long)(r.is_wall ? 1u : 0u) << 31) |
               (unsigned long long)(unsigned)r.slot_i;
    idx[rix] = (int)rix;
}

// The contact at canonical position j (record order[j]): its record and bin.
__global__ void __launch_bounds__(128) k_cg_prep_contacts(DevPtrs d, CGDev g, unsigned nrec, const int* order,
                                                           CGContact* out, unsigned* bin, int* pos, int* wmax)
{
    const unsigned j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nrec) return;
    const int npts = g.n[0] * g.n[1] * g.n[2];
    pos[j] = (int)j;
    bin[j] = npts;
    const ContactRecord& rec = d.records[order[j]];
    const int c = d.ctl->cur;
    const int4 ip = d.info[c][rec.slot_p];
    if (ip.z != g.instance) return;
    const bool p_fixed = (ip.w & FLAG_FIXED) != 0;
    const bool i_fixed = rec.is_wall ? true : ((d.info[c][rec.slot_i].w & FLAG_FIXED) != 0);
    int type;
    if (p_fixed)
        type = i_fixed ? CG_NONE : CG_I_TO_CONTACT;
    else
        type = i_fixed ? CG_CONTACT_TO_P : CG_I_TO_P;
    if (type == CG_NONE) return;
    const V3 P = xyz(d.pr[c][rec.slot_p]);
    const V3 C = v3(rec.contact_point[0], rec.contact_point[1], rec.contact_point[2]);
    V3 Ipos;
    if (rec.is_wall) {
        const dem_wall& w = d.walls[rec.slot_i];
        Ipos = v3(w.position[0], w.position[1], w.position[2]);
    } else {
        Ipos = xyz(d.pr[c][rec.slot_i]);
    }
    const V3 F = v3(rec.force[0], rec.force[1], rec.force[2]);
    const V3 n = v3(rec.normal[0], rec.normal[1], rec.normal[2]);
    // StandardFields::setFields(const BaseInteraction&, IntegralType); the
    // vectors of BaseInteraction.cc:459-476 (normal x distance, so a periodic
    // pair gets its image branch)
    V3 branch, ifd = zero3();
    const double dist = rec.is_wall ? 0.0 : sqrt(len2(v3(rec.branch[0], rec.branch[1], rec.branch[2])));
    if (type == CG_I_TO_P) {
        branch = n * dist;                  // getIP
    } else if (type == CG_I_TO_CONTACT) {
        ifd = -F;
        branch = n * dist + C - P;          // getIC
    } else {
        ifd = F;
        branch = P - C;                     // getCP
    }
    CGContact q;
    // point range between P and I (the contact point when I is fixed): CG.hcc:478-495
    const V3 Iend = i_fixed ? C : Ipos;
    for (int k = 0; k < 3; ++k) {
        if (g.n[k] == 1) {
            q.lo[k] = 0;
            q.hi[k] = 1;
            continue;
        }
        const double invDelta = g.n[k] / (g.max[k] - g.min[k]);
        const double pk = ((&P.x)[k] - g.min[k]) * invDelta - 0.5;
        const double ik = ((&Iend.x)[k] - g.min[k]) * invDelta - 0.5;
        const double ck = g.cutoff * invDelta;
        cg_range(g, k, fmin(pk, ik) - ck, fmax(pk, ik) + ck, q.lo[k], q.hi[k]);
        if (q.lo[k] >= q.hi[k]) return;
    }
    // Gauss::evaluateCGIntegral (Gauss.hcc:207-270)
    double nlen = 0.0;
    V3 nhat = n;
    if (g.coord == DEM_CG_XZ) {
        nlen = sqrt(n.x * n.x + n.z * n.z);
        nhat = n / nlen;
    } else if (g.coord == DEM_CG_XYZ) {
        nlen = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    }
    // the reference computes the integral prefactor at the first point of the
    // range (in i, j, k order) that passes the support test
    q.prefactor = 0.0;
    if (g.coord != DEM_CG_O && !(fabs(nlen) < 1e-10)) {
        const V3 ie = (type != CG_CONTACT_TO_P) ? Ipos : C;
        const V3 pe = (type != CG_I_TO_CONTACT) ? P : C;
        bool found = false;
        for (int i = q.lo[0]; i < q.hi[0] && !found; ++i)
            for (int jj = q.lo[1]; jj < q.hi[1] && !found; ++jj)
                for (int k = q.lo[2]; k < q.hi[2] && !found; ++k) {
                    const V3 r = cg_point(g, i, jj, k);
                    double iN, pN, t2;
                    if (g.coord == DEM_CG_XZ) {
                        iN = (ie.x - r.x) * nhat.x + (ie.z - r.z) * nhat.z;
                        pN = (pe.x - r.x) * nhat.x + (pe.z - r.z) * nhat.z;
                        t2 = (P.x - r.x) * (P.x - r.x) + (P.z - r.z) * (P.z - r.z) - pN * pN;
                    } else {
                        iN = dot(ie - r, n);
                        pN = dot(pe - r, n);
                        t2 = len2(P - r) - pN * pN;
                    }
                    if (!(iN > g.cutoff || pN < -g.cutoff || t2 > g.cutoff * g.cutoff)) {
                        q.prefactor = cg_integral_prefactor(g, pN - iN);
                        found = true;
                    }
                }
    }
    q.P[0] = P.x; q.P[1] = P.y; q.P[2] = P.z;
    q.C[0] = C.x; q.C[1] = C.y; q.C[2] = C.z;
    q.I[0] = Ipos.x; q.I[1] = Ipos.y; q.I[2] = Ipos.z;
    q.F[0] = F.x; q.F[1] = F.y; q.F[2] = F.z;
    q.n[0] = n.x; q.n[1] = n.y; q.n[2] = n.z;
    q.nhat[0] = nhat.x; q.nhat[1] = nhat.y; q.nhat[2] = nhat.z;
    q.branch[0] = branch.x; q.branch[1] = branch.y; q.branch[2] = branch.z;
    q.ifd[0] = ifd.x; q.ifd[1] = ifd.y; q.ifd[2] = ifd.z;
    q.nlen = nlen;
    q.type = type;
    q.pad = 0;
    out[j] = q;
    bin[j] = (unsigned)cg_bin(g, q.lo);
    cg_width_max(wmax + 3, q.lo, q.hi);
}

// Start and end of every bin in a list sorted by bin (empty bins keep 0, 0).
__global__ void k_cg_bin_bounds(const unsigned* sorted_bin, int m, int npts, int* start, int* end)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    const unsigned b = sorted_bin[p];
    if (b >= (unsigned)npts) return;
    if (p == 0 || sorted_bin[p - 1] != b) start[b] = p;
    if (p == m - 1 || sorted_bin[p + 1] != b) end[b] = p + 1;
}

constexpr int CG_GATHER = 128; // 4 points per block
constexpr int CG_ACC = 29;

// One warp per point: every particle and contact whose range covers the
// point, bins in index order, lane l taking entries l, l + 32, ... of each
// bin; the lanes' sums are added in a fixed butterfly.
__global__ void __launch_bounds__(CG_GATHER) k_cg_gather(CGDev g, const CGParticle* prec, const int* porder,
                                                         const int* pstart, const int* pend, const CGContact* crec,
                                                         const int* corder, const int* cstart, const int* cend,
                                                         int3 pw, int3 cw, double* out)
{
    const int lane = threadIdx.x & 31;
    const int pt = blockIdx.x * (CG_GATHER / 32) + (threadIdx.x >> 5);
    if (pt >= g.n[0] * g.n[1] * g.n[2]) return; // whole warps leave; no block barrier follows
    const int pk_ = pt % g.n[2], pj = (pt / g.n[2]) % g.n[1], pi = pt / (g.n[2] * g.n[1]);
    const int pidx[3] = {pi, pj, pk_};
    const V3 r = cg_point(g, pi, pj, pk_);
    double acc[CG_ACC];
#pragma unroll
    for (int f = 0; f < CG_ACC; ++f) acc[f] = 0.0;
    // particles: a range that covers this point starts at most pw - 1 points before it
    const int plo[3] = {max(0, pi - pw.x + 1), max(0, pj - pw.y + 1), max(0, pk_ - pw.z + 1)};
    for (int i = plo[0]; i <= pi; ++i)
        for (int j = plo[1]; j <= pj; ++j)
            for (int k = plo[2]; k <= pk_; ++k) {
                const int b = (i * g.n[1] + j) * g.n[2] + k;
                for (int e = pstart[b] + lane; e < pend[b]; e += 32) {
                    const CGParticle& q = prec[porder[e]];
                    bool in = true;
                    for (int dd = 0; dd < 3; ++dd) in = in && pidx[dd] < q.hi[dd];
                    if (!in) continue;
                    const double phi = cg_phi(g, v3(q.x[0], q.x[1], q.x[2]), r);
                    if (phi == 0.0) continue;
#pragma unroll
                    for (int f = 0; f < 17; ++f) acc[cg_pfield(f)] += q.val[f] * phi;
                }
            }
    const int clo[3] = {max(0, pi - cw.x + 1), max(0, pj - cw.y + 1), max(0, pk_ - cw.z + 1)};
    const double w_sqrt_2 = CG_SQRT_2 * g.width;
    for (int i = clo[0]; i <= pi; ++i)
        for (int j = clo[1]; j <= pj; ++j)
            for (int k = clo[2]; k <= pk_; ++k) {
                const int b = (i * g.n[1] + j) * g.n[2] + k;
                for (int e = cstart[b] + lane; e < cend[b]; e += 32) {
                    const CGContact& q = crec[corder[e]];
                    bool in = true;
                    for (int dd = 0; dd < 3; ++dd) in = in && pidx[dd] < q.hi[dd];
                    if (!in) continue;
                    const V3 P = v3(q.P[0], q.P[1], q.P[2]), C = v3(q.C[0], q.C[1], q.C[2]);
                    const V3 Ipos = v3(q.I[0], q.I[1], q.I[2]);
                    double psi;
                    if (g.coord == DEM_CG_O) {
                        psi = 1.0;
                    } else if (fabs(q.nlen) < 1e-10) {
                        psi = cg_phi(g, C, r);
                    } else {
                        double iN, pN, t2;
                        const V3 ie = (q.type != CG_CONTACT_TO_P) ? Ipos : C;
                        const V3 pe = (q.type != CG_I_TO_CONTACT) ? P : C;
                        if (g.coord == DEM_CG_XZ) {
                            iN = (ie.x - r.x) * q.nhat[0] + (ie.z - r.z) * q.nhat[2];
                            pN = (pe.x - r.x) * q.nhat[0] + (pe.z - r.z) * q.nhat[2];
                            t2 = (P.x - r.x) * (P.x - r.x) + (P.z - r.z) * (P.z - r.z) - pN * pN;
                        } else {
                            const V3 n = v3(q.n[0], q.n[1], q.n[2]);
                            iN = dot(ie - r, n);
                            pN = dot(pe - r, n);
                            t2 = len2(P - r) - pN * pN;
                        }
                        if (iN > g.cutoff || pN < -g.cutoff || t2 > g.cutoff * g.cutoff)
                            psi = 0.0;
                        else
                            psi = q.prefactor * (erf(pN / w_sqrt_2) - erf(iN / w_sqrt_2)) *
                                  exp(-0.5 * t2 / (g.width * g.width));
                    }
                    if (psi != 0.0) {
#pragma unroll
                        for (int a = 0; a < 3; ++a)
#pragma unroll
                            for (int bb = 0; bb < 3; ++bb) acc[11 + 3 * a + bb] += q.F[a] * q.branch[bb] * psi;
                    }
                    if (q.type != CG_I_TO_P) {
                        const double phi = cg_phi(g, C, r);
                        if (phi != 0.0) {
                            acc[20] += q.ifd[0] * phi;
                            acc[21] += q.ifd[1] * phi;
                            acc[22] += q.ifd[2] * phi;
                        }
                    }
                }
            }
    // fixed butterfly over the lanes; lane f writes field f
    double mine = 0.0;
#pragma unroll
    for (int f = 0; f < CG_ACC; ++f) {
        double v = acc[f];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == f) mine = v;
    }
    if (lane < CG_ACC) out[(size_t)pt * DEM_CG_NFIELDS + lane] = mine;
}

} // namespace dem

extern "C" int dem_cg_eval(dem_handle* hh, const dem_cg_grid* grid, double* fields_out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !grid || !fields_out) return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: bad arguments");
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    if (!h->records_valid)
        return fail(h, DEM_ERR_CAPACITY, "contact records of the last evaluation overflowed; step again");
    if (grid->coordinates != DEM_CG_O && grid->coordinates != DEM_CG_XZ && grid->coordinates != DEM_CG_XYZ)
        return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: coordinates must be DEM_CG_O, DEM_CG_XZ or DEM_CG_XYZ");
    if (grid->instance < 0 || grid->instance >= (int)h->inst.size())
        return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: instance out of range");
    if (!(grid->width > 0.0)) return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: width must be positive");
    CGDev g{};
    g.coord = grid->coordinates;
    g.instance = grid->instance;
    const bool res[3] = {g.coord != DEM_CG_O, g.coord == DEM_CG_XYZ, g.coord != DEM_CG_O};
    long long npts = 1;
    for (int k = 0; k < 3; ++k) {
        g.resolved[k] = res[k];
        g.n[k] = res[k] ? grid->n[k] : 1;
        if (g.n[k] < 1) return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: point counts must be >= 1");
        g.min[k] = grid->min[k];
        g.max[k] = grid->max[k];
        // spaceEvenly (Kernel/CG/Coordinates/XZ.h:136-152, XYZ.h:189-210)
        g.delta[k] = (g.max[k] - g.min[k]) / g.n[k];
        g.start[k] = g.min[k] + 0.5 * g.delta[k];
        npts *= g.n[k];
    }
    g.width = grid->width;
    g.cutoff = (grid->cutoff_factor > 0.0 ? grid->cutoff_factor : 3.0) * grid->width; // Gauss::setWidth
    // Coordinates::getGaussPrefactor
    const double pf = 1.0 / (CG_SQRT_2 * CG_SQRT_PI * g.width);
    if (g.coord == DEM_CG_XZ) {
        g.prefactor = pf * pf / (1.0 - exp(-0.5 * ((g.cutoff / g.width) * (g.cutoff / g.width))));
    } else if (g.coord == DEM_CG_XYZ) {
        const double cw = g.cutoff / g.width;
        g.prefactor = pf * pf * pf / (erf(cw / CG_SQRT_2) - CG_SQRT_2 / CG_SQRT_PI * cw * exp(-0.5 * (cw * cw)));
    } else {
        g.prefactor = 1.0;
    }
    // CG::volumeAverageVariables: volume of the averaged dimensions
    double volume = 1.0;
    if (g.coord == DEM_CG_XZ) volume = g.max[1] - g.min[1];
    if (g.coord == DEM_CG_O) volume = (g.max[0] - g.min[0]) * (g.max[1] - g.min[1]) * (g.max[2] - g.min[2]);
    CU(cudaSetDevice(h->device));
    using namespace dem;
    const int n = h->d.n;
    const int nrec = (int)h->n_records;
    const size_t nvals = (size_t)npts * DEM_CG_NFIELDS;
    if (npts > (1ll << 30)) return fail(h, DEM_ERR_BAD_INPUT, "dem_cg_eval: too many points");
    int bits = 1; // bin keys 0..npts (npts: the end marker)
    while ((1ll << bits) <= npts) ++bits;
    size_t t1 = 0, t2 = 0, t3 = 0;
    CU(cub::DeviceRadixSort::SortPairs(nullptr, t1, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                       (int*)nullptr, std::max(n, 1), 0, bits, h->stream));
    CU(cub::DeviceRadixSort::SortPairs(nullptr, t2, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                       (const int*)nullptr, (int*)nullptr, std::max(nrec, 1), 0, 64, h->stream));
    CU(cub::DeviceRadixSort::SortPairs(nullptr, t3, (const unsigned*)nullptr, (unsigned*)nullptr, (const int*)nullptr,
                                       (int*)nullptr, std::max(nrec, 1), 0, bits, h->stream));
    const size_t tmp_bytes = std::max(t1, std::max(t2, t3));
    // one scratch arena for the evaluation
    size_t total = 0;
    auto take = [&total](size_t bytes) {
        const size_t at = total;
        total += (bytes + 255) & ~(size_t)255;
        return at;
    };
    const size_t nn = std::max(n, 1), nr = std::max(nrec, 1);
    const size_t o_out = take(nvals * sizeof(double));
    const size_t o_prec = take(nn * sizeof(CGParticle));
    const size_t o_pbin0 = take(nn * 4), o_pbin1 = take(nn * 4), o_pslot0 = take(nn * 4), o_pslot1 = take(nn * 4);
    const size_t o_crec = take(nr * sizeof(CGContact));
    const size_t o_ckey0 = take(nr * 8), o_ckey1 = take(nr * 8), o_cidx0 = take(nr * 4), o_cidx1 = take(nr * 4);
    const size_t o_cbin0 = take(nr * 4), o_cbin1 = take(nr * 4), o_cpos0 = take(nr * 4), o_cpos1 = take(nr * 4);
    const size_t o_bounds = take(4 * (size_t)npts * 4);
    const size_t o_wmax = take(6 * sizeof(int));
    const size_t o_tmp = take(tmp_bytes);
    char* arena = nullptr;
    CU(cudaMallocAsync((void**)&arena, total, h->stream));
    auto at = [arena](size_t off) { return (void*)(arena + off); };
    double* dout = (double*)at(o_out);
    CGParticle* prec = (CGParticle*)at(o_prec);
    unsigned *pbin0 = (unsigned*)at(o_pbin0), *pbin1 = (unsigned*)at(o_pbin1);
    int *pslot0 = (int*)at(o_pslot0), *pslot1 = (int*)at(o_pslot1);
    CGContact* crec = (CGContact*)at(o_crec);
    unsigned long long *ckey0 = (unsigned long long*)at(o_ckey0), *ckey1 = (unsigned long long*)at(o_ckey1);
    int *cidx0 = (int*)at(o_cidx0), *cidx1 = (int*)at(o_cidx1);
    unsigned *cbin0 = (unsigned*)at(o_cbin0), *cbin1 = (unsigned*)at(o_cbin1);
    int *cpos0 = (int*)at(o_cpos0), *cpos1 = (int*)at(o_cpos1);
    int* pstart = (int*)at(o_bounds);
    int *pend = pstart + npts, *cstart = pstart + 2 * npts, *cend = pstart + 3 * npts;
    int* wmax = (int*)at(o_wmax);
    void* tmp = at(o_tmp);
    CU(cudaMemsetAsync(pstart, 0, 4 * (size_t)npts * sizeof(int), h->stream));
    CU(cudaMemsetAsync(wmax, 0, 6 * sizeof(int), h->stream));
    size_t tb;
    if (n > 0) {
        k_cg_prep_particles<<<grid_for(n, 128), 128, 0, h->stream>>>(h->d, g, prec, pbin0, pslot0, wmax);
        tb = tmp_bytes;
        CU(cub::DeviceRadixSort::SortPairs(tmp, tb, pbin0, pbin1, pslot0, pslot1, n, 0, bits, h->stream));
        k_cg_bin_bounds<<<grid_for(n, 256), 256, 0, h->stream>>>(pbin1, n, (int)npts, pstart, pend);
    }
    if (nrec > 0) {
        k_cg_contact_keys<<<grid_for(nrec, 128), 128, 0, h->stream>>>(h->d, (unsigned)nrec, ckey0, cidx0);
        tb = tmp_bytes;
        CU(cub::DeviceRadixSort::SortPairs(tmp, tb, ckey0, ckey1, cidx0, cidx1, nrec, 0, 64, h->stream));
        k_cg_prep_contacts<<<grid_for(nrec, 128), 128, 0, h->stream>>>(h->d, g, (unsigned)nrec, cidx1, crec, cbin0,
                                                                          cpos0, wmax);
        tb = tmp_bytes;
        CU(cub::DeviceRadixSort::SortPairs(tmp, tb, cbin0, cbin1, cpos0, cpos1, nrec, 0, bits, h->stream));
        k_cg_bin_bounds<<<grid_for(nrec, 256), 256, 0, h->stream>>>(cbin1, nrec, (int)npts, cstart, cend);
    }
    int w[6];
    CU(cudaMemcpyAsync(w, wmax, sizeof(w), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    k_cg_gather<<<(unsigned)((npts + CG_GATHER / 32 - 1) / (CG_GATHER / 32)), CG_GATHER, 0, h->stream>>>(g, prec, pslot1, pstart, pend, crec, cpos1, cstart, cend,
                                                            make_int3(w[0], w[1], w[2]), make_int3(w[3], w[4], w[5]),
                                                            dout);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(fields_out, dout, nvals * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaFreeAsync(arena, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < nvals; ++k) fields_out[k] /= volume;
    return DEM_OK;
}
