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
// One thread per particle / per contact record scatters into the point grid
// with FP64 atomics (sums reproducible to rounding, not bit-for-bit); the host
// divides by the volume of the averaged dimensions (CG::volumeAverageVariables).
// The contact records are those of the last force evaluation, i.e. the
// interactions the reference holds when writeOutputFiles evaluates CG at the
// start of the next step. Positions are the particles' own (for a pair that
// meets across a periodic boundary the reference's kept interaction joins the
// two real particles, InteractionHandler.cc:316-368, and CG uses those).
#pragma once

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

__device__ __forceinline__ void cg_add(double* out, int pt, int f, double v) { atomicAdd(out + (size_t)pt * DEM_CG_NFIELDS + f, v); }

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

__global__ void __launch_bounds__(128) k_cg_particles(DevPtrs d, CGDev g, double* out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.n) return;
    const int c = d.ctl->cur;
    const int4 is = d.info[c][s];
    if (is.z != g.instance || (is.w & FLAG_FIXED)) return; // StandardFields::evaluateFixedParticles() is false
    const double4 p4 = d.pr[c][s];
    const double4 v4 = d.vm[c][s];
    const V3 x = xyz(p4), v = xyz(v4);
    const double r = p4.w;
    const double m = 1.0 / v4.w;
    int lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        const double pos = (&x.x)[k] - g.min[k];
        const double invDelta = g.n[k] / (g.max[k] - g.min[k]);
        const double idPos = pos * invDelta - 0.5;
        const double idCutoff = g.cutoff * invDelta;
        cg_range(g, k, idPos - idCutoff, idPos + idCutoff, lo[k], hi[k]);
    }
    // StandardFields::setFields(const BaseParticle&)
    const double vol = 4.0 / 3.0 * CG_PI * r * r * r; // BaseParticle::getVolume (3D)
    const V3 mom = v * m;
    const double flux[6] = {v.x * v.x * m, v.x * v.y * m, v.x * v.z * m, v.y * v.y * m, v.y * v.z * m, v.z * v.z * m};
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                const int pt = (i * g.n[1] + j) * g.n[2] + k;
                const double phi = cg_phi(g, x, cg_point(g, i, j, k));
                if (phi == 0.0) continue;
                cg_add(out, pt, 0, vol * phi);
                cg_add(out, pt, 1, m * phi);
                cg_add(out, pt, 2, mom.x * phi);
                cg_add(out, pt, 3, mom.y * phi);
                cg_add(out, pt, 4, mom.z * phi);
                for (int f = 0; f < 6; ++f) cg_add(out, pt, 5 + f, flux[f] * phi);
                double ps = 1.0;
                for (int f = 0; f < 6; ++f) {
                    cg_add(out, pt, 23 + f, ps * phi);
                    ps *= r;
                }
            }
}

// IntegralType of CG::getIntegralType (CG.hcc:451-466)
enum CGIntegral { CG_NONE = 0, CG_I_TO_P, CG_CONTACT_TO_P, CG_I_TO_CONTACT };

__global__ void __launch_bounds__(128) k_cg_contacts(DevPtrs d, CGDev g, unsigned nrec, double* out)
{
    const unsigned rix = blockIdx.x * blockDim.x + threadIdx.x;
    if (rix >= nrec) return;
    const ContactRecord& rec = d.records[rix];
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
    const double stress[9] = {F.x * branch.x, F.x * branch.y, F.x * branch.z, F.y * branch.x, F.y * branch.y,
                              F.y * branch.z, F.z * branch.x, F.z * branch.y, F.z * branch.z};
    // point range between P and I (the contact point when I is fixed): CG.hcc:478-495
    const V3 Iend = i_fixed ? C : Ipos;
    int lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        if (g.n[k] == 1) {
            lo[k] = 0;
            hi[k] = 1;
            continue;
        }
        const double invDelta = g.n[k] / (g.max[k] - g.min[k]);
        const double pk = ((&P.x)[k] - g.min[k]) * invDelta - 0.5;
        const double ik = ((&Iend.x)[k] - g.min[k]) * invDelta - 0.5;
        const double ck = g.cutoff * invDelta;
        cg_range(g, k, fmin(pk, ik) - ck, fmax(pk, ik) + ck, lo[k], hi[k]);
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
    bool have_prefactor = false;
    double integral_prefactor = 0.0;
    const double w_sqrt_2 = CG_SQRT_2 * g.width;
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                const int pt = (i * g.n[1] + j) * g.n[2] + k;
                const V3 r = cg_point(g, i, j, k);
                double psi;
                if (g.coord == DEM_CG_O) {
                    psi = 1.0;
                } else if (fabs(nlen) < 1e-10) {
                    psi = cg_phi(g, C, r);
                } else {
                    double iN, pN, t2;
                    if (g.coord == DEM_CG_XZ) {
                        const V3 ie = (type != CG_CONTACT_TO_P) ? Ipos : C;
                        const V3 pe = (type != CG_I_TO_CONTACT) ? P : C;
                        iN = (ie.x - r.x) * nhat.x + (ie.z - r.z) * nhat.z;
                        pN = (pe.x - r.x) * nhat.x + (pe.z - r.z) * nhat.z;
                        t2 = (P.x - r.x) * (P.x - r.x) + (P.z - r.z) * (P.z - r.z) - pN * pN;
                    } else {
                        iN = dot(((type != CG_CONTACT_TO_P) ? Ipos : C) - r, n);
                        pN = dot(((type != CG_I_TO_CONTACT) ? P : C) - r, n);
                        t2 = len2(P - r) - pN * pN;
                    }
                    if (iN > g.cutoff || pN < -g.cutoff || t2 > g.cutoff * g.cutoff) {
                        psi = 0.0;
                    } else {
                        if (!have_prefactor) { // the reference computes it at the first point that passes
                            integral_prefactor = cg_integral_prefactor(g, pN - iN);
                            have_prefactor = true;
                        }
                        psi = integral_prefactor * (erf(pN / w_sqrt_2) - erf(iN / w_sqrt_2)) *
                              exp(-0.5 * t2 / (g.width * g.width));
                    }
                }
                if (psi != 0.0)
                    for (int f = 0; f < 9; ++f) cg_add(out, pt, 11 + f, stress[f] * psi);
                if (type != CG_I_TO_P) {
                    const double phi = cg_phi(g, C, r);
                    if (phi != 0.0) {
                        cg_add(out, pt, 20, ifd.x * phi);
                        cg_add(out, pt, 21, ifd.y * phi);
                        cg_add(out, pt, 22, ifd.z * phi);
                    }
                }
            }
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
    const size_t nvals = (size_t)npts * DEM_CG_NFIELDS;
    double* dout = nullptr;
    CU(cudaMallocAsync((void**)&dout, nvals * sizeof(double), h->stream));
    CU(cudaMemsetAsync(dout, 0, nvals * sizeof(double), h->stream));
    k_cg_particles<<<grid_for(h->d.n, 128), 128, 0, h->stream>>>(h->d, g, dout);
    if (h->n_records) k_cg_contacts<<<grid_for(h->n_records, 128), 128, 0, h->stream>>>(h->d, g, h->n_records, dout);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(fields_out, dout, nvals * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaFreeAsync(dout, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < nvals; ++k) fields_out[k] /= volume;
    return DEM_OK;
}
