// dem_engine.cu -- host side of the C ABI (include/dem_b200.h) and the
// device buffers, kernel launches and CUDA graphs of the DEM engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dem_engine.cuh"
#include "dem_walls.cuh"
#include "dem_kernels.cuh"
#include "dem_pipeline.cuh"
#include "dem_rebuild.cuh"
#include "dem_insert.cuh"

using namespace dem;

namespace {

constexpr unsigned FATAL_STATUS =
    (1u << DEM_ERR_CAPACITY) | (1u << DEM_ERR_NAN) | (1u << DEM_ERR_TIMEOUT) | (1u << INS_STATUS_NO_ROW);
constexpr int GRAPH_STEPS = 16;
constexpr int CONTROL_THREADS = 128;

struct Handle {
    dem_config cfg{};
    std::vector<dem_instance_desc> inst_desc;
    std::vector<InstanceDev> inst;
    std::vector<dem_species_pair> species;
    std::vector<dem_wall> walls;       // grouped by instance (stable)
    std::vector<WallGeom> wgeom;       // per wall, for intersection walls
    std::vector<int> wall_caller;      // grouped index -> caller index
    std::vector<int> wall_grouped;     // caller index -> grouped index
    std::vector<dem_deletion_boundary> deletions;
    std::vector<char> wall_removed;    // per wall (grouped order): taken out by dem_remove_wall
    // insertion boundaries (the caller's order) and the generators' seeds per
    // instance; they take effect at the next upload
    std::vector<dem_insertion_boundary> ins;
    std::vector<uint64_t> ins_seeds;
    std::vector<int> ins_order;        // device order (grouped by instance) -> caller index
    InsInstanceDev* d_ins_inst = nullptr;
    InsBoundaryDev* d_ins_bnd = nullptr;
    int* d_ins_rows = nullptr;
    int* d_ovf = nullptr;              // per cell, then per slot twice: k_insert's lists of placed particles
    // radii of a one-instance upload and their statistics (the grid is laid
    // out from them before the particle arrays are allocated)
    double* d_rtmp = nullptr;
    long long rtmp_cap = 0;
    unsigned long long* d_rstats = nullptr;
    int n_ins_inst = 0;                // instances with insertion boundaries or a fill (blocks of k_insert)
    int n_ins_launch = 0;              // blocks of k_insert per step (0: no insertion boundary)
    std::vector<dem_chute_fill> fills; // chute fills of the next upload
    std::vector<FillDev> fill_results; // and their outcome at the last upload
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevPtrs d{};
    // device allocations
    std::vector<void*> allocs;
    size_t alloc_bytes = 0;            // their sizes
    InstanceDev* d_inst = nullptr;
    dem_species_pair* d_species = nullptr;
    dem_wall* d_walls = nullptr;
    WallGeom* d_wgeom = nullptr;
    double* d_stage = nullptr;         // caller-layout particle staging (18 words per slot)
    double* d_batch = nullptr;         // per-instance balance rows of dem_reduce_batch
    std::vector<long long> layout;     // sizes the device arrays were allocated for
    Control* d_ctl = nullptr;
    ContactRecord* d_records = nullptr;
    unsigned record_capacity = 0;
    bool uploaded = false;
    bool initial_pending = false;
    bool records_valid = false;
    unsigned n_records = 0;
    long long steps_total = 0;
    double last_ms = 0.0;
    long long last_launches = 0;
    long long last_rebuilds = 0;
    long long launches_per_step = 0;
    // time steps that are not the last of a dem_step call (1 and GRAPH_STEPS
    // of them), and the last step, which also writes the contact records
    cudaGraphExec_t graph1 = nullptr, graphK = nullptr, graphF = nullptr;
    int ncomp = 3;
    int law_variant = 0;
    int sm_count = 148;
    int rb_grid = 148;                 // blocks of the cooperative rebuild (all resident)
    std::vector<int> level_buf;        // HGrid level of every particle (one-instance uploads)
    // launch shapes of the force kernels (dem_autotune / dem_set_tuning)
    dem_tuning tune{DETECT_BLOCK, 4, SUM_BLOCK, 0, 0.0, 0.0};
    // optional events between the force kernels, for the autotuner's
    // per-kernel times (null outside a measurement)
    cudaEvent_t* kev = nullptr;
};

int fail(Handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    return code;
}

#define CU(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(h, DEM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

template <typename T>
int dalloc(Handle* h, T** p, size_t count)
{
    void* ptr = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&ptr, bytes);
    if (e != cudaSuccess) return fail(h, DEM_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemsetAsync(ptr, 0, bytes, h->stream);
    if (e != cudaSuccess) return fail(h, DEM_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    h->allocs.push_back(ptr);
    h->alloc_bytes += bytes;
    *p = static_cast<T*>(ptr);
    return DEM_OK;
}

void free_graphs(Handle* h)
{
    if (h->graph1) cudaGraphExecDestroy(h->graph1);
    if (h->graphK) cudaGraphExecDestroy(h->graphK);
    if (h->graphF) cudaGraphExecDestroy(h->graphF);
    h->graph1 = h->graphK = h->graphF = nullptr;
}

void free_particle_arrays(Handle* h)
{
    free_graphs(h);
    for (void* p : h->allocs) cudaFree(p);
    h->allocs.clear();
    h->alloc_bytes = 0;
    h->d_records = nullptr;
    h->record_capacity = 0;
    h->d_stage = nullptr;
    h->d_batch = nullptr;
    h->d_ins_inst = nullptr;
    h->d_ins_bnd = nullptr;
    h->d_ins_rows = nullptr;
    h->d_ovf = nullptr;
    h->layout.clear();
}

inline unsigned grid_for(long long n, int block) { return (unsigned)std::max<long long>(1, (n + block - 1) / block); }

// ---- kernel launch sequences ------------------------------------------------
// The rebuild kernel (dem_rebuild.cuh): a cooperative launch, so that its
// grid barriers are safe; it returns at once unless the rebuild flag is set.
cudaError_t launch_rebuild(Handle* h, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)h->rb_grid);
    cfg.blockDim = dim3(RB_BLOCK);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_rebuild, h->d, h->d.rb_barrier);
}
constexpr int REBUILD_LAUNCHES = 1;

InsPtrs ins_ptrs(Handle* h)
{
    const size_t nc = (size_t)h->d.ncells + 1;
    int* o = h->d_ovf;
    return InsPtrs{h->d_ins_inst, h->d_ins_bnd, h->d_ins_rows, o, o ? o + nc : nullptr,
                   o ? o + nc + (size_t)h->d.ncap : nullptr};
}

// Insertion boundaries: one block per instance that has some (dem_insert.cuh),
// after k_control and before the rebuild it may request.
void launch_insert(Handle* h, cudaStream_t s)
{
    if (h->n_ins_launch > 0)
        k_insert<<<h->n_ins_inst, INS_THREADS, 0, s>>>(h->d, ins_ptrs(h));
}
constexpr int FORCE_LAUNCHES = 3;

// Law variants the force kernel is instantiated for; the handle uses a
// specialised one when every species pair shares the same law pair.
enum LawVariant { LAW_GENERIC = 0, LAW_LINEAR_SLIDING, LAW_LINEAR_ROLLING, LAW_HERTZ_MINDLIN, LAW_HERTZ_MINDLIN_RT };

// one force evaluation: detect -> contacts -> sum (+ integration for MODE 1);
// RECORD: the evaluation may be the last of the call (contact records)
template <int MODE, int NLAW, int FLAW, int NCOMP, bool RECORD>
void launch_pipeline(Handle* h, cudaStream_t s)
{
    DevPtrs& d = h->d;
    if (h->kev) cudaEventRecord(h->kev[0], s);
    switch (h->tune.detect_block) {
    case 64: k_detect<MODE, NCOMP, 64><<<grid_for(d.n, 64), 64, 0, s>>>(d); break;
    case 256: k_detect<MODE, NCOMP, 256><<<grid_for(d.n, 256), 256, 0, s>>>(d); break;
    default: k_detect<MODE, NCOMP, DETECT_BLOCK><<<grid_for(d.n, DETECT_BLOCK), DETECT_BLOCK, 0, s>>>(d);
    }
    if (h->kev) cudaEventRecord(h->kev[1], s);
    // one resident wave of tune.contacts_blocks_per_sm blocks of 128 per SM,
    // grid-stride over the items; the time-step variant without records is
    // compiled with that many blocks' register budget (3 to 6), the others
    // with 4 (128 registers)
    const int bpsm = (MODE == 1 && !RECORD) ? h->tune.contacts_blocks_per_sm : 4;
    const unsigned gc = (unsigned)std::max(1, std::min((d.item_cap + CONTACT_BLOCK - 1) / CONTACT_BLOCK,
                                                       h->sm_count * bpsm));
    if (MODE == 1 && !RECORD && bpsm == 3)
        k_contacts<MODE, NLAW, FLAW, NCOMP, RECORD, 3><<<gc, CONTACT_BLOCK, 0, s>>>(d);
    else if (MODE == 1 && !RECORD && bpsm == 5)
        k_contacts<MODE, NLAW, FLAW, NCOMP, RECORD, 5><<<gc, CONTACT_BLOCK, 0, s>>>(d);
    else if (MODE == 1 && !RECORD && bpsm == 6)
        k_contacts<MODE, NLAW, FLAW, NCOMP, RECORD, 6><<<gc, CONTACT_BLOCK, 0, s>>>(d);
    else
        k_contacts<MODE, NLAW, FLAW, NCOMP, RECORD, 4><<<gc, CONTACT_BLOCK, 0, s>>>(d);
    if (d.has_tri) { // at most one triangle item per particle
        const unsigned gt = (unsigned)std::max(1, std::min((d.n + TRI_BLOCK - 1) / TRI_BLOCK, h->sm_count * 4));
        k_tri<MODE, NLAW, FLAW, NCOMP><<<gt, TRI_BLOCK, 0, s>>>(d);
    }
    if (h->kev) cudaEventRecord(h->kev[2], s);
    switch (h->tune.sum_block) {
    case 64: k_sum<MODE, 64><<<grid_for(d.n, 64), 64, 0, s>>>(d); break;
    case 256: k_sum<MODE, 256><<<grid_for(d.n, 256), 256, 0, s>>>(d); break;
    default: k_sum<MODE, SUM_BLOCK><<<grid_for(d.n, SUM_BLOCK), SUM_BLOCK, 0, s>>>(d);
    }
    if (h->kev) cudaEventRecord(h->kev[3], s);
}
int force_launches(const Handle* h) { return FORCE_LAUNCHES + (h->d.has_tri ? 1 : 0); }

template <int MODE, bool RECORD>
void launch_force_mode(Handle* h, cudaStream_t s)
{
    DevPtrs& d = h->d;
    switch (h->law_variant) {
    case LAW_LINEAR_SLIDING:
        launch_pipeline<MODE, DEM_NORMAL_LINEAR_VISCOELASTIC, DEM_FRICTION_SLIDING, 3, RECORD>(h, s);
        break;
    case LAW_LINEAR_ROLLING:
        launch_pipeline<MODE, DEM_NORMAL_LINEAR_VISCOELASTIC, DEM_FRICTION_ROLLING_TORSION, 9, RECORD>(h, s);
        break;
    case LAW_HERTZ_MINDLIN:
        launch_pipeline<MODE, DEM_NORMAL_HERTZIAN_VISCOELASTIC, DEM_FRICTION_MINDLIN, 3, RECORD>(h, s);
        break;
    case LAW_HERTZ_MINDLIN_RT:
        launch_pipeline<MODE, DEM_NORMAL_HERTZIAN_VISCOELASTIC, DEM_FRICTION_MINDLIN_ROLLING_TORSION, 9, RECORD>(h, s);
        break;
    default:
        if (d.ncomp == 3)
            launch_pipeline<MODE, -1, -1, 3, RECORD>(h, s);
        else
            launch_pipeline<MODE, -1, -1, 9, RECORD>(h, s);
    }
}

// mode 0: the initial evaluation (always records); mode 1: a time step,
// `last` when it is the last step of the dem_step call
void launch_force(Handle* h, cudaStream_t s, int mode, bool last = true)
{
    if (mode == 0)
        launch_force_mode<0, true>(h, s);
    else if (last)
        launch_force_mode<1, true>(h, s);
    else
        launch_force_mode<1, false>(h, s);
}

// Captures `steps` time steps: control -> rebuild (returns at once unless
// the skin test fired) -> force; `last`: the final step is the last of the
// dem_step call (its force evaluation writes the contact records).
int build_graph(Handle* h, int steps, bool last, cudaGraphExec_t* out)
{
    cudaStream_t s = h->stream;
    CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < steps; ++k) {
        k_control<<<1, CONTROL_THREADS, 0, s>>>(h->d_ctl, h->d.walls, h->d_wgeom, h->d.n_walls, h->d.dt);
        launch_insert(h, s);
        const cudaError_t e = launch_rebuild(h, s);
        if (e != cudaSuccess) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            return fail(h, DEM_ERR_CUDA, std::string("rebuild launch in capture: ") + cudaGetErrorString(e));
        }
        launch_force(h, s, 1, last && k == steps - 1);
    }
    cudaGraph_t graph = nullptr;
    CU(cudaStreamEndCapture(s, &graph));
    cudaError_t e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(h, DEM_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return DEM_OK;
}

int read_control(Handle* h, Control* c)
{
    CU(cudaMemcpyAsync(c, h->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}

// Bands of radii (setup_instance_grid): ratio 2 from the smallest radius, at
// most DEM_MAX_LEVELS of them.
int band_count(double rmin, double rmax)
{
    int nl = 1;
    while (nl < DEM_MAX_LEVELS && rmax >= rmin * std::pow(2.0, nl)) ++nl;
    return nl;
}

// What setup_instance_grid needs of the radii, measured on the device for a
// one-instance upload: extremes and the largest radius of each band.
struct BandStats {
    double rmin, rmax;
    double lrmax[DEM_MAX_LEVELS];
};

// The radii of a one-instance upload on the device: extremes and validity
// (k_radius_extremes), then, if all are positive and finite, the largest
// radius of every band (k_radius_bands). `ok` is false when some radius is
// bad (the host check then names it).
int radius_stats(Handle* h, const double* radius, long long n, BandStats& st, bool& ok)
{
    if (n > h->rtmp_cap) {
        if (h->d_rtmp) cudaFree(h->d_rtmp);
        h->d_rtmp = nullptr;
        h->rtmp_cap = 0;
        CU(cudaMalloc(&h->d_rtmp, (size_t)n * sizeof(double)));
        h->rtmp_cap = n;
    }
    if (!h->d_rstats) CU(cudaMalloc(&h->d_rstats, (3 + DEM_MAX_LEVELS) * sizeof(unsigned long long)));
    unsigned long long init[3 + DEM_MAX_LEVELS] = {(unsigned long long)__builtin_bit_cast(long long, DBL_MAX), 0ull, 0ull};
    for (int k = 0; k < DEM_MAX_LEVELS; ++k) init[3 + k] = 0ull;
    CU(cudaMemcpyAsync(h->d_rtmp, radius, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->d_rstats, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
    const unsigned blocks = std::min<unsigned>(grid_for(n, 256), 4u * (unsigned)h->sm_count);
    k_radius_extremes<<<blocks, 256, 0, h->stream>>>(h->d_rtmp, (int)n, h->d_rstats);
    CU(cudaGetLastError());
    unsigned long long out[3 + DEM_MAX_LEVELS];
    CU(cudaMemcpyAsync(out, h->d_rstats, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    ok = out[2] == 0ull;
    if (!ok) return DEM_OK;
    st.rmin = __builtin_bit_cast(double, out[0]);
    st.rmax = __builtin_bit_cast(double, out[1]);
    const int nl = band_count(st.rmin, st.rmax);
    k_radius_bands<<<blocks, 256, 0, h->stream>>>(h->d_rtmp, (int)n, st.rmin, nl, h->d_rstats + 3);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out + 3, h->d_rstats + 3, DEM_MAX_LEVELS * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < DEM_MAX_LEVELS; ++k) st.lrmax[k] = __builtin_bit_cast(double, out[3 + k]);
    return DEM_OK;
}

int check_status(Handle* h, const Control& c)
{
    const unsigned st = c.status & FATAL_STATUS;
    if (!st) return DEM_OK;
    if (st & (1u << DEM_ERR_CAPACITY))
        return fail(h, DEM_ERR_CAPACITY, "neighbour-list capacity exceeded (max_neighbors=" +
                                             std::to_string(h->d.cap) + "); raise dem_config.max_neighbors");
    if (st & (1u << DEM_ERR_NAN)) return fail(h, DEM_ERR_NAN, "non-finite force detected");
    if (st & (1u << INS_STATUS_NO_ROW))
        return fail(h, DEM_ERR_CAPACITY, "an insertion boundary found no free row (upload more rows of radius 0)");
    // a rebuild block gave up at a grid barrier: the arrival counter no longer
    // sits on a multiple of the launch's barriers, so it starts again at zero
    if (h->d.rb_barrier) cudaMemsetAsync(h->d.rb_barrier, 0, sizeof(unsigned long long), h->stream);
    return fail(h, DEM_ERR_TIMEOUT, "device wait timed out");
}

// Levels and cell grid of one instance (MercuryBase::hGridRebuild,
// MercuryBase.cc:204-306, restated as dense per-level grids): radii are
// grouped in geometric bands of ratio 2 starting at the smallest radius; a
// level's cell edge is at least 2 r_max(level) + interaction distance + skin.
// [psd_lo, psd_hi] (psd_hi > 0): radii insertion boundaries may place later;
// every band they reach gets a level sized for its largest radius.
void setup_instance_grid(const dem_instance_desc& in, const double* radii, size_t count, double skin, double dmax,
                         double psd_lo, double psd_hi, InstanceDev& I, std::vector<int>& level_of, int& cell_base,
                         const BandStats* pre = nullptr)
{
    double rmin = 1e300, rmax = 0.0;
    if (pre) {
        rmin = pre->rmin;
        rmax = pre->rmax;
    } else {
        for (size_t i = 0; i < count; ++i) { rmin = std::min(rmin, radii[i]); rmax = std::max(rmax, radii[i]); }
    }
    const bool psd = psd_hi > 0.0;
    // a little above the largest PSD radius: PSD::drawSample's interpolation rounds
    const double phi = psd_hi * (1.0 + 1e-12);
    if (psd) {
        rmin = std::min(rmin, psd_lo);
        rmax = std::max(rmax, phi);
    }
    const bool empty = count == 0 && !psd;
    if (empty) { rmin = rmax = 1.0; }
    const int nl = band_count(rmin, rmax);
    std::vector<double> lrmax(nl, 0.0);
    std::vector<int> used(nl, 0);
    if (pre) // the levels themselves are computed by k_pack
        for (int l = 0; l < nl; ++l) {
            lrmax[l] = pre->lrmax[l];
            used[l] = pre->lrmax[l] > 0.0;
        }
    else
        level_of.resize(count);
    for (size_t i = 0; i < count && !pre; ++i) {
        // floor(log2(r / rmin)) is the binary exponent of r / rmin >= 1 (a
        // normal number): exact, and far cheaper than log2 for millions of
        // particles
        const double x = radii[i] / rmin;
        uint64_t bits;
        std::memcpy(&bits, &x, sizeof(bits));
        int l = (int)((bits >> 52) & 0x7ffu) - 1023;
        l = std::max(0, std::min(nl - 1, l));
        level_of[i] = l;
        lrmax[l] = std::max(lrmax[l], radii[i]);
        used[l] = 1;
    }
    if (psd) {
        auto band = [&](double r) {
            const double x = r / rmin;
            uint64_t bits;
            std::memcpy(&bits, &x, sizeof(bits));
            return std::max(0, std::min(nl - 1, (int)((bits >> 52) & 0x7ffu) - 1023));
        };
        const int b0 = band(psd_lo), b1 = band(phi);
        for (int l = b0; l <= b1; ++l) { // a band's radii lie below rmin 2^(l+1)
            used[l] = 1;
            lrmax[l] = std::max(lrmax[l], l == b1 ? phi : std::min(phi, std::ldexp(rmin, l + 1)));
        }
    }
    // drop empty levels
    std::vector<int> remap(nl, -1);
    int nu = 0;
    std::vector<double> lr;
    for (int l = 0; l < nl; ++l)
        if (used[l] || empty) { remap[l] = nu++; lr.push_back(lrmax[l] > 0 ? lrmax[l] : rmax); }
    if (nu != nl && !pre) // some level is empty: renumber (usually every level is used)
        for (size_t i = 0; i < count; ++i) level_of[i] = remap[level_of[i]];
    I.n_levels = nu;
    I.level_rmin = rmin;
    I.level_bands = nl;
    for (int l = 0; l < DEM_MAX_LEVELS; ++l) I.level_remap[l] = l < nl ? remap[l] : -1;
    for (int l = 0; l < nu; ++l) {
        const double cs = 2.0 * lr[l] + dmax + skin;
        I.level_rmax[l] = lr[l];
        I.cell_base[l] = cell_base;
        int total = 1;
        for (int k = 0; k < 3; ++k) {
            const bool per = (in.periodic_mask >> k) & 1u;
            int dim;
            if (per) {
                const double L = in.periodic_max[k] - in.periodic_min[k];
                dim = std::max(1, (int)std::floor(L / cs));
                I.inv_cell[l][k] = (double)dim / L;
            } else {
                const double ext = in.domain_max[k] - in.domain_min[k];
                dim = std::max(1, (int)std::ceil(ext / cs));
                I.inv_cell[l][k] = 1.0 / cs;
            }
            I.dims[l][k] = dim;
            total *= dim;
        }
        cell_base += total;
    }
}

} // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

int dem_create(const dem_config* config, const dem_instance_desc* instances, dem_handle** out)
{
    Handle* h = nullptr;
    if (!config || !out || !instances) return DEM_ERR_BAD_INPUT;
    if (config->n_instances < 1 || !(config->time_step > 0.0)) return DEM_ERR_BAD_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DEM_ERR_CUDA;
    if (config->device < 0 || config->device >= ndev) return DEM_ERR_BAD_INPUT;
    h = new Handle();
    h->cfg = *config;
    h->device = config->device;
    h->inst_desc.assign(instances, instances + config->n_instances);
    for (const auto& in : h->inst_desc) {
        for (int k = 0; k < 3; ++k) {
            if ((in.periodic_mask >> k) & 1u) {
                if (!(in.periodic_max[k] > in.periodic_min[k])) {
                    delete h;
                    return DEM_ERR_BAD_INPUT;
                }
            } else if (!(in.domain_max[k] > in.domain_min[k])) {
                delete h;
                return DEM_ERR_BAD_INPUT;
            }
        }
    }
    if (cudaSetDevice(h->device) != cudaSuccess || cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
        delete h;
        return DEM_ERR_CUDA;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess && sms > 0)
        h->sm_count = sms;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rebuild, RB_BLOCK, 0) != cudaSuccess || per_sm < 1) {
        cudaStreamDestroy(h->stream);
        cudaStreamDestroy(h->stream2);
        cudaEventDestroy(h->ev0);
        cudaEventDestroy(h->ev1);
        delete h;
        return DEM_ERR_CUDA;
    }
    h->rb_grid = h->sm_count * per_sm;
    *out = reinterpret_cast<dem_handle*>(h);
    return DEM_OK;
}

int dem_set_species(dem_handle* hh, const dem_species_pair* table, int n_entries)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !table || n_entries <= 0) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_species: empty table");
    size_t need = 0;
    for (const auto& in : h->inst_desc) {
        if (in.n_species <= 0 || in.species_offset < 0) return fail(h, DEM_ERR_BAD_INPUT, "instance without species");
        need = std::max(need, (size_t)in.species_offset + (size_t)in.n_species * in.n_species);
    }
    if ((size_t)n_entries < need) return fail(h, DEM_ERR_BAD_INPUT, "species table smaller than the instances need");
    h->species.assign(table, table + n_entries);
    h->ncomp = 3;
    const int n0 = table[0].normal_law, f0 = table[0].friction_law;
    bool same = true;
    for (const auto& s : h->species) same = same && s.normal_law == n0 && s.friction_law == f0;
    h->law_variant = LAW_GENERIC;
    if (same) {
        if (n0 == DEM_NORMAL_LINEAR_VISCOELASTIC && f0 == DEM_FRICTION_SLIDING) h->law_variant = LAW_LINEAR_SLIDING;
        if (n0 == DEM_NORMAL_LINEAR_VISCOELASTIC && f0 == DEM_FRICTION_ROLLING_TORSION) h->law_variant = LAW_LINEAR_ROLLING;
        if (n0 == DEM_NORMAL_HERTZIAN_VISCOELASTIC && f0 == DEM_FRICTION_MINDLIN) h->law_variant = LAW_HERTZ_MINDLIN;
        if (n0 == DEM_NORMAL_HERTZIAN_VISCOELASTIC && f0 == DEM_FRICTION_MINDLIN_ROLLING_TORSION)
            h->law_variant = LAW_HERTZ_MINDLIN_RT;
    }
    for (const auto& s : h->species) {
        if (s.friction_law == DEM_FRICTION_ROLLING_TORSION || s.friction_law == DEM_FRICTION_MINDLIN_ROLLING_TORSION)
            h->ncomp = 9;
        if (s.normal_law < 0 || s.normal_law > 1 || s.friction_law < 0 || s.friction_law > 4)
            return fail(h, DEM_ERR_BAD_INPUT, "unknown contact law");
    }
    return DEM_OK;
}

int dem_set_periodic(dem_handle* hh, int instance, const double lo[3], const double hi[3], uint32_t mask)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || mask > 7u || ((mask != 0u) && (!lo || !hi))) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_periodic: bad arguments");
    if (instance < 0 || instance >= (int)h->inst_desc.size())
        return fail(h, DEM_ERR_BAD_INPUT, "dem_set_periodic: instance out of range");
    if (h->uploaded) return fail(h, DEM_ERR_STATE, "dem_set_periodic must come before dem_upload_particles");
    dem_instance_desc in = h->inst_desc[instance];
    for (int k = 0; k < 3; ++k) {
        if ((mask >> k) & 1u) {
            if (!(std::isfinite(lo[k]) && std::isfinite(hi[k]) && hi[k] > lo[k]))
                return fail(h, DEM_ERR_BAD_INPUT, "dem_set_periodic: empty periodic interval");
            in.periodic_min[k] = lo[k];
            in.periodic_max[k] = hi[k];
        } else {
            if (!(in.domain_max[k] > in.domain_min[k]))
                return fail(h, DEM_ERR_BAD_INPUT, "dem_set_periodic: a non-periodic direction needs a domain");
            in.periodic_min[k] = 0.0;
            in.periodic_max[k] = 0.0;
        }
    }
    in.periodic_mask = mask;
    h->inst_desc[instance] = in;
    return DEM_OK;
}

int dem_set_walls(dem_handle* hh, const dem_wall* walls, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || (n > 0 && !walls)) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_walls: bad arguments");
    if (h->uploaded) return fail(h, DEM_ERR_STATE, "dem_set_walls must come before dem_upload_particles");
    std::vector<int> order(n);
    for (int k = 0; k < n; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return walls[a].instance < walls[b].instance; });
    std::vector<dem_wall> w(n);
    std::vector<WallGeom> g(n);
    std::vector<int> grouped(n);
    for (int k = 0; k < n; ++k) {
        const dem_wall& x = walls[order[k]];
        if (x.instance < 0 || x.instance >= (int)h->inst_desc.size())
            return fail(h, DEM_ERR_BAD_INPUT, "wall instance out of range");
        if (x.type != DEM_WALL_INFINITE && x.type != DEM_WALL_AXISYMMETRIC && x.type != DEM_WALL_INTERSECTION &&
            x.type != DEM_WALL_TRIANGLE)
            return fail(h, DEM_ERR_BAD_INPUT, "unknown wall type");
        if (x.type == DEM_WALL_TRIANGLE && (x.n_faces != 3 || x.group < 0))
            return fail(h, DEM_ERR_BAD_INPUT, "a triangle wall has n_faces 3 and a group >= 0");
        if (x.n_faces < 0 || x.n_faces > DEM_MAX_WALL_FACES) return fail(h, DEM_ERR_BAD_INPUT, "too many wall faces");
        if (x.species < 0 || x.species >= h->inst_desc[x.instance].n_species)
            return fail(h, DEM_ERR_BAD_INPUT, "wall species out of range");
        bool finite = true;
        for (int a = 0; a < 3; ++a)
            finite = finite && std::isfinite(x.position[a]) && std::isfinite(x.velocity[a]) &&
                     std::isfinite(x.angular_velocity[a]);
        for (int a = 0; a < 4; ++a) finite = finite && std::isfinite(x.orientation[a]);
        if (!finite) return fail(h, DEM_ERR_BAD_INPUT, "non-finite wall state");
        if (x.type == DEM_WALL_TRIANGLE) {
            for (int f = 0; f < 3; ++f)
                for (int a = 0; a < 3; ++a) finite = finite && std::isfinite(x.faces[f][a]);
            if (!finite) return fail(h, DEM_ERR_BAD_INPUT, "non-finite triangle vertex");
            const V3 e0 = row3(x.faces[1]) - row3(x.faces[0]), e1 = row3(x.faces[2]) - row3(x.faces[1]);
            if (!(len2(cross(e0, e1)) > 0.0)) return fail(h, DEM_ERR_BAD_INPUT, "degenerate triangle wall");
            build_wall_geom(x, g[k]);
        } else if (x.type != DEM_WALL_INFINITE) {
            for (int f = 0; f < x.n_faces; ++f) {
                const double l2 = x.faces[f][0] * x.faces[f][0] + x.faces[f][1] * x.faces[f][1] +
                                  x.faces[f][2] * x.faces[f][2];
                if (!(l2 > 0.0) || !std::isfinite(l2)) return fail(h, DEM_ERR_BAD_INPUT, "wall face normal of length 0");
            }
            build_wall_geom(x, g[k]);
        } else {
            std::memset(&g[k], 0, sizeof(WallGeom));
        }
        w[k] = x;
        grouped[order[k]] = k;
    }
    h->walls = std::move(w);
    h->wgeom = std::move(g);
    h->wall_caller = std::move(order);
    h->wall_grouped = std::move(grouped);
    h->wall_removed.assign(n, 0);
    return DEM_OK;
}

// DeletionBoundary planes of instance `in` (DeletionBoundary::set normalises,
// DeletionBoundary.cc:86-91).
static void fill_deletions(const Handle* h, InstanceDev& I, int in)
{
    I.n_del = 0;
    for (const auto& db : h->deletions)
        if (db.instance == in) {
            const double sf = 1. / std::sqrt(db.normal[0] * db.normal[0] + db.normal[1] * db.normal[1] +
                                             db.normal[2] * db.normal[2]);
            for (int a = 0; a < 3; ++a) I.del_n[I.n_del][a] = db.normal[a] * sf;
            I.del_d[I.n_del] = db.distance * sf;
            ++I.n_del;
        }
}

// The instance table changed between steps: the next launches read the new one.
static int push_instances(Handle* h)
{
    CU(cudaSetDevice(h->device));
    CU(cudaMemcpyAsync(h->d_inst, h->inst.data(), h->inst.size() * sizeof(InstanceDev), cudaMemcpyHostToDevice,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}

int dem_remove_wall(dem_handle* hh, int wall)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || wall < 0 || wall >= (int)h->walls.size()) return fail(h, DEM_ERR_BAD_INPUT, "dem_remove_wall: no such wall");
    const int g = h->wall_grouped[wall];
    if (h->walls[g].type == DEM_WALL_TRIANGLE)
        return fail(h, DEM_ERR_BAD_INPUT, "dem_remove_wall: triangle walls cannot be taken out");
    h->wall_removed[g] = 1;
    if (!h->uploaded) return DEM_OK; // applied when the particles are uploaded
    const int in = h->walls[g].instance;
    h->inst[in].wall_off_mask |= 1u << (g - h->inst[in].wall_begin);
    return push_instances(h);
}

int dem_set_insertion_boundaries(dem_handle* hh, const dem_insertion_boundary* b, int n, const uint64_t* seeds)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || (n > 0 && !b)) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_insertion_boundaries: bad arguments");
    const int ninst = (int)h->inst_desc.size();
    std::vector<int> per(ninst, 0);
    auto finite = [](double x) { return std::isfinite(x); };
    for (int k = 0; k < n; ++k) {
        const dem_insertion_boundary& x = b[k];
        if (x.kind != DEM_INSERTION_CUBE && x.kind != DEM_INSERTION_CHUTE)
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: unknown kind");
        if (x.instance < 0 || x.instance >= ninst) return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: instance out of range");
        if (++per[x.instance] > DEM_MAX_INSERTION_PER_INSTANCE)
            return fail(h, DEM_ERR_BAD_INPUT, "more than DEM_MAX_INSERTION_PER_INSTANCE insertion boundaries in an instance");
        if (x.species < 0 || x.species >= h->inst_desc[x.instance].n_species)
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: species out of range");
        if (x.max_failed < 0) return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: max_failed must be >= 0");
        if (x.n_psd < 2 || x.n_psd > DEM_MAX_PSD_POINTS)
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: n_psd must be in 2..DEM_MAX_PSD_POINTS");
        if (!(x.density > 0.0) || !finite(x.density)) return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: bad density");
        if (!(x.volume_flow_rate >= 0.0) || !finite(x.initial_volume))
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: bad volume flow rate or initial volume");
        for (int a = 0; a < 3; ++a)
            if (!finite(x.pos_min[a]) || !finite(x.pos_max[a]) || !(x.pos_min[a] <= x.pos_max[a]) ||
                !finite(x.vel_min[a]) || !finite(x.vel_max[a]) || !(x.vel_min[a] <= x.vel_max[a]))
                return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: bad position or velocity range");
        if (!finite(x.fixed_particle_radius) || !finite(x.inflow_velocity) || !(x.inflow_velocity_variance >= 0.0) ||
            !finite(x.inflow_velocity_variance))
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: bad chute inflow parameters");
        // a cumulative number distribution from 0 to 1 over positive radii
        // (PSD::validateCumulativeDistribution's result)
        for (int j = 0; j < x.n_psd; ++j) {
            if (!(x.psd_radius[j] > 0.0) || !finite(x.psd_radius[j]))
                return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: PSD radii must be positive");
            if (j > 0 && !(x.psd_probability[j] >= x.psd_probability[j - 1]))
                return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: PSD probabilities must not decrease");
        }
        if (x.psd_probability[0] != 0.0 || x.psd_probability[x.n_psd - 1] != 1.0)
            return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary: PSD probabilities must run from 0 to 1");
    }
    h->ins.assign(b, b + n);
    h->ins_seeds.assign(ninst, 0);
    if (seeds) h->ins_seeds.assign(seeds, seeds + ninst);
    return DEM_OK;
}

int dem_set_chute_fills(dem_handle* hh, const dem_chute_fill* f, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || (n > 0 && !f)) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_chute_fills: bad arguments");
    const int ninst = (int)h->inst_desc.size();
    std::vector<int> per(ninst, 0);
    for (int k = 0; k < n; ++k) {
        const dem_chute_fill& x = f[k];
        if (x.instance < 0 || x.instance >= ninst) return fail(h, DEM_ERR_BAD_INPUT, "chute fill: instance out of range");
        if (++per[x.instance] > 1) return fail(h, DEM_ERR_BAD_INPUT, "chute fill: at most one per instance");
        if (x.species < 0 || x.species >= h->inst_desc[x.instance].n_species)
            return fail(h, DEM_ERR_BAD_INPUT, "chute fill: species out of range");
        const double v[] = {x.density, x.x_min, x.x_max, x.y_min, x.y_max, x.z_min, x.inflow_height, x.min_radius,
                            x.max_radius, x.fixed_particle_radius};
        for (double a : v)
            if (!std::isfinite(a)) return fail(h, DEM_ERR_BAD_INPUT, "chute fill: non-finite parameter");
        if (!(x.density > 0.0) || !(x.min_radius > 0.0) || !(x.max_radius >= x.min_radius) ||
            !(x.fixed_particle_radius >= 0.0) || !(x.x_max > x.x_min) || !(x.y_max > x.y_min))
            return fail(h, DEM_ERR_BAD_INPUT, "chute fill: bad radii, density or ranges");
    }
    h->fills.assign(f, f + n);
    return DEM_OK;
}

int dem_get_chute_fill_results(dem_handle* hh, double* inflow_height, int64_t* added, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || n > (int)h->fill_results.size())
        return fail(h, DEM_ERR_BAD_INPUT, "dem_get_chute_fill_results: bad arguments");
    for (int k = 0; k < n; ++k) {
        if (inflow_height) inflow_height[k] = h->fill_results[k].height;
        if (added) added[k] = h->fill_results[k].added;
    }
    return DEM_OK;
}

int dem_get_insertion_counts(dem_handle* hh, int64_t* inserted, double* volume, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || n > (int)h->ins.size()) return fail(h, DEM_ERR_BAD_INPUT, "dem_get_insertion_counts: bad arguments");
    if (!h->uploaded || h->n_ins_inst == 0 || h->ins_order.size() != h->ins.size())
        return fail(h, DEM_ERR_STATE, "no insertion boundaries uploaded");
    CU(cudaSetDevice(h->device));
    std::vector<InsBoundaryDev> bnd(h->ins.size());
    CU(cudaMemcpyAsync(bnd.data(), h->d_ins_bnd, bnd.size() * sizeof(InsBoundaryDev), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < bnd.size(); ++k) {
        const int i = h->ins_order[k];
        if (i >= n) continue;
        if (inserted) inserted[i] = bnd[k].n_inserted;
        if (volume) volume[i] = bnd[k].volume_inserted;
    }
    return DEM_OK;
}

int dem_psd_draws(const dem_insertion_boundary* b, int n, double* out)
{
    if (!b || n < 0 || (n > 0 && !out) || b->n_psd < 2 || b->n_psd > DEM_MAX_PSD_POINTS) return DEM_ERR_BAD_INPUT;
    Lfg g;
    lfg_seed(b->psd_seed, g);
    for (int i = 0; i < n; ++i) out[i] = psd_draw(*b, g.v, g.head);
    return DEM_OK;
}

int dem_rng_draws(uint64_t seed, int n, double* out)
{
    if (n < 0 || (n > 0 && !out)) return DEM_ERR_BAD_INPUT;
    Lfg g;
    lfg_seed(seed, g);
    for (int i = 0; i < n; ++i) out[i] = lfg_uniform(g.v, g.head, 0.0, 1.0);
    return DEM_OK;
}

int dem_set_deletion_boundaries(dem_handle* hh, const dem_deletion_boundary* b, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || (n > 0 && !b)) return fail(h, DEM_ERR_BAD_INPUT, "dem_set_deletion_boundaries: bad arguments");
    std::vector<int> per(h->inst_desc.size(), 0);
    for (int k = 0; k < n; ++k) {
        if (b[k].instance < 0 || b[k].instance >= (int)h->inst_desc.size())
            return fail(h, DEM_ERR_BAD_INPUT, "deletion boundary instance out of range");
        if (++per[b[k].instance] > DEM_MAX_DELETION_PER_INSTANCE)
            return fail(h, DEM_ERR_BAD_INPUT, "too many deletion boundaries in one instance");
        bool finite = std::isfinite(b[k].distance);
        for (int a = 0; a < 3; ++a) finite = finite && std::isfinite(b[k].normal[a]);
        const double l2 = b[k].normal[0] * b[k].normal[0] + b[k].normal[1] * b[k].normal[1] +
                          b[k].normal[2] * b[k].normal[2];
        if (!finite || !(l2 > 0.0)) return fail(h, DEM_ERR_BAD_INPUT, "bad deletion boundary");
    }
    h->deletions.assign(b, b + n);
    if (!h->uploaded) return DEM_OK;
    // during the run (BoundaryHandler::copyAndAddObject between time steps):
    // the planes apply from the next drift on
    for (int in = 0; in < (int)h->inst.size(); ++in) fill_deletions(h, h->inst[in], in);
    return push_instances(h);
}

int dem_upload_particles(dem_handle* hh, const dem_particles_soa* p)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !p || p->n < 0 || p->n > (1ll << 30)) return fail(h, DEM_ERR_BAD_INPUT, "dem_upload_particles: bad arguments");
    if (h->species.empty()) return fail(h, DEM_ERR_STATE, "dem_set_species must come before dem_upload_particles");
    const long long n = p->n;
    if (n > 0 && (!p->position || !p->velocity || !p->radius || !p->inv_mass || !p->species || !p->id))
        return fail(h, DEM_ERR_BAD_INPUT, "missing particle arrays");
    CU(cudaSetDevice(h->device));
    const int ninst = (int)h->inst_desc.size();
    // ---- validate and collect per-instance radii
    std::vector<std::vector<double>> radii(ninst);
    std::vector<std::vector<long long>> members(ninst);
    const bool one = ninst == 1;
    // insertion boundaries: the radius range of each instance's PSDs; rows of
    // such an instance with radius 0 are its free rows
    std::vector<double> psd_lo(ninst, 0.0), psd_hi(ninst, 0.0);
    std::vector<char> has_ins(ninst, 0);
    for (const auto& b : h->ins) {
        if (b.instance >= ninst) return fail(h, DEM_ERR_BAD_INPUT, "insertion boundary instance out of range");
        for (int k = 0; k < b.n_psd; ++k) {
            const double r = b.psd_radius[k];
            psd_lo[b.instance] = has_ins[b.instance] ? std::min(psd_lo[b.instance], r) : r;
            psd_hi[b.instance] = std::max(psd_hi[b.instance], r);
            has_ins[b.instance] = 1;
        }
    }
    std::vector<int> fill_of(ninst, -1);
    for (size_t k = 0; k < h->fills.size(); ++k) {
        const dem_chute_fill& f = h->fills[k];
        if (f.instance >= ninst) return fail(h, DEM_ERR_BAD_INPUT, "chute fill instance out of range");
        fill_of[f.instance] = (int)k;
        for (double r : {f.min_radius, f.max_radius}) {
            psd_lo[f.instance] = has_ins[f.instance] ? std::min(psd_lo[f.instance], r) : r;
            psd_hi[f.instance] = std::max(psd_hi[f.instance], r);
            has_ins[f.instance] = 1;
        }
    }
    const bool any_free = !h->ins.empty() || !h->fills.empty();
    std::vector<std::vector<int>> free_rows(ninst);
    // one instance without insertion: members are 0..n-1, radii the caller's array itself
    const bool fast = one && !any_free;
    double rmin_all = 1e300;
    // one instance: the host reads only the radii (their minimum sets the skin
    // and the grid); k_pack checks every other array on the device, and the
    // loop below runs only to name a failure it reports
    bool checked = false;
    BandStats pre{};
    if (fast && n > 0) { // the radii's extremes and bands from the device, not host loops
        bool ok = false;
        if (int rc0 = radius_stats(h, p->radius, n, pre, ok)) return rc0;
        if (ok) {
            checked = true;
            rmin_all = pre.rmin;
        }
    }
    const bool levels_here = fast && checked; // k_pack computes the levels
    auto validate = [&]() -> int { // every particle on the host, in caller order: names the first violation
        for (long long i = 0; i < n; ++i) {
            const int in = p->instance ? p->instance[i] : 0;
            if (in < 0 || in >= ninst) return fail(h, DEM_ERR_BAD_INPUT, "particle instance out of range");
            const double r = p->radius[i];
            if (r == 0.0 && has_ins[in]) continue; // a free row
            if (!(r > 0.0) || !std::isfinite(r)) return fail(h, DEM_ERR_BAD_INPUT, "particle radius must be positive");
            if (p->species[i] < 0 || p->species[i] >= h->inst_desc[in].n_species)
                return fail(h, DEM_ERR_BAD_INPUT, "particle species out of range");
            if (!(p->inv_mass[i] >= 0.0)) return fail(h, DEM_ERR_BAD_INPUT, "inverse mass must be >= 0");
            for (int k = 0; k < 3; ++k)
                if (!std::isfinite(p->position[3 * i + k]) || !std::isfinite(p->velocity[3 * i + k]))
                    return fail(h, DEM_ERR_BAD_INPUT, "non-finite particle state");
        }
        return DEM_OK;
    };
    if (!checked) {
        if (int rc0 = validate()) return rc0;
        for (long long i = 0; i < n; ++i) {
            const int in = p->instance ? p->instance[i] : 0;
            const double r = p->radius[i];
            if (r == 0.0 && has_ins[in]) {
                free_rows[in].push_back((int)i);
                continue;
            }
            if (!fast) {
                radii[in].push_back(r);
                members[in].push_back(i);
            }
            rmin_all = std::min(rmin_all, r);
        }
    }
    for (int in = 0; in < ninst; ++in)
        if (has_ins[in]) rmin_all = std::min(rmin_all, psd_lo[in]);
    // ---- walls per instance
    std::vector<int> wbegin(ninst, 0), wend(ninst, 0);
    {
        int w = 0;
        for (int in = 0; in < ninst; ++in) {
            wbegin[in] = w;
            while (w < (int)h->walls.size() && h->walls[w].instance == in) ++w;
            wend[in] = w;
            if (wend[in] - wbegin[in] > DEM_MAX_WALLS_PER_INSTANCE)
                return fail(h, DEM_ERR_BAD_INPUT, "more than 32 walls in one instance");
        }
    }
    int wmax = 1;
    for (int in = 0; in < ninst; ++in) wmax = std::max(wmax, wend[in] - wbegin[in]);
    // ---- skin and levels
    double skin = h->cfg.skin;
    // auto: 0.4 of the smallest radius (measured on the 200k chute: 0.2 rebuilds
    // every 9 steps and costs 7 % more per step; the evaluation grows only 3 %)
    if (!(skin > 0.0)) skin = (n > 0) ? 0.4 * rmin_all : 1e-3;
    h->inst.assign(ninst, InstanceDev{});
    // levels of all particles; one instance fills the handle's buffer, which
    // keeps its size between uploads (no allocation or zeroing per upload)
    std::vector<int> level_multi(fast ? 0 : n, 0);
    std::vector<int>& level = fast ? h->level_buf : level_multi;
    double rmax_all = 0.0;
    int cell_base = 0;
    for (int in = 0; in < ninst; ++in) {
        const auto& D = h->inst_desc[in];
        InstanceDev& I = h->inst[in];
        double dmax = 0.0;
        for (int a = 0; a < D.n_species; ++a)
            for (int b = 0; b < D.n_species; ++b)
                dmax = std::max(dmax, h->species[D.species_offset + a * D.n_species + b].interaction_distance);
        I.max_interaction_distance = dmax;
        for (int k = 0; k < 3; ++k) {
            I.gravity[k] = D.gravity[k];
            const bool per = (D.periodic_mask >> k) & 1u;
            I.origin[k] = per ? D.periodic_min[k] : D.domain_min[k];
            I.per_lo[k] = D.periodic_min[k];
            I.per_hi[k] = D.periodic_max[k];
            I.per_L[k] = D.periodic_max[k] - D.periodic_min[k];
            I.per_half[k] = 0.5 * I.per_L[k];
        }
        I.per_mask = D.periodic_mask;
        I.species_offset = D.species_offset;
        I.n_species = D.n_species;
        I.wall_begin = wbegin[in];
        I.wall_end = wend[in];
        I.tri_mask = 0u;
        I.tri_static = 1;
        I.wall_still_mask = 0u;
        I.wall_off_mask = 0u;
        for (int w = wbegin[in]; w < wend[in]; ++w)
            if (h->wall_removed[w]) I.wall_off_mask |= 1u << (w - wbegin[in]);
        for (int w = wbegin[in]; w < wend[in]; ++w) {
            const dem_wall& x = h->walls[w];
            if (x.type == DEM_WALL_TRIANGLE) continue;
            bool still = x.velocity[0] == 0.0 && x.velocity[1] == 0.0 && x.velocity[2] == 0.0;
            const V3 om = v3(x.angular_velocity[0], x.angular_velocity[1], x.angular_velocity[2]);
            if (still && len2(om) != 0.0) {
                // a turn about the normal (infinite) or the axis (axisymmetric)
                // through the wall's position maps the wall onto itself
                const V3 ax = quat_axis(Q4{x.orientation[0], x.orientation[1], x.orientation[2], x.orientation[3]});
                still = (x.type == DEM_WALL_INFINITE || x.type == DEM_WALL_AXISYMMETRIC) &&
                        len2(cross(om, ax)) <= 1e-24 * len2(om) * len2(ax);
            }
            if (still) I.wall_still_mask |= 1u << (w - wbegin[in]);
        }
        for (int k = 0; k < 3; ++k) {
            I.tri_lo[k] = DBL_MAX;
            I.tri_hi[k] = -DBL_MAX;
        }
        for (int w = wbegin[in]; w < wend[in]; ++w) {
            const dem_wall& x = h->walls[w];
            if (x.type != DEM_WALL_TRIANGLE) continue;
            I.tri_mask |= 1u << (w - wbegin[in]);
            for (int k = 0; k < 3; ++k) {
                I.tri_static = I.tri_static && x.velocity[k] == 0.0 && x.angular_velocity[k] == 0.0;
                I.tri_lo[k] = std::min(I.tri_lo[k], h->wgeom[w].tlo[k]);
                I.tri_hi[k] = std::max(I.tri_hi[k], h->wgeom[w].thi[k]);
            }
        }
        fill_deletions(h, I, in);
        std::vector<int> lv_multi;
        std::vector<int>& lv = fast ? h->level_buf : lv_multi;
        const double* rad = fast ? p->radius : radii[in].data();
        const size_t nrad = fast ? (size_t)n : radii[in].size();
        setup_instance_grid(D, rad, nrad, skin, dmax, psd_lo[in], psd_hi[in], I, lv, cell_base,
                            levels_here ? &pre : nullptr);
        if (!fast)
            for (size_t k = 0; k < members[in].size(); ++k) level[members[in][k]] = lv[k];
        for (int r : free_rows[in]) level[r] = -1; // k_pack parks it dormant
        // a periodic dimension must be longer than twice the largest reach
        double rm = 0.0;
        if (nrad > 0 || has_ins[in])
            for (int l = 0; l < I.n_levels; ++l) rm = std::max(rm, I.level_rmax[l]);
        rmax_all = std::max(rmax_all, rm);
        for (int k = 0; k < 3; ++k)
            if (((D.periodic_mask >> k) & 1u) && I.per_L[k] <= 2.0 * (2.0 * rm + dmax + skin))
                return fail(h, DEM_ERR_BAD_INPUT, "periodic box too small for the particle size");
    }
    const long long ncells = cell_base + 1; // + the graveyard of deleted particles
    // ---- neighbour capacity
    int cap = h->cfg.max_neighbors;
    if (cap <= 0) {
        // auto: 48 for monodisperse-like packings, more when radii spread
        const double ratio = (n > 0) ? rmax_all / rmin_all : 1.0;
        cap = ratio < 1.5 ? 48 : (ratio < 2.5 ? 96 : 128);
    }
    cap = ((cap + 31) / 32) * 32;
    if (cap > 128) return fail(h, DEM_ERR_BAD_INPUT, "max_neighbors above 128 is not supported");

    // ---- contact capacity: items of one evaluation, and the springs of the
    // contacts (one record per item, two pools). Auto: at most min(cap, 16)
    // pairs owned per particle plus 4 walls; dem_config.max_contacts sets the
    // mean per particle instead (a dense packing has 2 to 4 owned contacts
    // per particle). Exceeding it is DEM_ERR_CAPACITY.
    if (h->cfg.max_contacts < 0) return fail(h, DEM_ERR_BAD_INPUT, "max_contacts must be >= 0");
    const long long item_cap =
        std::min<long long>(2000000000ll, h->cfg.max_contacts > 0
                                              ? (long long)n * h->cfg.max_contacts + 1024
                                              : (long long)n * std::min(cap, 16) + (long long)n * std::min(wmax, 4) + 1024);
    // ---- (re)allocate: a re-upload with the same sizes keeps the device arrays
    // and the captured graphs (their kernel arguments stay valid)
    const unsigned record_capacity = (unsigned)std::min<long long>(
        item_cap, std::min<long long>(2000000000ll, 8 * n + 1024 + (long long)n * std::min(wmax, 4)));
    int n_ins_inst = 0;
    for (int in = 0; in < ninst; ++in) n_ins_inst += has_ins[in];
    long long any_tri = 0;
    for (const auto& w : h->walls) any_tri = any_tri || w.type == DEM_WALL_TRIANGLE;
    const std::vector<long long> layout = {n, cap, wmax, ncells, (long long)h->inst.size(), (long long)h->species.size(),
                                           (long long)h->walls.size(), (long long)record_capacity, h->ncomp, any_tri,
                                           item_cap, (long long)h->ins.size(), (long long)n_ins_inst,
                                           (long long)h->fills.size()};
    const bool reuse = !h->layout.empty() && h->layout == layout;
    if (!reuse) free_particle_arrays(h);
    const DevPtrs kept = h->d;
    h->d = DevPtrs{};
    DevPtrs& d = h->d;
    d.n = (int)n;
    d.ncap = (int)std::max<long long>(32, ((n + 31) / 32) * 32);
    d.cap = cap;
    d.nwords = cap / 32;
    d.ncomp = h->ncomp;
    d.wmax = wmax;
    d.ncells = (int)ncells;
    d.rotation = h->cfg.rotation;
    d.single_instance = ninst == 1;
    d.n_instances = ninst;
    d.n_species_table = (int)h->species.size();
    d.zero_idist = 1;
    for (const auto& sp : h->species) d.zero_idist = d.zero_idist && sp.interaction_distance == 0.0;
    d.has_tri = 0;
    for (const auto& w : h->walls) d.has_tri = d.has_tri || w.type == DEM_WALL_TRIANGLE;
    d.dt = h->cfg.time_step;
    d.drag = h->cfg.background_drag;
    const size_t NC = d.ncap;
    int rc;
    if (reuse) {
        // graphs hold the kernel arguments by value: keep them only if nothing changed
        const bool same = d.n == kept.n && d.ncap == kept.ncap && d.cap == kept.cap && d.nwords == kept.nwords &&
                          d.ncomp == kept.ncomp && d.wmax == kept.wmax && d.ncells == kept.ncells &&
                          d.rotation == kept.rotation && d.single_instance == kept.single_instance &&
                          d.n_species_table == kept.n_species_table && d.zero_idist == kept.zero_idist &&
                          d.dt == kept.dt && d.drag == kept.drag && d.has_tri == kept.has_tri;
        if (!same) free_graphs(h);
        for (int b = 0; b < 2; ++b) {
            d.pr[b] = kept.pr[b]; d.vm[b] = kept.vm[b]; d.wi[b] = kept.wi[b]; d.qo[b] = kept.qo[b];
            d.info[b] = kept.info[b]; d.caller[b] = kept.caller[b]; d.nbr[b] = kept.nbr[b]; d.cnt[b] = kept.cnt[b];
            d.own[b] = kept.own[b];
            d.wcand[b] = kept.wcand[b];
            d.pool[b] = kept.pool[b]; d.hidx[b] = kept.hidx[b];
            d.act[b] = kept.act[b]; d.whist[b] = kept.whist[b]; d.wact[b] = kept.wact[b];
        }
        d.force = kept.force; d.torque = kept.torque; d.key = kept.key; d.perm = kept.perm; d.newidx = kept.newidx;
        d.cell_count = kept.cell_count; d.cell_start = kept.cell_start; d.cell_cursor = kept.cell_cursor;
        d.block_sums = kept.block_sums; d.rb_barrier = kept.rb_barrier; d.inst = kept.inst; d.species = kept.species; d.walls = kept.walls;
        d.wgeom = kept.wgeom; d.n_walls = kept.n_walls; d.ctl = kept.ctl; d.records = kept.records;
        d.n_instances = kept.n_instances;
        d.pf = kept.pf; d.rows = kept.rows; d.row_slot = kept.row_slot;
        d.rev = kept.rev; d.slot = kept.slot; d.slotw = kept.slotw; d.items = kept.items; d.shares = kept.shares;
        d.item_cap = kept.item_cap;
        d.tri_list = kept.tri_list;
        d.slott = kept.slott;
        d.tri_first = kept.tri_first;
        d.tri_first_n = kept.tri_first_n;
        for (int b = 0; b < 2; ++b) { // no history carries over from the previous simulation
            CU(cudaMemsetAsync(d.cnt[b], 0, NC * sizeof(int), h->stream));
            CU(cudaMemsetAsync(d.act[b], 0, (size_t)d.nwords * NC * sizeof(unsigned), h->stream));
            CU(cudaMemsetAsync(d.wact[b], 0, NC * sizeof(unsigned), h->stream));
        }
    } else {
    for (int b = 0; b < 2; ++b) {
        if ((rc = dalloc(h, &d.pr[b], NC))) return rc;
        if ((rc = dalloc(h, &d.vm[b], NC))) return rc;
        if ((rc = dalloc(h, &d.wi[b], NC))) return rc;
        if ((rc = dalloc(h, &d.qo[b], NC))) return rc;
        if ((rc = dalloc(h, &d.info[b], NC))) return rc;
        if ((rc = dalloc(h, &d.caller[b], NC))) return rc;
        if ((rc = dalloc(h, &d.nbr[b], (size_t)cap * NC))) return rc;
        if ((rc = dalloc(h, &d.cnt[b], NC))) return rc;
        if ((rc = dalloc(h, &d.own[b], (size_t)d.nwords * NC))) return rc;
        if ((rc = dalloc(h, &d.wcand[b], NC))) return rc;
        if ((rc = dalloc(h, &d.pool[b], (size_t)hist_stride(d.ncomp) * item_cap))) return rc;
        if ((rc = dalloc(h, &d.hidx[b], (size_t)cap * NC))) return rc;
        if ((rc = dalloc(h, &d.act[b], (size_t)d.nwords * NC))) return rc;
        if ((rc = dalloc(h, &d.whist[b], (size_t)hist_stride(d.ncomp) * wmax * NC))) return rc;
        if ((rc = dalloc(h, &d.wact[b], NC))) return rc;
    }
    if ((rc = dalloc(h, &d.rev, (size_t)cap * NC))) return rc;
    if ((rc = dalloc(h, &d.rows, (size_t)cap * NC))) return rc;
    if ((rc = dalloc(h, &d.pf, NC))) return rc;
    if (any_free) {
        if ((rc = dalloc(h, &d.row_slot, NC))) return rc;
        if ((rc = dalloc(h, &h->d_ins_inst, (size_t)n_ins_inst))) return rc;
        if ((rc = dalloc(h, &h->d_ins_bnd, h->ins.size()))) return rc;
        if ((rc = dalloc(h, &h->d_ins_rows, NC))) return rc;
        if ((rc = dalloc(h, &h->d_ovf, (size_t)ncells + 1 + 2 * NC))) return rc;
    }
    if ((rc = dalloc(h, &d.slot, (size_t)cap * NC))) return rc;
    if ((rc = dalloc(h, &d.slotw, (size_t)wmax * NC))) return rc;
    d.item_cap = (int)item_cap;
    if ((rc = dalloc(h, &d.items, (size_t)d.item_cap))) return rc;
    if ((rc = dalloc(h, &d.shares, (size_t)d.item_cap * SHARE))) return rc;
    if ((rc = dalloc(h, &d.tri_list, NC))) return rc;
    if ((rc = dalloc(h, &d.slott, NC))) return rc;
    if ((rc = dalloc(h, &d.tri_first_n, NC))) return rc;
    if ((rc = dalloc(h, &d.tri_first, any_tri ? NC * DEM_MAX_TRIANGLE_CONTACTS * TRI_REC : 1))) return rc;
    if ((rc = dalloc(h, &d.force, 3 * NC))) return rc;
    if ((rc = dalloc(h, &d.torque, 3 * NC))) return rc;
    if ((rc = dalloc(h, &d.key, NC))) return rc;
    if ((rc = dalloc(h, &d.perm, NC))) return rc;
    if ((rc = dalloc(h, &d.newidx, NC))) return rc;
    if ((rc = dalloc(h, &d.cell_count, (size_t)ncells + 1))) return rc;
    if ((rc = dalloc(h, &d.cell_start, (size_t)ncells + 1))) return rc;
    if ((rc = dalloc(h, &d.cell_cursor, (size_t)ncells + 1))) return rc;
    if ((rc = dalloc(h, &d.block_sums, (size_t)h->rb_grid + 1))) return rc;
    if ((rc = dalloc(h, &d.rb_barrier, 1))) return rc;
    if ((rc = dalloc(h, &h->d_inst, h->inst.size()))) return rc;
    if ((rc = dalloc(h, &h->d_species, h->species.size()))) return rc;
    if ((rc = dalloc(h, &h->d_walls, std::max<size_t>(1, h->walls.size())))) return rc;
    if ((rc = dalloc(h, &h->d_wgeom, std::max<size_t>(1, h->wgeom.size())))) return rc;
    if ((rc = dalloc(h, &h->d_ctl, 1))) return rc;
    h->record_capacity = record_capacity;
    if ((rc = dalloc(h, &h->d_records, h->record_capacity))) return rc;
    if ((rc = dalloc(h, &h->d_stage, 18 * NC))) return rc;
    d.inst = h->d_inst;
    d.species = h->d_species;
    d.walls = h->d_walls;
    d.wgeom = h->d_wgeom;
    d.n_walls = (int)h->walls.size();
    d.ctl = h->d_ctl;
    d.records = h->d_records;
    if ((rc = dalloc(h, &h->d_batch, h->inst.size() * (RED_SLOTS + 3)))) return rc;
    h->layout = layout;
    }

    // ---- the caller's arrays go to the device staging area as they are; k_pack
    // builds the state records there
    const StagePtrs st = stage_ptrs(h->d_stage, NC);
    auto put = [&](void* dst, const void* src, size_t bytes) -> int {
        if (src && bytes) CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
        return DEM_OK;
    };
    const size_t dn = (size_t)n * sizeof(double), in4 = (size_t)n * sizeof(int);
    if ((rc = put(st.pos, p->position, 3 * dn)) || (rc = put(st.vel, p->velocity, 3 * dn)) ||
        (rc = put(st.ang, p->angular_velocity, 3 * dn)) || (rc = put(st.ori, p->orientation, 4 * dn)) ||
        (rc = put(st.rad, p->radius, dn)) || (rc = put(st.im, p->inv_mass, dn)) ||
        (rc = put(st.ii, p->inv_inertia, dn)) || (rc = put(st.sp, p->species, in4)) || (rc = put(st.id, p->id, in4)) ||
        (rc = put(st.inst, p->instance, in4)) || (!levels_here && (rc = put(st.lvl, level.data(), in4))))
        return rc;
    CU(cudaMemcpyAsync(h->d_inst, h->inst.data(), h->inst.size() * sizeof(InstanceDev), cudaMemcpyHostToDevice, h->stream));
    Control c{};
    c.cur = 0;
    c.lbuf = 0;
    c.skin = skin;
    c.force_rebuild = 1;
    c.record = 1;
    c.record_capacity = h->record_capacity;
    CU(cudaMemcpyAsync(h->d_ctl, &c, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    if (n > 0)
        k_pack<<<grid_for(n, 256), 256, 0, h->stream>>>(d, st, p->angular_velocity != nullptr,
                                                        p->orientation != nullptr, p->inv_inertia != nullptr,
                                                        p->instance != nullptr,
                                                        one ? h->inst_desc[0].n_species : INT_MAX, one ? 1 : 0,
                                                        levels_here ? 1 : 0);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h->d_species, h->species.data(), h->species.size() * sizeof(dem_species_pair),
                       cudaMemcpyHostToDevice, h->stream));
    if (!h->walls.empty()) {
        CU(cudaMemcpyAsync(h->d_walls, h->walls.data(), h->walls.size() * sizeof(dem_wall), cudaMemcpyHostToDevice,
                           h->stream));
        CU(cudaMemcpyAsync(h->d_wgeom, h->wgeom.data(), h->wgeom.size() * sizeof(WallGeom), cudaMemcpyHostToDevice,
                           h->stream));
    }
    CU(cudaMemsetAsync(d.tri_first_n, 0, NC * sizeof(int), h->stream)); // filled by the initial evaluation
    // insertion boundaries: generators seeded, counters zero, free rows listed
    // per instance (InsertionBoundary's state at the start of a run)
    std::vector<InsInstanceDev> ins_inst;
    std::vector<InsBoundaryDev> ins_bnd;
    std::vector<int> ins_rows;
    h->ins_order.clear();
    for (int in = 0; in < ninst && any_free; ++in) {
        if (!has_ins[in]) continue;
        InsInstanceDev S{};
        lfg_seed(h->ins_seeds[in], S.rng);
        S.time = 0.0;
        for (double r : radii[in]) S.grid_rmax = std::max(S.grid_rmax, r);
        S.instance = in;
        S.first = (int)ins_bnd.size();
        for (size_t k = 0; k < h->ins.size(); ++k) {
            if (h->ins[k].instance != in) continue;
            InsBoundaryDev B{};
            B.b = h->ins[k];
            lfg_seed(B.b.psd_seed, B.psd);
            ins_bnd.push_back(B);
            h->ins_order.push_back((int)k);
        }
        S.count = (int)ins_bnd.size() - S.first;
        S.rows_begin = (int)ins_rows.size();
        ins_rows.insert(ins_rows.end(), free_rows[in].begin(), free_rows[in].end());
        S.rows_end = (int)ins_rows.size();
        S.next_row = S.rows_begin;
        S.filed_from = S.rows_begin;
        ins_inst.push_back(S);
    }
    h->n_ins_inst = (int)ins_inst.size();
    h->n_ins_launch = h->ins.empty() ? 0 : h->n_ins_inst;
    if (h->n_ins_inst > 0) {
        CU(cudaMemsetAsync(h->d_ovf, 0xff, ((size_t)d.ncells + 1) * sizeof(int), h->stream)); // lists empty
        CU(cudaMemcpyAsync(h->d_ins_inst, ins_inst.data(), ins_inst.size() * sizeof(InsInstanceDev),
                           cudaMemcpyHostToDevice, h->stream));
        CU(cudaMemcpyAsync(h->d_ins_bnd, ins_bnd.data(), ins_bnd.size() * sizeof(InsBoundaryDev),
                           cudaMemcpyHostToDevice, h->stream));
        if (!ins_rows.empty())
            CU(cudaMemcpyAsync(h->d_ins_rows, ins_rows.data(), ins_rows.size() * sizeof(int), cudaMemcpyHostToDevice,
                               h->stream));
    }
    // chute fills (Chute::addFlowParticlesCompactly), in the order given
    h->fill_results.assign(h->fills.size(), FillDev{});
    for (size_t k = 0; k < h->fills.size(); ++k) {
        const dem_chute_fill& f = h->fills[k];
        const int in = f.instance;
        const InstanceDev& I = h->inst[in];
        FillDev F{};
        F.f = f;
        F.height = f.inflow_height;
        for (size_t j = 0; j < ins_inst.size(); ++j)
            if (ins_inst[j].instance == in) F.instance_slot = (int)j;
        // N = ParticleHandler::getNumberOfObjects() + length width height / r_in^3 / 8 (Chute.cc:1086-1087)
        const unsigned n_objects = (unsigned)(fast ? n : (long long)radii[in].size());
        const double r_in = 0.5 * (f.min_radius + f.max_radius);
        const unsigned N = (unsigned)(n_objects + f.x_max * f.y_max * f.inflow_height / (r_in * r_in * r_in) / 8);
        F.target = N > n_objects ? (long long)(N - n_objects) : 0;
        F.tries_left = 100 * F.target + 10000000ll;
        // a linked-list grid of the instance, cells at least one reach wide
        double rmax = 0.0;
        for (int l = 0; l < I.n_levels; ++l) rmax = std::max(rmax, I.level_rmax[l]);
        double cs = 2.0 * rmax + I.max_interaction_distance;
        FillGrid g{};
        const auto& D = h->inst_desc[in];
        for (int pass = 0; pass < 64; ++pass) {
            long long cells = 1;
            for (int a = 0; a < 3; ++a) {
                g.origin[a] = I.origin[a];
                if ((D.periodic_mask >> a) & 1u) {
                    const double L = I.per_L[a];
                    g.dims[a] = std::max(1, (int)std::floor(L / cs));
                    g.inv[a] = (double)g.dims[a] / L;
                } else {
                    const double ext = D.domain_max[a] - D.domain_min[a];
                    g.dims[a] = (int)std::min(1024.0, std::max(1.0, std::ceil(ext / cs)));
                    g.inv[a] = 1.0 / cs;
                }
                cells *= g.dims[a];
            }
            if (cells <= (1ll << 24)) break;
            cs *= 2.0;
        }
        const size_t ncells = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
        FillDev* dF = nullptr;
        CU(cudaMalloc(&g.head, ncells * sizeof(int)));
        CU(cudaMalloc(&g.next, NC * sizeof(int)));
        CU(cudaMalloc(&dF, sizeof(FillDev)));
        CU(cudaMemsetAsync(g.head, 0xff, ncells * sizeof(int), h->stream)); // -1: empty
        CU(cudaMemcpyAsync(dF, &F, sizeof(FillDev), cudaMemcpyHostToDevice, h->stream));
        if (F.target > 0) {
            k_fill_grid<<<grid_for(n, 256), 256, 0, h->stream>>>(d, g, in);
            k_fill<<<1, INS_THREADS, 0, h->stream>>>(d, ins_ptrs(h), dF, g);
        }
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(&h->fill_results[k], dF, sizeof(FillDev), cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        cudaFree(g.head);
        cudaFree(g.next);
        cudaFree(dF);
        if (h->fill_results[k].status == 1)
            return fail(h, DEM_ERR_CAPACITY, "chute fill: no free row left (upload more rows of radius 0)");
        if (h->fill_results[k].status == 2)
            return fail(h, DEM_ERR_CAPACITY, "chute fill: gave up before placing every particle");
    }
    unsigned int status = 0;
    CU(cudaMemcpyAsync(&status, &h->d_ctl->status, sizeof(status), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (status & (1u << DEM_ERR_BAD_INPUT)) { // k_pack found bad input: name it
        h->uploaded = false;
        const int rc1 = validate();
        return rc1 ? rc1 : fail(h, DEM_ERR_BAD_INPUT, "particle arrays out of range");
    }
    h->uploaded = true;
    h->initial_pending = true;
    h->records_valid = false;
    h->steps_total = 0;
    return DEM_OK;
}

// Runs the forced rebuild that a pending initial evaluation needs (without
// the force evaluation itself); used by dem_upload_contacts.
static int ensure_lists(Handle* h)
{
    Control c;
    int rc = read_control(h, &c);
    if (rc) return rc;
    if (!c.force_rebuild) return DEM_OK;
    c.rebuild = 1;
    c.force_rebuild = 0;
    CU(cudaMemcpyAsync(h->d_ctl, &c, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    CU(launch_rebuild(h, h->stream));
    return read_control(h, &c);
}

int dem_upload_contacts(dem_handle* hh, const dem_contacts_soa* cs)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !cs || cs->n < 0) return fail(h, DEM_ERR_BAD_INPUT, "dem_upload_contacts: bad arguments");
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "upload particles first");
    if (!h->initial_pending) return fail(h, DEM_ERR_STATE, "contacts can only be injected before the first step");
    int rc = ensure_lists(h);
    if (rc) return rc;
    Control c;
    if ((rc = read_control(h, &c))) return rc;
    DevPtrs& d = h->d;
    const int n = d.n, cur = c.cur, l = c.lbuf;
    const size_t NC = d.ncap;
    std::vector<int4> info(n);
    std::vector<double4> pr(n);
    std::vector<int> cnt(n), nbr((size_t)d.cap * NC);
    std::vector<unsigned> act((size_t)d.nwords * NC), wact(NC);
    std::vector<int> hidx((size_t)d.cap * NC, 0);
    std::vector<double> pool, whist((size_t)hist_stride(d.ncomp) * d.wmax * NC);
    CU(cudaMemcpyAsync(info.data(), d.info[cur], n * sizeof(int4), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(pr.data(), d.pr[cur], n * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(cnt.data(), d.cnt[l], n * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(nbr.data(), d.nbr[l], nbr.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(act.data(), d.act[cur], act.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(wact.data(), d.wact[cur], wact.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(whist.data(), d.whist[cur], whist.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(hidx.data(), d.hidx[cur], hidx.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    // springs injected by an earlier call stay where they are in the pool
    const int stride = hist_stride(d.ncomp);
    long long used = 0;
    for (int s = 0; s < n; ++s)
        for (int k = 0; k < std::min(cnt[s], d.cap); ++k)
            if ((act[(size_t)(k >> 5) * NC + s] >> (k & 31)) & 1u)
                used = std::max<long long>(used, (long long)hidx[nbr_at(d.ncap, s, k)] + 1);
    pool.resize((size_t)used * stride);
    if (used) {
        CU(cudaMemcpyAsync(pool.data(), d.pool[c.pcur], pool.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    // id -> sorted slot
    std::vector<std::pair<int, int>> ids(n);
    for (int s = 0; s < n; ++s) ids[s] = {info[s].x, s};
    std::sort(ids.begin(), ids.end());
    auto slot_of = [&](int id) -> int {
        auto it = std::lower_bound(ids.begin(), ids.end(), std::make_pair(id, -1));
        return (it != ids.end() && it->first == id) ? it->second : -1;
    };
    // an entry with a new spring gets the next record of the pool
    auto set_entry = [&](int s, int t, const double* spr, double sign) -> bool {
        for (int k = 0; k < cnt[s]; ++k) {
            if (nbr[nbr_at(d.ncap, s, k)] != t) continue;
            const size_t e = nbr_at(d.ncap, s, k);
            if (!((act[(size_t)(k >> 5) * NC + s] >> (k & 31)) & 1u)) {
                hidx[e] = (int)(pool.size() / stride);
                pool.resize(pool.size() + stride, 0.0);
            }
            for (int comp = 0; comp < d.ncomp; ++comp) pool[(size_t)hidx[e] * stride + comp] = sign * spr[comp];
            act[(size_t)(k >> 5) * NC + s] |= 1u << (k & 31);
            return true;
        }
        return false;
    };
    for (long long r = 0; r < cs->n; ++r) {
        const double* spr = cs->springs ? cs->springs + 9 * r : nullptr;
        double zero[9] = {0};
        if (!spr) spr = zero;
        const int sp = slot_of(cs->id_p[r]);
        if (sp < 0) return fail(h, DEM_ERR_BAD_INPUT, "contact refers to an unknown particle id");
        if (cs->is_wall && cs->is_wall[r]) {
            const int in = info[sp].z;
            const int wc = cs->id_i[r];
            if (wc < 0 || wc >= (int)h->walls.size()) return fail(h, DEM_ERR_BAD_INPUT, "contact refers to an unknown wall");
            const int w = h->wall_grouped[wc] - h->inst[in].wall_begin;
            if (w < 0 || w >= h->inst[in].wall_end - h->inst[in].wall_begin)
                return fail(h, DEM_ERR_BAD_INPUT, "contact refers to a wall outside the particle's instance");
            for (int comp = 0; comp < d.ncomp; ++comp) whist[whist_at(d.ncap, d.ncomp, sp, w) + comp] = spr[comp];
            wact[sp] |= 1u << w;
            continue;
        }
        const int si = slot_of(cs->id_i[r]);
        if (si < 0) return fail(h, DEM_ERR_BAD_INPUT, "contact refers to an unknown particle id");
        const bool per = cs->periodic && cs->periodic[r];
        // P's own entry carries the spring; I's entry carries the same spring for
        // a direct pair and the reversed one for a periodic pair
        // (BaseInteraction::copySwitchPointer / reverseHistory).
        if (!set_entry(sp, si, spr, 1.0) || !set_entry(si, sp, spr, per ? -1.0 : 1.0))
            return fail(h, DEM_ERR_BAD_INPUT, "injected contact is not within the neighbour list");
    }
    if (pool.size() / stride > (size_t)d.item_cap)
        return fail(h, DEM_ERR_CAPACITY, "more contact springs than the contact capacity (raise dem_config.max_contacts)");
    CU(cudaMemcpyAsync(d.act[cur], act.data(), act.size() * sizeof(unsigned), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(d.wact[cur], wact.data(), wact.size() * sizeof(unsigned), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(d.hidx[cur], hidx.data(), hidx.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    if (!pool.empty())
        CU(cudaMemcpyAsync(d.pool[c.pcur], pool.data(), pool.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(d.whist[cur], whist.data(), whist.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}

int dem_step(dem_handle* hh, int nsteps)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (nsteps < 0) return fail(h, DEM_ERR_BAD_INPUT, "nsteps must be >= 0");
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "dem_upload_particles must come before dem_step");
    CU(cudaSetDevice(h->device));
    DevPtrs& d = h->d;
    long long launches = 0;
    Control c0;
    int rc = read_control(h, &c0);
    if (rc) return rc;
    const long long rebuilds0 = c0.n_rebuilds;
    const bool evaluates = d.n > 0 && (h->initial_pending || nsteps > 0);
    c0.status = 0;
    if (evaluates) c0.n_records = 0;
    if (h->initial_pending && d.n > 0) {
        // DPMBase::initialiseSolve: first force evaluation at the uploaded state.
        // If dem_upload_contacts already built the lists, they are kept.
        c0.rebuild = c0.force_rebuild ? 1 : 0;
        c0.force_rebuild = 0;
        c0.pending_flip = 1;
    }
    CU(cudaMemcpyAsync(h->d_ctl, &c0, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    CU(cudaEventRecord(h->ev0, h->stream));
    if (d.n > 0) {
        if (h->initial_pending) {
            if (c0.rebuild) {
                CU(launch_rebuild(h, h->stream));
                launches += REBUILD_LAUNCHES;
            }
            launch_force(h, h->stream, 0);
            k_flip<<<1, 32, 0, h->stream>>>(h->d_ctl);
            launches += force_launches(h) + 1;
            CU(cudaGetLastError());
            h->initial_pending = false;
        }
        if (nsteps > 0) {
            long long sl = nsteps;
            CU(cudaMemcpyAsync(&h->d_ctl->steps_left, &sl, sizeof(long long), cudaMemcpyHostToDevice, h->stream));
            k_kick_drift<<<grid_for(d.n, 256), 256, 0, h->stream>>>(d);
            launches += 1;
            if (h->cfg.use_graphs) {
                if (!h->graph1) {
                    if ((rc = build_graph(h, 1, false, &h->graph1))) return rc;
                    if ((rc = build_graph(h, GRAPH_STEPS, false, &h->graphK))) return rc;
                    if ((rc = build_graph(h, 1, true, &h->graphF))) return rc;
                }
                int left = nsteps - 1; // the last step: graphF
                while (left >= GRAPH_STEPS) {
                    CU(cudaGraphLaunch(h->graphK, h->stream));
                    left -= GRAPH_STEPS;
                }
                while (left-- > 0) CU(cudaGraphLaunch(h->graph1, h->stream));
                CU(cudaGraphLaunch(h->graphF, h->stream));
                launches += (1ll + REBUILD_LAUNCHES + force_launches(h) + (h->n_ins_launch > 0)) * nsteps;
            } else {
                for (int k = 0; k < nsteps; ++k) {
                    k_control<<<1, CONTROL_THREADS, 0, h->stream>>>(h->d_ctl, d.walls, h->d_wgeom, d.n_walls, d.dt);
                    launch_insert(h, h->stream);
                    CU(launch_rebuild(h, h->stream));
                    launch_force(h, h->stream, 1, k == nsteps - 1);
                }
                CU(cudaGetLastError());
                launches += (1ll + force_launches(h) + REBUILD_LAUNCHES + (h->n_ins_launch > 0)) * nsteps;
            }
            k_flip<<<1, 32, 0, h->stream>>>(h->d_ctl);
            launches += 1;
        }
    }
    CU(cudaEventRecord(h->ev1, h->stream));
    Control c;
    if ((rc = read_control(h, &c))) return rc;
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->last_ms = ms;
    const long long rb = c.n_rebuilds - rebuilds0;
    h->last_rebuilds = rb;
    h->last_launches = launches;
    h->steps_total += nsteps;
    if (evaluates) {
        h->n_records = c.n_records;
        h->records_valid = c.n_records <= c.record_capacity;
        if (!h->records_valid) {
            // grow the record buffer so that the next evaluation keeps every contact
            const unsigned need = (unsigned)std::min<unsigned long long>(2000000000ull, 2ull * c.n_records);
            void* p = nullptr;
            if (cudaMalloc(&p, (size_t)need * sizeof(ContactRecord)) == cudaSuccess) {
                h->allocs.push_back(p);
                h->alloc_bytes += (size_t)need * sizeof(ContactRecord);
                h->d_records = static_cast<ContactRecord*>(p);
                h->record_capacity = need;
                d.records = h->d_records;
                free_graphs(h); // the captured kernels hold the old pointer
                c.record_capacity = need;
                c.n_records = 0;
                CU(cudaMemcpyAsync(h->d_ctl, &c, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
                CU(cudaStreamSynchronize(h->stream));
            }
        }
    }
    return check_status(h, c);
}

int dem_download_particles(dem_handle* hh, dem_particles_soa* p)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !p) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_particles: bad arguments");
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "nothing uploaded");
    if (p->n != h->d.n) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_particles: n does not match the upload");
    CU(cudaSetDevice(h->device));
    Control c;
    int rc = read_control(h, &c);
    if (rc) return rc;
    const int n = h->d.n, b = c.cur;
    const StagePtrs st = stage_ptrs(h->d_stage, (size_t)h->d.ncap);
    if (n > 0) k_unpack<<<grid_for(n, 256), 256, 0, h->stream>>>(h->d, b, st);
    CU(cudaGetLastError());
    auto get = [&](void* dst, const void* src, size_t bytes) -> int {
        if (dst && bytes) CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
        return DEM_OK;
    };
    const size_t dn = (size_t)n * sizeof(double), in4 = (size_t)n * sizeof(int);
    if ((rc = get(p->position, st.pos, 3 * dn)) || (rc = get(p->velocity, st.vel, 3 * dn)) ||
        (rc = get(p->angular_velocity, st.ang, 3 * dn)) || (rc = get(p->orientation, st.ori, 4 * dn)) ||
        (rc = get(p->radius, st.rad, dn)) || (rc = get(p->inv_mass, st.im, dn)) ||
        (rc = get(p->inv_inertia, st.ii, dn)) || (rc = get(p->species, st.sp, in4)) || (rc = get(p->id, st.id, in4)) ||
        (rc = get(p->instance, st.inst, in4)))
        return rc;
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}

int dem_download_forces(dem_handle* hh, double* force, double* torque)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    CU(cudaSetDevice(h->device));
    Control c;
    int rc = read_control(h, &c);
    if (rc) return rc;
    const int n = h->d.n;
    std::vector<double> f(3 * (size_t)n), t(3 * (size_t)n);
    std::vector<int> caller(n);
    CU(cudaMemcpyAsync(f.data(), h->d.force, f.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(t.data(), h->d.torque, t.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(caller.data(), h->d.caller[c.cur], n * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (int s = 0; s < n; ++s) {
        const int i = caller[s];
        for (int k = 0; k < 3; ++k) {
            if (force) force[3 * i + k] = f[3 * (size_t)s + k];
            if (torque) torque[3 * i + k] = t[3 * (size_t)s + k];
        }
    }
    return DEM_OK;
}

int dem_download_walls(dem_handle* hh, dem_wall* walls, int n)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || n < 0 || (n > 0 && !walls)) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_walls: bad arguments");
    if (n != (int)h->walls.size()) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_walls: wrong wall count");
    if (n == 0) return DEM_OK;
    std::vector<dem_wall> w(h->walls);
    if (h->uploaded) {
        CU(cudaSetDevice(h->device));
        CU(cudaMemcpyAsync(w.data(), h->d_walls, n * sizeof(dem_wall), cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    for (int k = 0; k < n; ++k) walls[h->wall_caller[k]] = w[k];
    return DEM_OK;
}

// The contact records of the last evaluation in the order the contact
// downloads report them: particle pairs first, then wall contacts, each by
// (id of P, id of I or the caller's wall index).
static int sorted_records(Handle* h, std::vector<ContactRecord>& rec)
{
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    if (!h->records_valid)
        return fail(h, DEM_ERR_CAPACITY, "contact records of the last evaluation overflowed; the buffer has grown, "
                                         "the next dem_step records all contacts");
    CU(cudaSetDevice(h->device));
    const unsigned nr = h->n_records;
    rec.resize(nr);
    if (nr) CU(cudaMemcpyAsync(rec.data(), h->d_records, nr * sizeof(ContactRecord), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (auto& x : rec)
        if (x.is_wall) x.id_i = h->wall_caller[x.id_i]; // report the caller's wall index
    std::sort(rec.begin(), rec.end(), [](const ContactRecord& a, const ContactRecord& b) {
        if (a.is_wall != b.is_wall) return a.is_wall < b.is_wall;
        if (a.id_p != b.id_p) return a.id_p < b.id_p;
        return a.id_i < b.id_i;
    });
    return DEM_OK;
}

int dem_download_contact_geometry(dem_handle* hh, double* contact_point, double* normal, double* tangential_force,
                                  int64_t capacity, int64_t* count)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !count || capacity < 0) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_contact_geometry: bad arguments");
    std::vector<ContactRecord> rec;
    int rc = sorted_records(h, rec);
    if (rc) return rc;
    *count = (int64_t)rec.size();
    const int64_t m = std::min<int64_t>(capacity, (int64_t)rec.size());
    for (int64_t r = 0; r < m; ++r)
        for (int k = 0; k < 3; ++k) {
            if (contact_point) contact_point[3 * r + k] = rec[r].contact_point[k];
            if (normal) normal[3 * r + k] = rec[r].normal[k];
            if (tangential_force) tangential_force[3 * r + k] = rec[r].tangential[k];
        }
    return DEM_OK;
}

int dem_download_contacts(dem_handle* hh, dem_contacts_soa* cs, int64_t capacity, int64_t* count)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !count || capacity < 0) return fail(h, DEM_ERR_BAD_INPUT, "dem_download_contacts: bad arguments");
    std::vector<ContactRecord> rec;
    int rc = sorted_records(h, rec);
    if (rc) return rc;
    const unsigned nr = (unsigned)rec.size();
    *count = nr;
    if (!cs) return DEM_OK;
    const int64_t m = std::min<int64_t>(capacity, nr);
    for (int64_t r = 0; r < m; ++r) {
        const ContactRecord& x = rec[r];
        if (cs->id_p) cs->id_p[r] = x.id_p;
        if (cs->id_i) cs->id_i[r] = x.id_i;
        if (cs->is_wall) cs->is_wall[r] = x.is_wall;
        if (cs->periodic) cs->periodic[r] = x.periodic;
        if (cs->overlap) cs->overlap[r] = x.overlap;
        for (int k = 0; k < 3; ++k)
            if (cs->force) cs->force[3 * r + k] = x.force[k];
        for (int k = 0; k < 9; ++k)
            if (cs->springs) cs->springs[9 * r + k] = x.springs[k];
    }
    cs->n = m;
    return DEM_OK;
}

int dem_reduce(dem_handle* hh, int instance, dem_globals* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !out) return DEM_ERR_BAD_INPUT;
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "nothing uploaded");
    if (instance < 0 || instance >= (int)h->inst.size()) return fail(h, DEM_ERR_BAD_INPUT, "instance out of range");
    CU(cudaSetDevice(h->device));
    std::memset(out, 0, sizeof(*out));
    const int n = h->d.n;
    const unsigned nb = grid_for(n, 256);
    const unsigned nr = h->records_valid && !h->initial_pending ? h->n_records : 0;
    const unsigned nbr = grid_for(nr, 256);
    double* dpart = nullptr;
    const size_t slots = (size_t)nb * RED_SLOTS + (size_t)nbr * 3;
    CU(cudaMallocAsync((void**)&dpart, slots * sizeof(double), h->stream));
    k_reduce_particles<<<nb, 256, 0, h->stream>>>(h->d, instance, dpart);
    if (nr) k_reduce_records<<<nbr, 256, 0, h->stream>>>(h->d, instance, nr, dpart + (size_t)nb * RED_SLOTS);
    std::vector<double> part(slots);
    CU(cudaMemcpyAsync(part.data(), dpart, slots * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaFreeAsync(dpart, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    double acc[RED_SLOTS] = {0};
    for (unsigned b = 0; b < nb; ++b)
        for (int k = 0; k < RED_SLOTS; ++k) acc[k] += part[(size_t)b * RED_SLOTS + k];
    double racc[3] = {0, 0, 0};
    for (unsigned b = 0; b < (nr ? nbr : 0); ++b)
        for (int k = 0; k < 3; ++k) racc[k] += part[(size_t)nb * RED_SLOTS + (size_t)b * 3 + k];
    out->kinetic_energy = acc[0];
    out->rotational_energy = acc[1];
    out->gravitational_energy = acc[2];
    out->mass = acc[3];
    for (int k = 0; k < 3; ++k) {
        out->momentum[k] = acc[4 + k];
        out->centre_of_mass[k] = acc[3] > 0 ? acc[7 + k] / acc[3] : 0.0;
        out->angular_momentum[k] = acc[10 + k];
    }
    out->elastic_energy = racc[0];
    out->n_contacts = (int64_t)llround(racc[1]);
    out->n_wall_contacts = (int64_t)llround(racc[2]);
    out->time = h->steps_total * h->cfg.time_step;
    out->n_steps = h->steps_total;
    return DEM_OK;
}

int dem_reduce_batch(dem_handle* hh, int first, int count, dem_globals* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !out || count < 0) return DEM_ERR_BAD_INPUT;
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "nothing uploaded");
    if (h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    if (first < 0 || first + count > (int)h->inst.size()) return fail(h, DEM_ERR_BAD_INPUT, "instance range out of range");
    if (count == 0) return DEM_OK;
    CU(cudaSetDevice(h->device));
    const unsigned nr = h->records_valid ? h->n_records : 0;
    const size_t row = RED_SLOTS + 3;
    k_reduce_instances<<<count, 256, 0, h->stream>>>(h->d, first, h->d_batch);
    if (nr) k_reduce_records_instances<<<grid_for(nr, 256), 256, 0, h->stream>>>(h->d, first, count, nr, h->d_batch);
    CU(cudaGetLastError());
    std::vector<double> r((size_t)count * row);
    CU(cudaMemcpyAsync(r.data(), h->d_batch, r.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < count; ++k) {
        const double* a = r.data() + (size_t)k * row;
        dem_globals& g = out[k];
        std::memset(&g, 0, sizeof(g));
        g.kinetic_energy = a[0];
        g.rotational_energy = a[1];
        g.gravitational_energy = a[2];
        g.mass = a[3];
        for (int q = 0; q < 3; ++q) {
            g.momentum[q] = a[4 + q];
            g.centre_of_mass[q] = a[3] > 0 ? a[7 + q] / a[3] : 0.0;
            g.angular_momentum[q] = a[10 + q];
        }
        g.elastic_energy = a[RED_SLOTS];
        g.n_contacts = (int64_t)llround(a[RED_SLOTS + 1]);
        g.n_wall_contacts = (int64_t)llround(a[RED_SLOTS + 2]);
        g.time = h->steps_total * h->cfg.time_step;
        g.n_steps = h->steps_total;
    }
    return DEM_OK;
}

} // extern "C"

// ---- balances without device allocation ------------------------------------
// The partial sums of dem_reduce_noalloc live in this file-scope array, which
// every GPU that loads the library holds until the process exits. One block
// of 256 particles (or contact records) leaves one partial row, so the array
// bounds the sizes the entry point accepts.
namespace {
constexpr unsigned NOALLOC_MAX_BLOCKS = 8192;  // 2,097,152 particles / contact records
constexpr size_t NOALLOC_PART_ROWS = (size_t)NOALLOC_MAX_BLOCKS * RED_SLOTS;
constexpr size_t NOALLOC_REC_ROWS = (size_t)NOALLOC_MAX_BLOCKS * 3;
constexpr size_t NOALLOC_RESULT = NOALLOC_PART_ROWS + NOALLOC_REC_ROWS; // 16 result slots follow
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_scratch[NOALLOC_MAX_DEVICES] = {nullptr};
} // namespace

static __device__ __align__(256) double g_reduce_scratch[NOALLOC_RESULT + 16];

// Sums the per-block rows in block order, exactly as dem_reduce does on the host.
__global__ void k_reduce_finish(const double* part, unsigned nb, unsigned nbr, double* result)
{
    const int k = threadIdx.x;
    if (k < RED_SLOTS) {
        double a = 0.0;
        for (unsigned b = 0; b < nb; ++b) a += part[(size_t)b * RED_SLOTS + k];
        result[k] = a;
    } else if (k < RED_SLOTS + 3) {
        double a = 0.0;
        for (unsigned b = 0; b < nbr; ++b) a += part[NOALLOC_PART_ROWS + (size_t)b * 3 + (k - RED_SLOTS)];
        result[k] = a;
    }
}

extern "C" {

int dem_reduce_noalloc(dem_handle* hh, int instance, dem_globals* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !out) return DEM_ERR_BAD_INPUT;
    if (!h->uploaded) return fail(h, DEM_ERR_STATE, "nothing uploaded");
    if (instance < 0 || instance >= (int)h->inst.size()) return fail(h, DEM_ERR_BAD_INPUT, "instance out of range");
    if (h->device < 0 || h->device >= NOALLOC_MAX_DEVICES)
        return fail(h, DEM_ERR_BAD_INPUT, "dem_reduce_noalloc: device ordinal above 63");
    const int n = h->d.n;
    const unsigned nb = grid_for(n, 256);
    const unsigned nr = h->records_valid && !h->initial_pending ? h->n_records : 0;
    const unsigned nbr = grid_for(nr, 256);
    if (nb > NOALLOC_MAX_BLOCKS || nbr > NOALLOC_MAX_BLOCKS)
        return fail(h, DEM_ERR_CAPACITY,
                    "dem_reduce_noalloc: more than 2,097,152 particles or contact records (the size of its "
                    "static scratch array); use dem_reduce");
    CU(cudaSetDevice(h->device));
    double* scratch = nullptr;
    {
        // set-up, once per device with that device current: the host-side name
        // of a __device__ array is not a device address
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_scratch[h->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_reduce_scratch);
            if (e != cudaSuccess)
                return fail(h, DEM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_noalloc_scratch[h->device] = static_cast<double*>(p);
        }
        scratch = g_noalloc_scratch[h->device];
    }
    // every row the kernels write is overwritten before it is read: nothing to clear
    k_reduce_particles<<<nb, 256, 0, h->stream>>>(h->d, instance, scratch);
    if (nr) k_reduce_records<<<nbr, 256, 0, h->stream>>>(h->d, instance, nr, scratch + NOALLOC_PART_ROWS);
    k_reduce_finish<<<1, 32, 0, h->stream>>>(scratch, nb, nr ? nbr : 0, scratch + NOALLOC_RESULT);
    CU(cudaGetLastError());
    double res[16];
    CU(cudaMemcpyAsync(res, scratch + NOALLOC_RESULT, sizeof(res), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    std::memset(out, 0, sizeof(*out));
    out->kinetic_energy = res[0];
    out->rotational_energy = res[1];
    out->gravitational_energy = res[2];
    out->mass = res[3];
    for (int k = 0; k < 3; ++k) {
        out->momentum[k] = res[4 + k];
        out->centre_of_mass[k] = res[3] > 0 ? res[7 + k] / res[3] : 0.0;
        out->angular_momentum[k] = res[10 + k];
    }
    out->elastic_energy = res[RED_SLOTS];
    out->n_contacts = (int64_t)llround(res[RED_SLOTS + 1]);
    out->n_wall_contacts = (int64_t)llround(res[RED_SLOTS + 2]);
    out->time = h->steps_total * h->cfg.time_step;
    out->n_steps = h->steps_total;
    return DEM_OK;
}

int dem_last_step_stats(dem_handle* hh, double* ms, int64_t* kernel_launches, int64_t* rebuilds)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (ms) *ms = h->last_ms;
    if (kernel_launches) *kernel_launches = h->last_launches;
    if (rebuilds) *rebuilds = h->last_rebuilds;
    return DEM_OK;
}

int dem_get_info(dem_handle* hh, int64_t* n_particles, int64_t* max_neighbors, int64_t* n_cells)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (n_particles) *n_particles = h->d.n;
    if (max_neighbors) *max_neighbors = h->d.cap;
    if (n_cells) *n_cells = h->d.ncells;
    return DEM_OK;
}

int dem_get_memory(dem_handle* hh, int64_t* device_bytes, int64_t* contact_capacity)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (device_bytes) *device_bytes = (int64_t)h->alloc_bytes;
    if (contact_capacity) *contact_capacity = h->d.item_cap;
    return DEM_OK;
}

int dem_get_counts(dem_handle* hh, int64_t* list_entries, int64_t* contacts, int64_t* wall_contacts)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return DEM_ERR_BAD_INPUT;
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    CU(cudaSetDevice(h->device));
    Control c;
    int rc = read_control(h, &c);
    if (rc) return rc;
    std::vector<int> cnt(h->d.n);
    CU(cudaMemcpyAsync(cnt.data(), h->d.cnt[c.lbuf], cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    std::vector<ContactRecord> rec(h->records_valid ? h->n_records : 0);
    if (!rec.empty())
        CU(cudaMemcpyAsync(rec.data(), h->d_records, rec.size() * sizeof(ContactRecord), cudaMemcpyDeviceToHost,
                           h->stream));
    CU(cudaStreamSynchronize(h->stream));
    long long e = 0, pc = 0, wc = 0;
    for (int v : cnt) e += v;
    for (const auto& r : rec) (r.is_wall ? wc : pc) += 1;
    if (list_entries) *list_entries = e;
    if (contacts) *contacts = pc;
    if (wall_contacts) *wall_contacts = wc;
    return DEM_OK;
}

int dem_time_force_kernel(dem_handle* hh, int reps, double* ms_per_launch)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || reps <= 0 || !ms_per_launch) return fail(h, DEM_ERR_BAD_INPUT, "dem_time_force_kernel: bad arguments");
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    CU(cudaSetDevice(h->device));
    Control saved;
    int rc = read_control(h, &saved);
    if (rc) return rc;
    // a mid-batch step: second half-kick, next half-kick and drift, written to
    // the spare buffers; nothing is flipped, so the state stays as it was
    Control probe = saved;
    probe.final_step = 0;
    probe.first_step = 0;
    probe.pending_flip = 0;
    probe.record = 0;
    CU(cudaMemcpyAsync(h->d_ctl, &probe, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    launch_force(h, h->stream, 1, false); // warm-up
    CU(cudaEventRecord(h->ev0, h->stream));
    for (int r = 0; r < reps; ++r) launch_force(h, h->stream, 1, false);
    CU(cudaEventRecord(h->ev1, h->stream));
    CU(cudaGetLastError());
    CU(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    *ms_per_launch = ms / reps;
    CU(cudaMemcpyAsync(h->d_ctl, &saved, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}

} // extern "C"

namespace {
// Mean device time of each force kernel (detect, contacts + triangle walls,
// sum) over `reps` time-step force evaluations on the current state, written
// to the spare buffers (the probe control of dem_time_force_kernel); the best
// of three rounds.
int time_force_parts(Handle* h, int reps, double ms[3])
{
    std::vector<cudaEvent_t> ev(4 * (size_t)reps);
    for (auto& e : ev) CU(cudaEventCreate(&e));
    double best[3] = {1e30, 1e30, 1e30};
    int rc = DEM_OK;
    launch_force(h, h->stream, 1, false); // warm-up of this shape
    for (int round = 0; round < 3 && rc == DEM_OK; ++round) {
        for (int r = 0; r < reps; ++r) {
            h->kev = ev.data() + 4 * r;
            launch_force(h, h->stream, 1, false);
        }
        h->kev = nullptr;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
            rc = fail(h, DEM_ERR_CUDA, "dem_autotune: a measured launch failed");
            break;
        }
        double sum[3] = {0, 0, 0};
        for (int r = 0; r < reps; ++r)
            for (int k = 0; k < 3; ++k) {
                float t = 0.f;
                cudaEventElapsedTime(&t, ev[4 * r + k], ev[4 * r + k + 1]);
                sum[k] += t;
            }
        for (int k = 0; k < 3; ++k) best[k] = std::min(best[k], sum[k] / reps);
    }
    h->kev = nullptr;
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 3; ++k) ms[k] = best[k];
    return rc;
}

bool valid_tuning(const dem_tuning& t)
{
    const bool blk = (t.detect_block == 64 || t.detect_block == 128 || t.detect_block == 256) &&
                     (t.sum_block == 64 || t.sum_block == 128 || t.sum_block == 256);
    return blk && t.contacts_blocks_per_sm >= 3 && t.contacts_blocks_per_sm <= 6;
}
} // namespace

extern "C" {

int dem_autotune(dem_handle* hh, int reps, dem_tuning* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || reps <= 0 || !out) return fail(h, DEM_ERR_BAD_INPUT, "dem_autotune: bad arguments");
    if (!h->uploaded || h->initial_pending) return fail(h, DEM_ERR_STATE, "no force evaluation yet (call dem_step)");
    if (h->d.n == 0) return fail(h, DEM_ERR_STATE, "no particles");
    CU(cudaSetDevice(h->device));
    Control saved;
    int rc = read_control(h, &saved);
    if (rc) return rc;
    Control probe = saved;
    probe.final_step = 0;
    probe.first_step = 0;
    probe.pending_flip = 0;
    probe.record = 0;
    CU(cudaMemcpyAsync(h->d_ctl, &probe, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    const dem_tuning start = h->tune;
    double ms[3];
    double before = 0.0;
    if ((rc = time_force_parts(h, reps, ms)) == DEM_OK) {
        before = ms[0] + ms[1] + ms[2];
        // one kernel at a time, the others kept: the three kernels share no
        // launch parameter, and each one's time is measured on its own
        const int blocks[3] = {64, 128, 256};
        const int per_sm[4] = {3, 4, 5, 6};
        double best = 1e30;
        int pick = h->tune.detect_block;
        for (int b : blocks) {
            h->tune.detect_block = b;
            if ((rc = time_force_parts(h, reps, ms))) break;
            if (ms[0] < best) { best = ms[0]; pick = b; }
        }
        h->tune.detect_block = pick;
        best = 1e30;
        pick = h->tune.contacts_blocks_per_sm;
        for (int b : per_sm) {
            if (rc) break;
            h->tune.contacts_blocks_per_sm = b;
            if ((rc = time_force_parts(h, reps, ms))) break;
            if (ms[1] < best) { best = ms[1]; pick = b; }
        }
        h->tune.contacts_blocks_per_sm = pick;
        best = 1e30;
        pick = h->tune.sum_block;
        for (int b : blocks) {
            if (rc) break;
            h->tune.sum_block = b;
            if ((rc = time_force_parts(h, reps, ms))) break;
            if (ms[2] < best) { best = ms[2]; pick = b; }
        }
        h->tune.sum_block = pick;
        if (!rc) rc = time_force_parts(h, reps, ms);
    }
    CU(cudaMemcpyAsync(h->d_ctl, &saved, sizeof(Control), cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (rc) {
        h->tune = start;
        return rc;
    }
    const double after = ms[0] + ms[1] + ms[2];
    if (after > before) h->tune = start; // the measurement did not find a faster shape
    h->tune.ms_before = before;
    h->tune.ms_after = std::min(after, before);
    free_graphs(h); // captured with the previous shapes
    *out = h->tune;
    return DEM_OK;
}

int dem_set_tuning(dem_handle* hh, const dem_tuning* t)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !t) return DEM_ERR_BAD_INPUT;
    if (!valid_tuning(*t))
        return fail(h, DEM_ERR_BAD_INPUT, "dem_set_tuning: blocks of 64, 128 or 256 threads, 3-6 contact blocks per SM");
    h->tune.detect_block = t->detect_block;
    h->tune.contacts_blocks_per_sm = t->contacts_blocks_per_sm;
    h->tune.sum_block = t->sum_block;
    free_graphs(h);
    return DEM_OK;
}

int dem_get_tuning(dem_handle* hh, dem_tuning* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !out) return DEM_ERR_BAD_INPUT;
    *out = h->tune;
    return DEM_OK;
}

const char* dem_last_error(dem_handle* hh)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    return h ? h->err.c_str() : "null handle";
}

void dem_destroy(dem_handle* hh)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_particle_arrays(h);
    if (h->d_rtmp) cudaFree(h->d_rtmp);
    if (h->d_rstats) cudaFree(h->d_rstats);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    delete h;
}

int dem_cg_eval(dem_handle* hh, const dem_cg_grid* grid, double* fields_out);

} // extern "C"

#include "dem_cg.cuh"

int dem_batch_create(const dem_config* config, int n_instances, const dem_instance_desc* instances, dem_handle** out)
{
    if (!config || n_instances < 1) return DEM_ERR_BAD_INPUT;
    dem_config c = *config;
    c.n_instances = n_instances;
    return dem_create(&c, instances, out);
}

int dem_batch_run(dem_handle* hh, int nsteps, dem_globals* out)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !out) return fail(h, DEM_ERR_BAD_INPUT, "dem_batch_run: bad arguments");
    int rc = dem_step(hh, nsteps);
    if (rc) return rc;
    return dem_reduce_batch(hh, 0, (int)h->inst.size(), out);
}

int dem_selftest_wait_expiry(dem_handle* hh, int64_t polls, uint32_t* status)
{
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !status || polls < 1 || polls > (1ll << 24)) return fail(h, DEM_ERR_BAD_INPUT, "dem_selftest_wait_expiry: bad arguments");
    CU(cudaSetDevice(h->device));
    unsigned long long* ctr = nullptr;
    unsigned int* st = nullptr;
    CU(cudaMallocAsync(reinterpret_cast<void**>(&ctr), sizeof(unsigned long long) + 16, h->stream));
    st = reinterpret_cast<unsigned int*>(ctr + 1);
    CU(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) + 16, h->stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)h->rb_grid);
    cfg.blockDim = dim3(RB_BLOCK);
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const long long limit = polls;
    CU(cudaLaunchKernelEx(&cfg, k_barrier_expiry, ctr, st, limit));
    CU(cudaMemcpyAsync(status, st, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaFreeAsync(ctr, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return DEM_OK;
}
