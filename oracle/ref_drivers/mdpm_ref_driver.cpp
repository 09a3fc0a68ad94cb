// mdpm_ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A MercuryDPM driver written against the reference's own public API
// (Mercury3D, SpeciesHandler, ParticleHandler, WallHandler, BoundaryHandler),
// compiled together with the reference Kernel by oracle/ref.mk into
// oracle/_ref/libmdpm_ref_{serial,omp}.so. It takes the same input structures
// as the engine's C ABI (include/dem_b200.h), runs the reference's
// initialiseSolve + computeOneTimeStep loop, and returns its state, forces and
// contact list, or the wall time of a timed window (the CPU baseline).
#include <algorithm>
#include <limits>
#include <utility>

#include "ref_driver.h"

#include "Chute.h"

namespace {
using RefDriver = RefDriverT<Mercury3D>;

// A Chute driver whose set-up is the checker's, followed by the chute's
// compact inflow fill (Chute.cc:1083-1115) from a freshly seeded generator.
class ChuteFillDriver : public RefDriverT<Chute> {
public:
    void setupInitialConditions() override
    {
        RefDriverT<Chute>::setupInitialConditions();
        this->setInflowParticleRadius(g_fill.min_radius, g_fill.max_radius);
        this->setFixedParticleRadius(g_fill.fixed_particle_radius);
        this->setInflowHeight(g_fill.inflow_height);
        this->random.setRandomSeed(g_insertion_seed);
        this->addFlowParticlesCompactly();
        g_fill_height = this->getInflowHeight();
    }
};
} // namespace

extern "C" {

// DeletionBoundary planes for the following runs (instance field ignored).
void mdpm_ref_set_deletion(const dem_deletion_boundary* b, int n) { g_deletions.assign(b, b + n); }
// the between-steps change of the next mdpm_ref_run (step < 0: none)
void mdpm_ref_set_event(long long step, int wall, const dem_deletion_boundary* b, int n)
{
    g_event_step = step;
    g_event_wall = wall;
    g_event_deletions.assign(b, b + n);
}
// CubeInsertionBoundary objects of the following runs and DPMBase::random's seed
// (the input rows of radius 0 are then skipped: they are the engine's free rows)
void mdpm_ref_set_insertion(const dem_insertion_boundary* b, int n, unsigned long long seed)
{
    g_insertions.assign(b, b + n);
    g_insertion_seed = (unsigned long)seed;
}
// RNG::getRandomNumber(0, 1) n times after RNG::setRandomSeed(seed)
void mdpm_ref_rng_draws(unsigned long long seed, int n, double* out)
{
    RNG r;
    r.setRandomSeed((unsigned long)seed);
    for (int i = 0; i < n; ++i) out[i] = r.getRandomNumber(0, 1);
}
// PSD::drawSample n times from setDistributionUniform(rmin, rmax, bins) and setFixedSeed(seed)
void mdpm_ref_psd_draws(double rmin, double rmax, int bins, int seed, int n, double* out)
{
    PSD psd;
    psd.setDistributionUniform(rmin, rmax, bins);
    psd.setFixedSeed(seed);
    for (int i = 0; i < n; ++i) out[i] = psd.drawSample();
}
// particles and volume placed by each insertion boundary in the last run
int mdpm_ref_insertion_counts(long long* inserted, double* volume, int capacity)
{
    const int n = (int)g_inserted.size();
    for (int k = 0; k < n && k < capacity; ++k) {
        inserted[k] = g_inserted[k];
        volume[k] = g_inserted_volume[k];
    }
    return n;
}

} // extern "C"

extern "C" {

} // extern "C"

namespace {
template <class Driver>
int run_and_report(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                   const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int nsteps,
                   dem_particles_soa* out, double* force, double* torque, dem_contacts_soa* contacts_out,
                   int64_t contacts_capacity, int64_t* contacts_count, double* energies)
{
    Driver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    const int64_t n = in->n;
    // Rows are matched by id. The uploaded particles have ids 0, 1, ... in the
    // order of the rows (of nonzero radius, when insertion boundaries or a fill
    // are set); placed particles take the rows of radius 0 in the order they
    // were placed, whose ids the engine uses (the ids of contacts are reported
    // as those). The reference gives them the ids after the uploaded ones, with
    // gaps where periodic ghost particles drew ids, and a placed particle may
    // be deleted later, so each one is given its row as soon as it appears: a
    // particle placed in a step is still there at its end (deletions come
    // before the placements of a step). Rows of deleted or never filled
    // particles keep instance -1.
    std::vector<int64_t> live_rows, free_rows;
    for (int64_t i = 0; i < n; ++i) ((free_rows_in_use() && in->radius[i] == 0.0) ? free_rows : live_rows).push_back(i);
    std::vector<std::pair<unsigned, int64_t>> placed_row; // reference id -> row, in placement order
    unsigned next_new_id = (unsigned)live_rows.size();    // ids below were uploaded or already seen
    auto note_placed = [&]() {
        if (!free_rows_in_use()) return;
        std::vector<unsigned> fresh;
        for (unsigned r = 0; r < d.particleHandler.getSize(); ++r) {
            const unsigned id = d.particleHandler.getObject(r)->getId();
            if (id >= next_new_id) fresh.push_back(id);
        }
        std::sort(fresh.begin(), fresh.end());
        for (unsigned id : fresh)
            if (placed_row.size() < free_rows.size()) placed_row.emplace_back(id, free_rows[placed_row.size()]);
        if (!fresh.empty()) next_new_id = fresh.back() + 1;
    };
    d.initialiseSolve();
    note_placed(); // a fill made by the set-up
    for (int k = 0; k < nsteps; ++k) {
        d.computeOneTimeStep();
        note_placed();
        apply_event(d, k + 1);
    }
    collect_insertions(d);
    std::vector<std::pair<unsigned, int64_t>> id_row(placed_row); // reference id -> row
    for (unsigned r = 0; r < d.particleHandler.getSize(); ++r) {
        const unsigned id = d.particleHandler.getObject(r)->getId();
        if (id < live_rows.size()) id_row.emplace_back(id, live_rows[id]);
    }
    std::sort(id_row.begin(), id_row.end());
    auto row_of = [&](unsigned id) -> int64_t {
        auto it = std::lower_bound(id_row.begin(), id_row.end(), std::make_pair(id, (int64_t)-1));
        return (it != id_row.end() && it->first == id) ? it->second : -1;
    };
    auto our_id = [&](unsigned id) -> int { const int64_t r = row_of(id); return r < 0 ? -1 : in->id[r]; };
    if (out && out->instance)
        for (int64_t i = 0; i < n; ++i) out->instance[i] = -1;
    for (int64_t r = 0; r < (int64_t)d.particleHandler.getSize(); ++r) {
        const BaseParticle* p = d.particleHandler.getObject((unsigned)r);
        const int64_t i = row_of(p->getId());
        if (i < 0 || i >= n) continue;
        if (out && out->instance) out->instance[i] = 0;
        const Vec3D x = p->getPosition(), v = p->getVelocity(), w = p->getAngularVelocity();
        const Quaternion q = p->getOrientation();
        if (out && out->position) { out->position[3 * i] = x.X; out->position[3 * i + 1] = x.Y; out->position[3 * i + 2] = x.Z; }
        if (out && out->velocity) { out->velocity[3 * i] = v.X; out->velocity[3 * i + 1] = v.Y; out->velocity[3 * i + 2] = v.Z; }
        if (out && out->angular_velocity) {
            out->angular_velocity[3 * i] = w.X; out->angular_velocity[3 * i + 1] = w.Y; out->angular_velocity[3 * i + 2] = w.Z;
        }
        if (out && out->orientation) {
            out->orientation[4 * i] = q.getComponent(0); out->orientation[4 * i + 1] = q.getComponent(1);
            out->orientation[4 * i + 2] = q.getComponent(2); out->orientation[4 * i + 3] = q.getComponent(3);
        }
        if (out && out->inv_mass) out->inv_mass[i] = p->getInvMass();
        if (out && out->inv_inertia) out->inv_inertia[i] = p->getInvInertia().XX;
        if (out && out->radius) out->radius[i] = p->getRadius();
        const Vec3D f = p->getForce(), t = p->getTorque();
        if (force) { force[3 * i] = f.X; force[3 * i + 1] = f.Y; force[3 * i + 2] = f.Z; }
        if (torque) { torque[3 * i] = t.X; torque[3 * i + 1] = t.Y; torque[3 * i + 2] = t.Z; }
    }
    int64_t cnt = 0;
    const unsigned last = nsteps > 0 ? (unsigned)nsteps : 1u;
    for (BaseInteraction* c : d.interactionHandler) {
        if (c->getTimeStamp() != last) continue;
        const bool wall = dynamic_cast<BaseParticle*>(c->getI()) == nullptr;
        if (contacts_out && cnt < contacts_capacity) {
            contacts_out->id_p[cnt] = our_id(c->getP()->getId());
            contacts_out->id_i[cnt] = wall ? (int)c->getI()->getIndex() : our_id(c->getI()->getId());
            if (contacts_out->is_wall) contacts_out->is_wall[cnt] = wall;
            if (contacts_out->periodic) {
                bool per = false;
                if (!wall)
                    for (int k = 0; k < 3; ++k)
                        if ((inst->periodic_mask >> k) & 1u) {
                            const double dx = c->getP()->getPosition().getComponent(k) - c->getI()->getPosition().getComponent(k);
                            if (std::fabs(dx) > 0.5 * (inst->periodic_max[k] - inst->periodic_min[k])) per = true;
                        }
                contacts_out->periodic[cnt] = per;
            }
            if (contacts_out->overlap) contacts_out->overlap[cnt] = c->getOverlap();
            if (contacts_out->force) {
                const Vec3D f = c->getForce();
                contacts_out->force[3 * cnt] = f.X; contacts_out->force[3 * cnt + 1] = f.Y; contacts_out->force[3 * cnt + 2] = f.Z;
            }
            if (contacts_out->springs) {
                double* s = contacts_out->springs + 9 * cnt;
                for (int k = 0; k < 9; ++k) s[k] = 0.0;
                Vec3D sl(0, 0, 0), ro(0, 0, 0), to(0, 0, 0);
                if (auto* fi = dynamic_cast<SlidingFrictionInteraction*>(c)) sl = fi->getSlidingSpring();
                if (dynamic_cast<MindlinInteraction*>(c)) sl = mindlin_sliding_spring(c);
                if (auto* fi = dynamic_cast<FrictionInteraction*>(c)) { ro = fi->getRollingSpring(); to = fi->getTorsionSpring(); }
                if (auto* fi = dynamic_cast<MindlinRollingTorsionInteraction*>(c)) { ro = fi->getRollingSpring(); to = fi->getTorsionSpring(); }
                s[0] = sl.X; s[1] = sl.Y; s[2] = sl.Z; s[3] = ro.X; s[4] = ro.Y; s[5] = ro.Z; s[6] = to.X; s[7] = to.Y; s[8] = to.Z;
            }
        }
        ++cnt;
    }
    if (contacts_count) *contacts_count = cnt;
    if (contacts_out) contacts_out->n = cnt < contacts_capacity ? cnt : contacts_capacity;
    if (energies) {
        energies[0] = d.getKineticEnergy();
        energies[1] = d.getRotationalEnergy();
        energies[2] = d.getGravitationalEnergy();
        energies[3] = d.getElasticEnergy();
    }
    return 0;
}
} // namespace

extern "C" {

// Same contract as oracle_run (oracle/dem_oracle.cpp), with the species
// densities the reference needs to derive the particle masses.
int mdpm_ref_run(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                 const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int nsteps,
                 dem_particles_soa* out, double* force, double* torque, dem_contacts_soa* contacts_out,
                 int64_t contacts_capacity, int64_t* contacts_count, double* energies /* kin, rot, grav, ela */)
{
    return run_and_report<RefDriver>(cfg, inst, species, density, walls, nwalls, in, nsteps, out, force, torque,
                                     contacts_out, contacts_capacity, contacts_count, energies);
}

// mdpm_ref_run on a Chute whose set-up ends with the compact inflow fill
// `fill` (DPMBase::random seeded with `seed` first); *inflow_height receives
// the height the fill ended with.
int mdpm_ref_run_chute_fill(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                            const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                            const dem_chute_fill* fill, unsigned long long seed, int nsteps, dem_particles_soa* out,
                            double* force, double* torque, dem_contacts_soa* contacts_out, int64_t contacts_capacity,
                            int64_t* contacts_count, double* inflow_height)
{
    g_fill = *fill;
    g_fill_set = true;
    g_insertion_seed = (unsigned long)seed;
    const int rc = run_and_report<ChuteFillDriver>(cfg, inst, species, density, walls, nwalls, in, nsteps, out, force,
                                                   torque, contacts_out, contacts_capacity, contacts_count, nullptr);
    g_fill_set = false;
    if (inflow_height) *inflow_height = g_fill_height;
    return rc;
}

} // extern "C"

namespace {

template <class Coordinates>
void reference_cg(RefDriver& d, const dem_cg_grid* grid, double* out)
{
    CG<Coordinates, CGFunctions::Gauss, CGFields::StandardFields> cg;
    cg.setNX(grid->n[0]);
    cg.setNY(grid->n[1]);
    cg.setNZ(grid->n[2]);
    cg.setMin(Vec3D(grid->min[0], grid->min[1], grid->min[2]));
    cg.setMax(Vec3D(grid->max[0], grid->max[1], grid->max[2]));
    cg.setWidth(grid->width);
    auto* p = d.cgHandler.copyAndAddObject(cg);
    p->statFile.setFileType(FileType::NO_FILE);
    // CG::initialise opens the stat file whatever its type (CG.hcc:179): send it nowhere
    p->statFile.setName("/dev/null");
    p->initialise();
    p->evaluate();
    size_t k = 0;
    for (const auto& pt : p->getPoints()) {
        double* f = out + 29 * k++;
        f[0] = pt.getVolumeFraction();
        f[1] = pt.getDensity();
        const Vec3D m = pt.getMomentum();
        f[2] = m.X; f[3] = m.Y; f[4] = m.Z;
        const MatrixSymmetric3D mf = pt.getMomentumFlux();
        f[5] = mf.XX; f[6] = mf.XY; f[7] = mf.XZ; f[8] = mf.YY; f[9] = mf.YZ; f[10] = mf.ZZ;
        const Matrix3D cs = pt.getContactStress();
        f[11] = cs.XX; f[12] = cs.XY; f[13] = cs.XZ; f[14] = cs.YX; f[15] = cs.YY; f[16] = cs.YZ;
        f[17] = cs.ZX; f[18] = cs.ZY; f[19] = cs.ZZ;
        const Vec3D ifd = pt.getInteractionForceDensity();
        f[20] = ifd.X; f[21] = ifd.Y; f[22] = ifd.Z;
        for (size_t i = 0; i < 6; ++i) f[23 + i] = pt.getParticleSizeDensity(i);
    }
}

} // namespace

extern "C" {

// The reference's own CG<Coordinates, Gauss, StandardFields> evaluated after
// `nsteps` time steps (what writeOutputFiles would compute at the start of the
// next step). coordinates: 0 = O, 1 = XZ, 2 = XYZ; 29 fields per point.
int mdpm_ref_cg(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int nsteps,
                const dem_cg_grid* grid, double* fields_out)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.initialiseSolve();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    if (grid->coordinates == DEM_CG_O)
        reference_cg<CGCoordinates::O>(d, grid, fields_out);
    else if (grid->coordinates == DEM_CG_XZ)
        reference_cg<CGCoordinates::XZ>(d, grid, fields_out);
    else
        reference_cg<CGCoordinates::XYZ>(d, grid, fields_out);
    return 0;
}

// The reference's .ene, .fstat and .data outputs after `nsteps` time steps,
// written to prefix.ene / prefix.fstat / prefix.data with the precision of
// the reference's file streams (10, DPMBase.cc:211-213).
int mdpm_ref_write_outputs(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                           const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                           int nsteps, const char* prefix)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.initialiseSolve();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    const std::string pre(prefix);
    std::ofstream ene(pre + ".ene"), fstat(pre + ".fstat"), data(pre + ".data");
    ene.precision(10);
    fstat.precision(10);
    data.precision(10);
    d.write_outputs(ene, fstat, data);
    return 0;
}

// The reference restarted from a .restart file (DPMBase::readRestartFile,
// DPMBase.cc:3015-3060, then initialiseSolve without setupInitialConditions)
// and advanced `nsteps` time steps; returns its state (rows by particle id,
// which the tests set to the upload index), forces, and the contacts of its
// last force evaluation with their springs. The restart path must end in
// ".restart".
int mdpm_ref_restart_run(const char* path, int nsteps, int64_t n, dem_particles_soa* out, double* force,
                         double* torque, dem_contacts_soa* contacts_out, int64_t contacts_capacity,
                         int64_t* contacts_count)
{
    Mercury3D d;
    d.setName("mdpm_ref_restart");
    if (!d.readRestartFile(std::string(path))) return 1;
    d.setFileType(FileType::NO_FILE);
    d.setTimeMax(1e300);
    const unsigned n0 = d.getNumberOfTimeSteps();
    d.initialiseSolve();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    unsigned per_mask = 0;
    double per_lo[3] = {0, 0, 0}, per_hi[3] = {0, 0, 0};
    for (BaseBoundary* b : d.boundaryHandler)
        if (auto* pb = dynamic_cast<PeriodicBoundary*>(b))
            for (int k = 0; k < 3; ++k)
                if (pb->getNormal().getComponent(k) != 0) {
                    per_mask |= 1u << k;
                    per_lo[k] = pb->getDistanceLeft();
                    per_hi[k] = pb->getDistanceRight();
                }
    for (int64_t r = 0; r < (int64_t)d.particleHandler.getSize(); ++r) {
        const BaseParticle* p = d.particleHandler.getObject((unsigned)r);
        const int64_t i = (int64_t)p->getId();
        if (i < 0 || i >= n) continue;
        const Vec3D x = p->getPosition(), v = p->getVelocity(), w = p->getAngularVelocity(), f = p->getForce(),
                    t = p->getTorque();
        for (int k = 0; k < 3; ++k) {
            if (out && out->position) out->position[3 * i + k] = x.getComponent(k);
            if (out && out->velocity) out->velocity[3 * i + k] = v.getComponent(k);
            if (out && out->angular_velocity) out->angular_velocity[3 * i + k] = w.getComponent(k);
            if (force) force[3 * i + k] = f.getComponent(k);
            if (torque) torque[3 * i + k] = t.getComponent(k);
        }
    }
    int64_t cnt = 0;
    const unsigned last = n0 + (nsteps > 0 ? (unsigned)nsteps : 1u);
    for (BaseInteraction* c : d.interactionHandler) {
        if (c->getTimeStamp() != last) continue;
        const bool wall = dynamic_cast<BaseParticle*>(c->getI()) == nullptr;
        if (contacts_out && cnt < contacts_capacity) {
            contacts_out->id_p[cnt] = (int)c->getP()->getId();
            contacts_out->id_i[cnt] = (int)(wall ? c->getI()->getIndex() : c->getI()->getId());
            if (contacts_out->is_wall) contacts_out->is_wall[cnt] = wall;
            if (contacts_out->periodic) {
                bool per = false;
                if (!wall)
                    for (int k = 0; k < 3; ++k)
                        if ((per_mask >> k) & 1u) {
                            const double dx = c->getP()->getPosition().getComponent(k) -
                                              c->getI()->getPosition().getComponent(k);
                            if (std::fabs(dx) > 0.5 * (per_hi[k] - per_lo[k])) per = true;
                        }
                contacts_out->periodic[cnt] = per;
            }
            if (contacts_out->overlap) contacts_out->overlap[cnt] = c->getOverlap();
            if (contacts_out->force) {
                const Vec3D f = c->getForce();
                for (int k = 0; k < 3; ++k) contacts_out->force[3 * cnt + k] = f.getComponent(k);
            }
            if (contacts_out->springs) {
                double* s = contacts_out->springs + 9 * cnt;
                for (int k = 0; k < 9; ++k) s[k] = 0.0;
                Vec3D sl(0, 0, 0), ro(0, 0, 0), to(0, 0, 0);
                if (auto* fi = dynamic_cast<SlidingFrictionInteraction*>(c)) sl = fi->getSlidingSpring();
                if (dynamic_cast<MindlinInteraction*>(c)) sl = mindlin_sliding_spring(c);
                if (auto* fi = dynamic_cast<FrictionInteraction*>(c)) { ro = fi->getRollingSpring(); to = fi->getTorsionSpring(); }
                if (auto* fi = dynamic_cast<MindlinRollingTorsionInteraction*>(c)) { ro = fi->getRollingSpring(); to = fi->getTorsionSpring(); }
                for (int k = 0; k < 3; ++k) {
                    s[k] = sl.getComponent(k);
                    s[3 + k] = ro.getComponent(k);
                    s[6 + k] = to.getComponent(k);
                }
            }
        }
        ++cnt;
    }
    if (contacts_count) *contacts_count = cnt;
    return 0;
}

// The reference's restart file (DPMBase::write, DPMBase.cc:3550) after
// `nsteps` time steps, written to `path` with the precision of its restart
// stream (std::numeric_limits<double>::digits10 = 15, DPMBase.cc:214-215).
int mdpm_ref_write_restart(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                           const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                           int nsteps, const char* path)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.initialiseSolve();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    std::ofstream os(path);
    os.precision(std::numeric_limits<double>::digits10);
    d.write(os, true);
    return 0;
}

// CPU baseline: builds the same simulation, runs `warmup` steps, then times
// `nsteps` calls of computeOneTimeStep with std::chrono (set-up and output
// excluded). `threads` is the OpenMP thread count (ignored by the serial build).
int mdpm_ref_time(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                  const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int warmup,
                  int nsteps, int threads, double* seconds)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, threads);
    d.initialiseSolve();
    for (int k = 0; k < warmup; ++k) d.computeOneTimeStep();
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    const auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    return 0;
}

// The reference's own run of `nsteps` time steps through DPMBase::solve(),
// writing its .ene file (prefix.ene) every `save_count` steps and at the end.
// timeMax sits half a step short of nsteps * dt, so that the solve loop
// (while time < timeMax) takes exactly nsteps steps.
int mdpm_ref_solve_ene(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                       const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                       int nsteps, int save_count, int threads, const char* prefix)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, threads);
    d.setTimeMax((nsteps - 0.5) * cfg->time_step);
    d.solve_writing_ene(prefix, (unsigned)save_count);
    return 0;
}

// mdpm_ref_time, also reporting the interactions the handler holds (particle
// pairs and wall contacts) when the timed window starts and when it ends, so
// that a caller can show which phase of the run the window sampled.
int mdpm_ref_time_window(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                         const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                         int warmup, int nsteps, int threads, double* seconds, int64_t* interactions_start,
                         int64_t* interactions_end)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, threads);
    d.initialiseSolve();
    for (int k = 0; k < warmup; ++k) d.computeOneTimeStep();
    *interactions_start = (int64_t)d.interactionHandler.getNumberOfObjects();
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    const auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    *interactions_end = (int64_t)d.interactionHandler.getNumberOfObjects();
    return 0;
}

} // extern "C"

extern "C" {

// The procedure of Drivers/Calibration/CalibrationHeap.cpp (GranuHeap::
// actionsAfterTimeStep, CalibrationHeap.cpp:119-160) on the reference
// Kernel, for a heap set up by the caller: a fill stage inside the casing
// (wall `casing`, the last one), then, at the first check with kinetic
// energy below 1e-2 of the elastic energy, the casing is removed and a
// DeletionBoundary z < 0 added; from twice that time on, the first quiet
// check gives the angle of repose atan(4 COM_z / R_base) and ends the run
// 0.05 s later, every quiet check until then measuring it again. Checks
// come every `check_every` time steps, as in the reference (every 1000th).
// The reference keeps the removal time in an uninitialised local variable
// (`double fillTime;`, read at a later call); this restatement uses the time
// the casing was removed, which is what the code intends.
// out: [angle of repose (deg, NaN if never measured), removal time, end time,
//       time steps, particles left, centre of mass z]
int mdpm_ref_heap_procedure(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                            const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                            int casing, double base_radius, int check_every, long long max_steps, int threads,
                            double* out)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, threads);
    bool fill = true, first_aor = true;
    double removal_time = 0.0, aor = std::nan("");
    long long count = 0;
    d.setTimeMax(1e300);
    d.after_step = [&]() {
        if (++count % check_every) return;
        const double ke = d.getKineticEnergy(), ee = d.getElasticEnergy();
        if (fill) {
            if (ke < 1e-2 * ee) {
                fill = false;
                removal_time = d.getTime();
                d.wallHandler.removeObject((unsigned)casing);
                DeletionBoundary b;
                b.set(Vec3D(0, 0, -1), 0);
                d.boundaryHandler.copyAndAddObject(b);
            }
        } else if (d.getTime() > 2.0 * removal_time && ke < 1e-2 * ee) {
            aor = std::atan(4.0 * d.getCentreOfMass().Z / base_radius) * 180.0 / constants::pi;
            if (first_aor) {
                d.setTimeMax(d.getTime() + 0.05);
                first_aor = false;
            }
        }
    };
    d.initialiseSolve();
    long long steps = 0;
    while (d.getTime() < d.getTimeMax() && steps < max_steps) {
        d.computeOneTimeStep();
        ++steps;
    }
    out[0] = aor;
    out[1] = removal_time;
    out[2] = d.getTime();
    out[3] = (double)steps;
    out[4] = (double)d.particleHandler.getSize();
    out[5] = d.particleHandler.getSize() ? d.getCentreOfMass().Z : std::nan("");
    return 0;
}

} // extern "C"
