// mdpm_ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A MercuryDPM driver written against the reference's own public API
// (Mercury3D, SpeciesHandler, ParticleHandler, WallHandler, BoundaryHandler),
// compiled together with the reference Kernel by oracle/ref.mk into
// oracle/_ref/libmdpm_ref_{serial,omp}.so. It takes the same input structures
// as the engine's C ABI (include/dem_b200.h), runs the reference's
// initialiseSolve + computeOneTimeStep loop, and returns its state, forces and
// contact list, or the wall time of a timed window (the CPU baseline).
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <vector>

#include "Boundaries/DeletionBoundary.h"
#include "Boundaries/PeriodicBoundary.h"
#include "CG/CG.h"
#include "CG/Coordinates/O.h"
#include "CG/Coordinates/XYZ.h"
#include "CG/Coordinates/XZ.h"
#include "CG/Fields/StandardFields.h"
#include "CG/Functions/Gauss.h"
#include "Interactions/FrictionForceInteractions/FrictionInteraction.h"
#include "Interactions/FrictionForceInteractions/MindlinRollingTorsionInteraction.h"
#include "Interactions/FrictionForceInteractions/SlidingFrictionInteraction.h"
#include "Mercury3D.h"
#include "Particles/SphericalParticle.h"
#include "Species/HertzianViscoelasticMindlinRollingTorsionSpecies.h"
#include "Species/HertzianViscoelasticMindlinSpecies.h"
#include "Species/HertzianViscoelasticSlidingFrictionSpecies.h"
#include "Species/HertzianViscoelasticSpecies.h"
#include "Species/LinearViscoelasticFrictionSpecies.h"
#include "Species/LinearViscoelasticSlidingFrictionSpecies.h"
#include "Species/LinearViscoelasticSpecies.h"
#include "Walls/AxisymmetricIntersectionOfWalls.h"
#include "Walls/InfiniteWall.h"
#include "Walls/IntersectionOfWalls.h"
#include "Walls/TriangleWall.h"

#include "../../include/dem_b200.h"

namespace {

std::vector<dem_deletion_boundary> g_deletions; // DeletionBoundary planes of the next run

// MindlinInteraction keeps its sliding spring without a getter; its public
// write() prints it after the token "slidingSpring" (MindlinInteraction.cc:166-170).
Vec3D mindlin_sliding_spring(const BaseInteraction* c)
{
    std::ostringstream os;
    os.precision(17);
    c->write(os);
    std::istringstream is(os.str());
    std::string tok;
    while (is >> tok)
        if (tok == "slidingSpring") {
            Vec3D v;
            is >> v.X >> v.Y >> v.Z;
            return v;
        }
    return Vec3D(0, 0, 0);
}

void apply_parts(BaseSpecies* s, const dem_species_pair& p)
{
    if (auto* n = dynamic_cast<LinearViscoelasticNormalSpecies*>(s)) {
        n->setStiffness(p.stiffness);
        n->setDissipation(p.dissipation);
        n->setConstantRestitution(p.constant_restitution != 0);
    }
    if (auto* n = dynamic_cast<HertzianViscoelasticNormalSpecies*>(s)) {
        n->setEffectiveElasticModulus(p.elastic_modulus);
        n->setDissipation(p.dissipation);
    }
    if (auto* f = dynamic_cast<SlidingFrictionSpecies*>(s)) {
        f->setSlidingStiffness(p.sliding_stiffness);
        f->setSlidingDissipation(p.sliding_dissipation);
        f->setSlidingFrictionCoefficient(p.sliding_mu);
        f->setSlidingFrictionCoefficientStatic(p.sliding_mu_static);
    }
    if (auto* f = dynamic_cast<FrictionSpecies*>(s)) {
        f->setRollingStiffness(p.rolling_stiffness);
        f->setRollingDissipation(p.rolling_dissipation);
        f->setRollingFrictionCoefficient(p.rolling_mu);
        f->setRollingFrictionCoefficientStatic(p.rolling_mu_static);
        f->setTorsionStiffness(p.torsion_stiffness);
        f->setTorsionDissipation(p.torsion_dissipation);
        f->setTorsionFrictionCoefficient(p.torsion_mu);
        f->setTorsionFrictionCoefficientStatic(p.torsion_mu_static);
    }
    if (auto* f = dynamic_cast<MindlinSpecies*>(s)) {
        f->setEffectiveShearModulus(p.shear_modulus);
        f->setSlidingDissipation(p.sliding_dissipation);
        f->setSlidingFrictionCoefficient(p.sliding_mu);
        f->setSlidingFrictionCoefficientStatic(p.sliding_mu_static);
    }
    if (auto* f = dynamic_cast<MindlinRollingTorsionSpecies*>(s)) {
        f->setRollingDissipation(p.rolling_dissipation);
        f->setRollingFrictionCoefficient(p.rolling_mu);
        f->setRollingFrictionCoefficientStatic(p.rolling_mu_static);
        f->setTorsionDissipation(p.torsion_dissipation);
        f->setTorsionFrictionCoefficient(p.torsion_mu);
        f->setTorsionFrictionCoefficientStatic(p.torsion_mu_static);
    }
}

ParticleSpecies* make_species(const dem_species_pair& p)
{
    if (p.normal_law == DEM_NORMAL_LINEAR_VISCOELASTIC) {
        if (p.friction_law == DEM_FRICTION_SLIDING) return new LinearViscoelasticSlidingFrictionSpecies();
        if (p.friction_law == DEM_FRICTION_ROLLING_TORSION) return new LinearViscoelasticFrictionSpecies();
        return new LinearViscoelasticSpecies();
    }
    if (p.friction_law == DEM_FRICTION_MINDLIN_ROLLING_TORSION) return new HertzianViscoelasticMindlinRollingTorsionSpecies();
    if (p.friction_law == DEM_FRICTION_MINDLIN) return new HertzianViscoelasticMindlinSpecies();
    if (p.friction_law == DEM_FRICTION_SLIDING) return new HertzianViscoelasticSlidingFrictionSpecies();
    return new HertzianViscoelasticSpecies();
}

class RefDriver : public Mercury3D {
public:
    // The reference's own writers of the .ene, .fstat and .data outputs
    // (DPMBase::writeEneHeader / writeEneTimeStep, writeFstatHeader,
    // outputXBallsData) into the given streams.
    void write_outputs(std::ostream& ene, std::ostream& fstat, std::ostream& data) const
    {
        writeEneHeader(ene);
        writeEneTimeStep(ene);
        writeFstatHeader(fstat);
        outputXBallsData(data);
    }

    // DPMBase::solve with the .ene file as the only output, a line every
    // save_count time steps (DPMBase::writeEneTimeStep, DPMBase.cc:2100-2123),
    // to name.ene. The soft stop stays off: it would replace the host
    // process's SIGINT / SIGTERM handlers.
    void solve_writing_ene(const std::string& name, unsigned save_count)
    {
        setName(name);
        eneFile.setFileType(FileType::ONE_FILE);
        eneFile.setSaveCount(save_count);
        disableSoftStop();
        solve();
    }

    const dem_config* cfg = nullptr;
    const dem_instance_desc* inst = nullptr;
    const dem_species_pair* species = nullptr;
    const double* density = nullptr;
    const dem_wall* walls = nullptr;
    int nwalls = 0;
    const dem_particles_soa* in = nullptr;

    void setupInitialConditions() override
    {
        const int ns = inst->n_species;
        for (int a = 0; a < ns; ++a) {
            const dem_species_pair& p = species[inst->species_offset + a * ns + a];
            ParticleSpecies* s = make_species(p);
            s->setDensity(density[a]);
            apply_parts(s, p);
            speciesHandler.addObject(s);
        }
        for (int a = 0; a < ns; ++a)
            for (int b = a + 1; b < ns; ++b)
                apply_parts(speciesHandler.getMixedObject(a, b), species[inst->species_offset + a * ns + b]);
        setRotation(cfg->rotation != 0);
        for (int w = 0; w < nwalls; ++w) {
            const dem_wall& x = walls[w];
            BaseWall* wall = nullptr;
            if (x.type == DEM_WALL_INFINITE) {
                wall = new InfiniteWall();
            } else if (x.type == DEM_WALL_TRIANGLE) {
                TriangleWall* tw = new TriangleWall();
                tw->setVertices(Vec3D(x.faces[0][0], x.faces[0][1], x.faces[0][2]),
                                Vec3D(x.faces[1][0], x.faces[1][1], x.faces[1][2]),
                                Vec3D(x.faces[2][0], x.faces[2][1], x.faces[2][2]),
                                Vec3D(x.position[0], x.position[1], x.position[2]));
                tw->setGroupId((unsigned)x.group);
                wall = tw;
            } else {
                IntersectionOfWalls* iw = (x.type == DEM_WALL_AXISYMMETRIC) ? new AxisymmetricIntersectionOfWalls()
                                                                           : new IntersectionOfWalls();
                for (int f = 0; f < x.n_faces; ++f)
                    iw->addObject(Vec3D(x.faces[f][0], x.faces[f][1], x.faces[f][2]),
                                  Vec3D(x.faces[f][3], x.faces[f][4], x.faces[f][5]));
                wall = iw;
            }
            wall->setSpecies(speciesHandler.getObject(x.species));
            wall->setOrientation(Quaternion(x.orientation[0], x.orientation[1], x.orientation[2], x.orientation[3]));
            wall->setPosition(Vec3D(x.position[0], x.position[1], x.position[2]));
            wall->setVelocity(Vec3D(x.velocity[0], x.velocity[1], x.velocity[2]));
            wall->setAngularVelocity(Vec3D(x.angular_velocity[0], x.angular_velocity[1], x.angular_velocity[2]));
            wallHandler.copyAndAddObject(*wall);
            delete wall;
        }
        for (int k = 0; k < 3; ++k) {
            if (!((inst->periodic_mask >> k) & 1u)) continue;
            PeriodicBoundary b;
            Vec3D n(k == 0, k == 1, k == 2);
            b.set(n, inst->periodic_min[k], inst->periodic_max[k]);
            boundaryHandler.copyAndAddObject(b);
        }
        for (const auto& db : g_deletions) {
            DeletionBoundary b;
            b.set(Vec3D(db.normal[0], db.normal[1], db.normal[2]), db.distance);
            boundaryHandler.copyAndAddObject(b);
        }
        SphericalParticle p;
        for (int64_t i = 0; i < in->n; ++i) {
            p.setSpecies(speciesHandler.getObject(in->species[i]));
            p.setRadius(in->radius[i]);
            p.setPosition(Vec3D(in->position[3 * i], in->position[3 * i + 1], in->position[3 * i + 2]));
            p.setVelocity(Vec3D(in->velocity[3 * i], in->velocity[3 * i + 1], in->velocity[3 * i + 2]));
            if (in->angular_velocity)
                p.setAngularVelocity(
                    Vec3D(in->angular_velocity[3 * i], in->angular_velocity[3 * i + 1], in->angular_velocity[3 * i + 2]));
            else
                p.setAngularVelocity(Vec3D(0, 0, 0));
            if (in->orientation)
                p.setOrientation(Quaternion(in->orientation[4 * i], in->orientation[4 * i + 1],
                                            in->orientation[4 * i + 2], in->orientation[4 * i + 3]));
            else
                p.setOrientation(Quaternion(1, 0, 0, 0));
            BaseParticle* q = particleHandler.copyAndAddObject(p);
            if (in->inv_mass[i] == 0.0) q->fixParticle();
        }
    }
};

void setup(RefDriver& d, const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
           const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int threads)
{
    d.cfg = cfg;
    d.inst = inst;
    d.species = species;
    d.density = density;
    d.walls = walls;
    d.nwalls = nwalls;
    d.in = in;
    d.setName("mdpm_ref_driver");
    d.setFileType(FileType::NO_FILE);
    d.setTimeStep(cfg->time_step);
    d.setTimeMax(1e300);
    d.setGravity(Vec3D(inst->gravity[0], inst->gravity[1], inst->gravity[2]));
    d.setBackgroundDrag(cfg->background_drag);
    Vec3D lo(inst->domain_min[0], inst->domain_min[1], inst->domain_min[2]);
    Vec3D hi(inst->domain_max[0], inst->domain_max[1], inst->domain_max[2]);
    for (int k = 0; k < 3; ++k)
        if ((inst->periodic_mask >> k) & 1u) {
            lo.setComponent(k, inst->periodic_min[k]);
            hi.setComponent(k, inst->periodic_max[k]);
        }
    d.setDomain(lo, hi);
#ifdef MERCURYDPM_USE_OMP
    d.setNumberOfOMPThreads(threads > 0 ? threads : 1);
#else
    (void)threads;
#endif
}

} // namespace

extern "C" {

// DeletionBoundary planes for the following runs (instance field ignored).
void mdpm_ref_set_deletion(const dem_deletion_boundary* b, int n) { g_deletions.assign(b, b + n); }

} // extern "C"

extern "C" {

// Same contract as oracle_run (oracle/dem_oracle.cpp), with the species
// densities the reference needs to derive the particle masses.
int mdpm_ref_run(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                 const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in, int nsteps,
                 dem_particles_soa* out, double* force, double* torque, dem_contacts_soa* contacts_out,
                 int64_t contacts_capacity, int64_t* contacts_count, double* energies /* kin, rot, grav, ela */)
{
    RefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.initialiseSolve();
    for (int k = 0; k < nsteps; ++k) d.computeOneTimeStep();
    const int64_t n = in->n;
    // deleted particles leave the handler (and reorder it): rows are matched by
    // id, which the tests set to the caller index; rows of deleted particles
    // keep instance -1
    if (out && out->instance)
        for (int64_t i = 0; i < n; ++i) out->instance[i] = -1;
    for (int64_t r = 0; r < (int64_t)d.particleHandler.getSize(); ++r) {
        const BaseParticle* p = d.particleHandler.getObject((unsigned)r);
        const int64_t i = (int64_t)p->getId();
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
            contacts_out->id_p[cnt] = (int)c->getP()->getId();
            contacts_out->id_i[cnt] = (int)(wall ? c->getI()->getIndex() : c->getI()->getId());
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
