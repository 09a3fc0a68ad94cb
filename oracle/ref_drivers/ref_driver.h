// ref_driver.h -- TEST INFRASTRUCTURE ONLY.
//
// The MercuryDPM driver of the checker, written against the reference's own
// public API (SpeciesHandler, ParticleHandler, WallHandler, BoundaryHandler)
// and templated on its base class: RefDriverT<Mercury3D> is the reference
// itself (oracle/ref_drivers/mdpm_ref_driver.cpp), RefDriverT<GpuMercury3D>
// the same driver with the engine's drop-in base class
// (oracle/ref_drivers/gpu/gpu_binding_driver.cpp). It takes the engine's C
// ABI structures (include/dem_b200.h) as its input.
#pragma once
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <vector>
#include "Boundaries/ChuteInsertionBoundary.h"
#include "Boundaries/CubeInsertionBoundary.h"
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
// CubeInsertionBoundary objects of the next run and the seed of DPMBase::random
std::vector<dem_insertion_boundary> g_insertions;
unsigned long g_insertion_seed = 0;
// Chute::addFlowParticlesCompactly of the next Chute run (ChuteFillDriver)
dem_chute_fill g_fill{};
bool g_fill_set = false;
double g_fill_height = 0.0; // Chute::getInflowHeight after it
// rows of radius 0 are the engine's free rows, not particles
inline bool free_rows_in_use() { return !g_insertions.empty() || g_fill_set; }
// particles and volume each insertion boundary placed in the last run
std::vector<long long> g_inserted;
std::vector<double> g_inserted_volume;

// A change between two time steps of the next run (as a driver's
// actionsAfterTimeStep makes it, e.g. Drivers/Calibration/CalibrationHeap.cpp:
// 119-131): after step g_event_step, wall g_event_wall (handler index, -1:
// none) is removed and the planes g_event_deletions are added.
long long g_event_step = -1;
int g_event_wall = -1;
std::vector<dem_deletion_boundary> g_event_deletions;

template <class Driver>
void apply_event(Driver& d, long long step)
{
    if (step != g_event_step) return;
    if (g_event_wall >= 0) d.wallHandler.removeObject((unsigned)g_event_wall);
    for (const auto& db : g_event_deletions) {
        DeletionBoundary b;
        b.set(Vec3D(db.normal[0], db.normal[1], db.normal[2]), db.distance);
        d.boundaryHandler.copyAndAddObject(b);
    }
}

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

template <class Base>
class RefDriverT : public Base {
public:
    // a driver's hook, run where the reference runs actionsAfterTimeStep
    // (DPMBase::computeOneTimeStep: after the forces, before the second
    // half-kick and the time increment)
    std::function<void()> after_step;
    void actionsAfterTimeStep() override
    {
        if (after_step) after_step();
    }

    // The reference's own writers of the .ene, .fstat and .data outputs
    // (DPMBase::writeEneHeader / writeEneTimeStep, writeFstatHeader,
    // outputXBallsData) into the given streams.
    void write_outputs(std::ostream& ene, std::ostream& fstat, std::ostream& data) const
    {
        this->writeEneHeader(ene);
        this->writeEneTimeStep(ene);
        this->writeFstatHeader(fstat);
        this->outputXBallsData(data);
    }

    // DPMBase::solve with the .ene file as the only output, a line every
    // save_count time steps (DPMBase::writeEneTimeStep, DPMBase.cc:2100-2123),
    // to name.ene. The soft stop stays off: it would replace the host
    // process's SIGINT / SIGTERM handlers.
    void solve_writing_ene(const std::string& name, unsigned save_count)
    {
        this->setName(name);
        this->eneFile.setFileType(FileType::ONE_FILE);
        this->eneFile.setSaveCount(save_count);
        this->disableSoftStop();
        this->solve();
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
            this->speciesHandler.addObject(s);
        }
        for (int a = 0; a < ns; ++a)
            for (int b = a + 1; b < ns; ++b)
                apply_parts(this->speciesHandler.getMixedObject(a, b), species[inst->species_offset + a * ns + b]);
        this->setRotation(cfg->rotation != 0);
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
            wall->setSpecies(this->speciesHandler.getObject(x.species));
            wall->setOrientation(Quaternion(x.orientation[0], x.orientation[1], x.orientation[2], x.orientation[3]));
            wall->setPosition(Vec3D(x.position[0], x.position[1], x.position[2]));
            wall->setVelocity(Vec3D(x.velocity[0], x.velocity[1], x.velocity[2]));
            wall->setAngularVelocity(Vec3D(x.angular_velocity[0], x.angular_velocity[1], x.angular_velocity[2]));
            this->wallHandler.copyAndAddObject(*wall);
            delete wall;
        }
        for (int k = 0; k < 3; ++k) {
            if (!((inst->periodic_mask >> k) & 1u)) continue;
            PeriodicBoundary b;
            Vec3D n(k == 0, k == 1, k == 2);
            b.set(n, inst->periodic_min[k], inst->periodic_max[k]);
            this->boundaryHandler.copyAndAddObject(b);
        }
        for (const auto& db : g_deletions) {
            DeletionBoundary b;
            b.set(Vec3D(db.normal[0], db.normal[1], db.normal[2]), db.distance);
            this->boundaryHandler.copyAndAddObject(b);
        }
        if (!g_insertions.empty()) this->random.setRandomSeed(g_insertion_seed);
        for (const auto& ib : g_insertions) {
            // the engine's PSD table is the reference's own setDistributionUniform
            // here; a 50-point table of one radius is left to generateParticle's
            // default (InsertionBoundary.cc:119-124)
            CubeInsertionBoundary cube;
            ChuteInsertionBoundary chute;
            InsertionBoundary& b = ib.kind == DEM_INSERTION_CHUTE ? static_cast<InsertionBoundary&>(chute)
                                                                  : static_cast<InsertionBoundary&>(cube);
            SphericalParticle tmpl;
            tmpl.setSpecies(this->speciesHandler.getObject(ib.species));
            tmpl.setRadius(ib.psd_radius[0]);
            const Vec3D lo(ib.pos_min[0], ib.pos_min[1], ib.pos_min[2]), hi(ib.pos_max[0], ib.pos_max[1], ib.pos_max[2]);
            if (ib.kind == DEM_INSERTION_CHUTE)
                chute.set(&tmpl, (unsigned)ib.max_failed, lo, hi, ib.fixed_particle_radius, ib.inflow_velocity,
                          ib.inflow_velocity_variance);
            else
                cube.set(&tmpl, (unsigned)ib.max_failed, lo, hi, Vec3D(ib.vel_min[0], ib.vel_min[1], ib.vel_min[2]),
                         Vec3D(ib.vel_max[0], ib.vel_max[1], ib.vel_max[2]));
            const bool default_psd = ib.n_psd == 50 && ib.psd_radius[0] == ib.psd_radius[49] && ib.psd_seed == 0;
            if (!default_psd) {
                PSD psd;
                psd.setDistributionUniform(ib.psd_radius[0], ib.psd_radius[ib.n_psd - 1], ib.n_psd);
                psd.setFixedSeed((int)ib.psd_seed);
                b.setPSD(psd);
            }
            // setInitialVolume zeroes an infinite flow rate: the rate is set after it
            b.setInitialVolume(ib.initial_volume);
            b.setVolumeFlowRate(ib.volume_flow_rate);
            if (ib.kind == DEM_INSERTION_CHUTE)
                this->boundaryHandler.copyAndAddObject(chute);
            else
                this->boundaryHandler.copyAndAddObject(cube);
        }
        SphericalParticle p;
        for (int64_t i = 0; i < in->n; ++i) {
            if (free_rows_in_use() && in->radius[i] == 0.0) continue; // a free row of the engine
            p.setSpecies(this->speciesHandler.getObject(in->species[i]));
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
            BaseParticle* q = this->particleHandler.copyAndAddObject(p);
            if (in->inv_mass[i] == 0.0) q->fixParticle();
        }
    }
};

// The insertion boundaries' counters after a run (g_inserted, g_inserted_volume).
template <class Driver>
void collect_insertions(Driver& d)
{
    g_inserted.clear();
    g_inserted_volume.clear();
    for (BaseBoundary* b : d.boundaryHandler)
        if (auto* ib = dynamic_cast<InsertionBoundary*>(b)) {
            g_inserted.push_back(ib->getNumberOfParticlesInserted());
            g_inserted_volume.push_back(ib->getVolumeOfParticlesInserted());
        }
}

template <class Driver>
void setup(Driver& d, const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
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
