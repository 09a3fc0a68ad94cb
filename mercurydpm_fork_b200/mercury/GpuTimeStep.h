// GpuTimeStep.h -- MercuryDPM drivers whose time steps run on the B200 engine.
//
// A driver that derives from Mercury3D (Mercury2D, DPMBase) derives from
// GpuMercury3D (GpuMercury2D, GpuDPMBase) instead and changes nothing else: DPMBase::solve() runs as
// before (Kernel/DPMBase.cc:4279-4297) -- initialiseSolve with the driver's
// setupInitialConditions on the host, the loop of
// DPMBase::computeOneTimeStep (DPMBase.cc:4315-4389) with every user hook,
// output check, time and step counter of the reference, then finaliseSolve.
// What changes is the work inside the step: the virtual members that the
// reference's computeOneTimeStep calls for it are overridden here
// (the plug points of Kernel/DPMBase.h:1045-1204):
//
//   computeAllForces          the first call (inside initialiseSolve, after
//                             computeAllMasses) hands species, walls,
//                             periodic boundaries and particles to the engine
//                             (dem_create ... dem_upload_particles) and runs
//                             its initial force evaluation (dem_step(h, 0));
//                             every later call is one whole time step on the
//                             device (dem_step(h, 1): half-kick, drift, walls,
//                             forces, second half-kick)
//   integrateBefore/AfterForceComputation, hGridActionsBeforeIntegration /
//   AfterIntegration, checkInteractionWithBoundaries
//                             nothing: the engine integrates, keeps its own
//                             neighbour grid and wraps periodic positions
//   hGridActionsBeforeTimeLoop  ends the engine of a previous solve(), then
//                             the base's own set-up
//   hGridActionsBeforeTimeStep  the base's own grid in initialiseSolve and
//                             the first step (restart files describe it),
//                             nothing afterwards
//   writeEneTimeStep          the reference's .ene line (DPMBase.cc:2100-2123)
//                             from the engine's balances (dem_reduce)
//
// The host's ParticleHandler is refreshed from the device (positions,
// velocities, angular velocities, orientations, forces and torques) after
// every gpuSyncInterval()-th step (default 1: every step), before a step at
// which an output file is due, and after the last step before timeMax, so
// that hooks, the .data writer and the caller read the engine's state.
// Hooks that run between computeAllForces and integrateAfterForceComputation
// in the reference (actionsAfterTimeStep) see the state after the whole step
// (velocities after the second half-kick). At the same refreshes the
// InteractionHandler is rebuilt from the engine's contacts of the last step
// (dem_download_contacts, dem_download_contact_geometry): one interaction of
// the pair's mixed species per contact with its force, contact point,
// normal, overlap, distance and springs, so that hooks and the reference's
// writers (getElasticEnergy, .fstat, .restart) see them. Between refreshes it
// holds the last refresh's contacts. The refresh interval defaults to 1, or
// to the value of the environment variable MERCURYDPM_GPU_SYNC_INTERVAL (for
// drivers that read the state only every k steps and are built unmodified).
//
// Between time steps a driver may take walls out (WallHandler::removeObject)
// and add DeletionBoundary objects (BoundaryHandler::copyAndAddObject), as
// Drivers/Calibration/CalibrationHeap.cpp does in its actionsAfterTimeStep:
// the next computeAllForces hands the change to the engine (dem_remove_wall,
// dem_set_deletion_boundaries). Particles the engine deletes leave the
// ParticleHandler at the next refresh of the host copy.
//
// Supported set-ups: spherical particles; species whose normal law is
// LinearViscoelastic or HertzianViscoelastic and whose friction law is none,
// SlidingFriction, Friction (rolling and torsion), Mindlin or
// MindlinRollingTorsion, with mixed species (a ReversibleAdhesive part is
// accepted when its maximum adhesive force is 0, where it exerts none);
// InfiniteWall, IntersectionOfWalls, AxisymmetricIntersectionOfWalls and
// TriangleWall; PeriodicBoundary and DeletionBoundary. Anything else (other
// walls and boundaries, particles or walls added during the run) stops the
// run with logger(ERROR).
//
// Build: compile the driver against the MercuryDPM Kernel as usual, with
// -I<this repository>/include -I<this directory>, and link
// mercurydpm_fork_b200/libdem_b200.so.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "Boundaries/DeletionBoundary.h"
#include "Boundaries/PeriodicBoundary.h"
#include "DPMBase.h"
#include "Logger.h"
#include "Mercury2D.h"
#include "Mercury3D.h"
#include "Particles/BaseParticle.h"
#include "Species/FrictionForceSpecies/FrictionSpecies.h"
#include "Species/FrictionForceSpecies/MindlinRollingTorsionSpecies.h"
#include "Species/FrictionForceSpecies/MindlinSpecies.h"
#include "Species/AdhesiveForceSpecies/ReversibleAdhesiveSpecies.h"
#include "Interactions/FrictionForceInteractions/FrictionInteraction.h"
#include "Interactions/FrictionForceInteractions/MindlinRollingTorsionInteraction.h"
#include "Interactions/FrictionForceInteractions/SlidingFrictionInteraction.h"
#include "Species/FrictionForceSpecies/SlidingFrictionSpecies.h"
#include "Species/NormalForceSpecies/HertzianViscoelasticNormalSpecies.h"
#include "Species/NormalForceSpecies/LinearViscoelasticNormalSpecies.h"
#include "Walls/AxisymmetricIntersectionOfWalls.h"
#include "Walls/InfiniteWall.h"
#include "Walls/IntersectionOfWalls.h"
#include "Walls/TriangleWall.h"

#include "dem_b200.h"

template <class Base>
class GpuTimeStep : public Base
{
public:
    ~GpuTimeStep() override
    {
        if (h_) dem_destroy(h_);
    }

    /// CUDA device ordinal of the engine (before solve()).
    void setGpuDevice(int device) { device_ = device; }

    /// The host copy of the particles is refreshed after every k-th time step
    /// (and whenever an output is due or the run ends); k = 1 refreshes it
    /// after every step.
    void setGpuSyncInterval(unsigned k) { syncInterval_ = k ? k : 1; }
    unsigned gpuSyncInterval() const { return syncInterval_; }

    /// Copies the device state into the ParticleHandler now.
    void gpuSync()
    {
        if (!h_) return;
        const size_t n = real_.size();
        dem_particles_soa s{(int64_t)n, x_.data(), v_.data(), w_.data(), q_.data(), nullptr, nullptr, nullptr,
                            nullptr, nullptr, inst_.data()};
        check(dem_download_particles(h_, &s), "dem_download_particles");
        check(dem_download_forces(h_, f_.data(), t_.data()), "dem_download_forces");
        for (size_t i = 0; i < n; ++i) {
            BaseParticle* p = real_[i];
            if (!p) continue;
            if (inst_[i] < 0) { // deleted by a DeletionBoundary on the device
                const unsigned id = p->getId();
                if (id < byId_.size()) byId_[id] = nullptr;
                this->particleHandler.removeObject(p->getIndex());
                real_[i] = nullptr;
                --live_;
                continue;
            }
            p->setPosition(Vec3D(x_[3 * i], x_[3 * i + 1], x_[3 * i + 2]));
            p->setVelocity(Vec3D(v_[3 * i], v_[3 * i + 1], v_[3 * i + 2]));
            p->setAngularVelocity(Vec3D(w_[3 * i], w_[3 * i + 1], w_[3 * i + 2]));
            p->setOrientation(Quaternion(q_[4 * i], q_[4 * i + 1], q_[4 * i + 2], q_[4 * i + 3]));
            p->setForce(Vec3D(f_[3 * i], f_[3 * i + 1], f_[3 * i + 2]));
            p->setTorque(Vec3D(t_[3 * i], t_[3 * i + 1], t_[3 * i + 2]));
        }
        sinceSync_ = 0;
        mirrorInteractions();
    }

    /// The engine's handle (after the first force evaluation), for the rest of
    /// the C ABI: contacts, coarse-graining, timing.
    dem_handle* gpuHandle() const { return h_; }

protected:
    void computeAllForces() override
    {
        if (!h_) {
            upload();
            check(dem_step(h_, 0), "dem_step"); // the initial evaluation of initialiseSolve
            gpuSync();
            return;
        }
        if (countReal() != live_)
            logger(ERROR, "GpuTimeStep: particles were added or removed during the run (not supported)");
        handOverChanges();
        check(dem_step(h_, 1), "dem_step");
        ++sinceSync_;
        // this step's time and counter are advanced after computeAllForces
        const unsigned next = this->getNumberOfTimeSteps() + 1;
        const bool last = !(this->getTime() + this->getTimeStep() < this->getTimeMax());
        if (sinceSync_ >= syncInterval_ || last || outputDue(next)) gpuSync();
    }

    void integrateBeforeForceComputation() override {}
    void integrateAfterForceComputation() override {}
    /// Called once by every initialiseSolve, before its force evaluation: a
    /// driver that calls solve() again (with changed species, particles or
    /// walls) starts a new engine at the next computeAllForces. The base's
    /// own set-up (Mercury3D's HGrid cell sizes) still runs once, so restart
    /// files print the same grid description as the reference's.
    void hGridActionsBeforeTimeLoop() override
    {
        if (h_) dem_destroy(h_);
        h_ = nullptr;
        baseGridCalls_ = 0;
        Base::hGridActionsBeforeTimeLoop();
    }
    /// The base's own grid runs in initialiseSolve (Mercury3D / Mercury2D size
    /// their cells there) and in the first time step (its first update resets
    /// the displacement bookkeeping), so that restart files describe it as the
    /// reference's do; later steps use the engine's grid only.
    void hGridActionsBeforeTimeStep() override
    {
        if (baseGridCalls_ < 2) {
            Base::hGridActionsBeforeTimeStep();
            ++baseGridCalls_;
        }
    }
    void hGridActionsBeforeIntegration() override {}
    void hGridActionsAfterIntegration() override {}
    void checkInteractionWithBoundaries() override {}

    /// DPMBase::writeEneTimeStep (DPMBase.cc:2100-2123) with the balances of
    /// the engine: time, -g . sum(m x), translational and rotational kinetic
    /// energy, elastic energy, centre of mass, number of interactions.
    void writeEneTimeStep(std::ostream& os) const override
    {
        if (!h_) {
            Base::writeEneTimeStep(os);
            return;
        }
        if (this->eneFile.getCounter() == 1 || this->eneFile.getFileType() == FileType::MULTIPLE_FILES ||
            this->eneFile.getFileType() == FileType::MULTIPLE_FILES_PADDED)
            this->writeEneHeader(os);
        dem_globals g{};
        if (dem_reduce(h_, 0, &g) != DEM_OK) logger(ERROR, "GpuTimeStep: dem_reduce: %", dem_last_error(h_));
        const Vec3D com(g.centre_of_mass[0], g.centre_of_mass[1], g.centre_of_mass[2]);
        const Vec3D mx = g.mass * com;
        const int width = (int)os.precision() + 6;
        os << std::setw(width) << this->getTime() << " " << std::setw(width) << -Vec3D::dot(this->getGravity(), mx)
           << " " << std::setw(width) << g.kinetic_energy << " " << std::setw(width) << g.rotational_energy << " "
           << std::setw(width) << g.elastic_energy << " " << std::setw(width)
           << (g.mass == 0 ? constants::NaN : com.X) << " " << std::setw(width)
           << (g.mass == 0 ? constants::NaN : com.Y) << " " << std::setw(width)
           << (g.mass == 0 ? constants::NaN : com.Z) << " " << std::setw(width)
           << (g.n_contacts + g.n_wall_contacts) << std::endl;
    }

private:
    dem_handle* h_ = nullptr;
    int device_ = 0;
    unsigned syncInterval_ = defaultSyncInterval();
    int baseGridCalls_ = 0;
    unsigned sinceSync_ = 0;
    std::vector<BaseParticle*> real_;  // engine order; nullptr once deleted
    size_t live_ = 0;
    std::vector<double> x_, v_, w_, q_, f_, t_;
    std::vector<int32_t> inst_;
    std::vector<BaseWall*> walls_;        // dem_set_walls order; nullptr once taken out
    std::vector<BaseParticle*> byId_;     // particle of each id (nullptr: none, or deleted)

    static unsigned defaultSyncInterval()
    {
        const char* e = std::getenv("MERCURYDPM_GPU_SYNC_INTERVAL");
        const long k = e ? std::strtol(e, nullptr, 10) : 1;
        return k > 0 ? (unsigned)k : 1u;
    }

    // The engine's contacts of the last time step as the InteractionHandler's
    // interactions (InteractionHandler::getInteraction creates each with the
    // pair's mixed species, as the reference's contact detection does).
    void mirrorInteractions()
    {
        int64_t count = 0;
        check(dem_download_contacts(h_, nullptr, 0, &count), "dem_download_contacts");
        std::vector<int32_t> ip(count), ii(count), iw(count), per(count);
        std::vector<double> spr(9 * count), f(3 * count), ov(count), cp(3 * count), nr(3 * count);
        dem_contacts_soa c{count, ip.data(), ii.data(), iw.data(), per.data(), spr.data(), f.data(), ov.data()};
        check(dem_download_contacts(h_, &c, count, &count), "dem_download_contacts");
        check(dem_download_contact_geometry(h_, cp.data(), nr.data(), nullptr, count, &count),
              "dem_download_contact_geometry");
        this->interactionHandler.clear();
        const unsigned stamp = this->getNumberOfTimeSteps() + 1;
        for (int64_t r = 0; r < count; ++r) {
            BaseParticle* P = (ip[r] >= 0 && ip[r] < (int)byId_.size()) ? byId_[ip[r]] : nullptr;
            BaseInteractable* I = nullptr;
            if (iw[r]) {
                if (ii[r] >= 0 && ii[r] < (int)walls_.size()) I = walls_[ii[r]];
            } else if (ii[r] >= 0 && ii[r] < (int)byId_.size()) {
                I = byId_[ii[r]];
            }
            if (!P || !I) continue;
            BaseInteraction* x = this->interactionHandler.getInteraction(P, I, stamp);
            x->setForce(Vec3D(f[3 * r], f[3 * r + 1], f[3 * r + 2]));
            x->setContactPoint(Vec3D(cp[3 * r], cp[3 * r + 1], cp[3 * r + 2]));
            x->setNormal(Vec3D(nr[3 * r], nr[3 * r + 1], nr[3 * r + 2]));
            x->setOverlap(ov[r]);
            const double reach = P->getRadius() + (iw[r] ? 0.0 : static_cast<BaseParticle*>(I)->getRadius());
            x->setDistance(reach - ov[r]);
            const double* sp = &spr[9 * r];
            if (auto* sf = dynamic_cast<SlidingFrictionInteraction*>(x)) sf->setSlidingSpring(Vec3D(sp[0], sp[1], sp[2]));
            if (auto* fr = dynamic_cast<FrictionInteraction*>(x)) {
                fr->setRollingSpring(Vec3D(sp[3], sp[4], sp[5]));
                fr->setTorsionSpring(Vec3D(sp[6], sp[7], sp[8]));
            }
            if (auto* mr = dynamic_cast<MindlinRollingTorsionInteraction*>(x)) {
                mr->setRollingSpring(Vec3D(sp[3], sp[4], sp[5]));
                mr->setTorsionSpring(Vec3D(sp[6], sp[7], sp[8]));
            }
        }
    }
    std::vector<const BaseBoundary*> deletions_;

    // Walls taken out and DeletionBoundary objects added since the last step
    // go to the engine before the next one.
    void handOverChanges()
    {
        if (this->wallHandler.getSize() != countWalls()) {
            std::vector<const BaseWall*> now(this->wallHandler.begin(), this->wallHandler.end());
            for (const BaseWall* w : now)
                if (std::find(walls_.begin(), walls_.end(), w) == walls_.end())
                    logger(ERROR, "GpuTimeStep: walls were added during the run (not supported)");
            for (size_t k = 0; k < walls_.size(); ++k)
                if (walls_[k] && std::find(now.begin(), now.end(), walls_[k]) == now.end()) {
                    check(dem_remove_wall(h_, (int)k), "dem_remove_wall");
                    walls_[k] = nullptr;
                }
        }
        std::vector<const BaseBoundary*> dels;
        for (BaseBoundary* b : this->boundaryHandler)
            if (dynamic_cast<DeletionBoundary*>(b)) dels.push_back(b);
        if (dels != deletions_) {
            std::vector<dem_deletion_boundary> planes;
            for (BaseBoundary* b : this->boundaryHandler) {
                if (dynamic_cast<DeletionBoundary*>(b))
                    planes.push_back(deletionPlane(b));
                else if (!dynamic_cast<PeriodicBoundary*>(b))
                    logger(ERROR, "GpuTimeStep: boundary % is not supported", b->getName());
            }
            check(dem_set_deletion_boundaries(h_, planes.data(), (int)planes.size()), "dem_set_deletion_boundaries");
            deletions_ = dels;
        }
    }

    size_t countWalls() const
    {
        size_t n = 0;
        for (const BaseWall* w : walls_)
            if (w) ++n;
        return n;
    }

    // DeletionBoundary::set keeps the unit normal and the scaled distance; its
    // restart line carries both (DeletionBoundary::write)
    static dem_deletion_boundary deletionPlane(const BaseBoundary* b)
    {
        dem_deletion_boundary d{};
        std::ostringstream os;
        os.precision(17);
        b->write(os);
        std::istringstream is(os.str());
        std::string tok;
        while (is >> tok) {
            if (tok == "normal") is >> d.normal[0] >> d.normal[1] >> d.normal[2];
            if (tok == "distance") is >> d.distance;
        }
        return d;
    }

    // The faces of an IntersectionOfWalls (AxisymmetricIntersectionOfWalls:
    // in its (r, 0, a) frame): normal and point of each of its InfiniteWalls,
    // read from the wall's restart line (IntersectionOfWalls::write) and the
    // normal taken from the face's orientation as the face itself does
    static void fillFaces(const BaseWall* w, dem_wall& d)
    {
        std::ostringstream os;
        os.precision(17);
        w->write(os);
        std::istringstream is(os.str());
        std::string tok;
        while (is >> tok && tok != "numIntersectionOfWalls") {
        }
        unsigned n = 0;
        is >> n;
        if (n > DEM_MAX_WALL_FACES) logger(ERROR, "GpuTimeStep: wall % has more than % faces", w->getIndex(), DEM_MAX_WALL_FACES);
        d.n_faces = (int)n;
        for (unsigned f = 0; f < n; ++f) {
            Vec3D p;
            double q[4];
            is >> tok >> p.X >> p.Y >> p.Z >> tok >> q[0] >> q[1] >> q[2] >> q[3];
            InfiniteWall face;
            face.setOrientation(Quaternion(q[0], q[1], q[2], q[3]));
            copy3(d.faces[f], face.getNormal());
            copy3(d.faces[f] + 3, p);
        }
    }

    void check(int rc, const char* what) const
    {
        if (rc != DEM_OK) logger(ERROR, "GpuTimeStep: % failed (status %): %", what, rc, dem_last_error(h_));
    }

    static bool isReal(const BaseParticle* p)
    {
        return !p->isPeriodicGhostParticle() && !p->isMPIParticle();
    }

    size_t countReal() const
    {
        size_t n = 0;
        for (const BaseParticle* p : this->particleHandler)
            if (isReal(p)) ++n;
        return n;
    }

    static bool due(const File& f, unsigned step)
    {
        if (f.getFileType() == FileType::NO_FILE) return false;
        return f.getLastSavedTimeStep() == NEVER || step >= f.getLastSavedTimeStep() + f.getSaveCount();
    }

    // DPMBase::writeOutputFiles writes these at the start of a step
    bool outputDue(unsigned step) const
    {
        return due(this->dataFile, step) || due(this->fStatFile, step) || due(this->restartFile, step) ||
               due(this->eneFile, step);
    }

    static void fillSpecies(BaseSpecies* s, dem_species_pair& p)
    {
        if (auto* n = dynamic_cast<LinearViscoelasticNormalSpecies*>(s)) {
            p.normal_law = DEM_NORMAL_LINEAR_VISCOELASTIC;
            p.stiffness = n->getStiffness();
            p.dissipation = n->getDissipation();
            p.constant_restitution = n->getConstantRestitution() ? 1 : 0;
        } else if (auto* n = dynamic_cast<HertzianViscoelasticNormalSpecies*>(s)) {
            p.normal_law = DEM_NORMAL_HERTZIAN_VISCOELASTIC;
            p.elastic_modulus = n->getEffectiveElasticModulus();
            p.dissipation = n->getDissipation();
        } else {
            logger(ERROR, "GpuTimeStep: species % has a normal force law the engine does not have", s->getName());
        }
        p.friction_law = DEM_FRICTION_NONE;
        if (auto* f = dynamic_cast<MindlinRollingTorsionSpecies*>(s)) {
            p.friction_law = DEM_FRICTION_MINDLIN_ROLLING_TORSION;
            p.rolling_dissipation = f->getRollingDissipation();
            p.rolling_mu = f->getRollingFrictionCoefficient();
            p.rolling_mu_static = f->getRollingFrictionCoefficientStatic();
            p.torsion_dissipation = f->getTorsionDissipation();
            p.torsion_mu = f->getTorsionFrictionCoefficient();
            p.torsion_mu_static = f->getTorsionFrictionCoefficientStatic();
        } else if (dynamic_cast<MindlinSpecies*>(s)) {
            p.friction_law = DEM_FRICTION_MINDLIN;
        } else if (auto* f = dynamic_cast<FrictionSpecies*>(s)) {
            p.friction_law = DEM_FRICTION_ROLLING_TORSION;
            p.rolling_stiffness = f->getRollingStiffness();
            p.rolling_dissipation = f->getRollingDissipation();
            p.rolling_mu = f->getRollingFrictionCoefficient();
            p.rolling_mu_static = f->getRollingFrictionCoefficientStatic();
            p.torsion_stiffness = f->getTorsionStiffness();
            p.torsion_dissipation = f->getTorsionDissipation();
            p.torsion_mu = f->getTorsionFrictionCoefficient();
            p.torsion_mu_static = f->getTorsionFrictionCoefficientStatic();
        } else if (!dynamic_cast<SlidingFrictionSpecies*>(s) && s->getName().find("Friction") != std::string::npos) {
            logger(ERROR, "GpuTimeStep: species % has a friction law the engine does not have", s->getName());
        }
        if (auto* f = dynamic_cast<MindlinSpecies*>(s)) {
            p.shear_modulus = f->getEffectiveShearModulus();
            p.sliding_dissipation = f->getSlidingDissipation();
            p.sliding_mu = f->getSlidingFrictionCoefficient();
            p.sliding_mu_static = f->getSlidingFrictionCoefficientStatic();
        } else if (auto* f = dynamic_cast<SlidingFrictionSpecies*>(s)) {
            if (p.friction_law == DEM_FRICTION_NONE) p.friction_law = DEM_FRICTION_SLIDING;
            p.sliding_stiffness = f->getSlidingStiffness();
            p.sliding_dissipation = f->getSlidingDissipation();
            p.sliding_mu = f->getSlidingFrictionCoefficient();
            p.sliding_mu_static = f->getSlidingFrictionCoefficientStatic();
        }
        if (auto* a = dynamic_cast<ReversibleAdhesiveSpecies*>(s))
            if (a->getAdhesionForceMax() != 0)
                logger(ERROR, "GpuTimeStep: species % has an adhesive force the engine does not have", s->getName());
        p.interaction_distance = s->getInteractionDistance();
    }

    static void copy3(double* dst, const Vec3D& v)
    {
        dst[0] = v.X;
        dst[1] = v.Y;
        dst[2] = v.Z;
    }

    void upload()
    {
        dem_config cfg{};
        cfg.time_step = this->getTimeStep();
        cfg.background_drag = this->getBackgroundDrag();
        cfg.rotation = this->getRotation() ? 1 : 0;
        cfg.device = device_;
        cfg.use_graphs = 1;
        cfg.n_instances = 1;
        dem_instance_desc in{};
        copy3(in.domain_min, this->getMin());
        copy3(in.domain_max, this->getMax());
        copy3(in.gravity, this->getGravity());
        // the domain only lays out the engine's cell grid (particles outside it
        // are kept in its border cells): a flat dimension (Mercury2D, or a
        // domain thinner than a few particles) is widened by two radii each side
        double rmax = 0.0;
        for (const BaseParticle* p : this->particleHandler)
            if (p->getRadius() > rmax) rmax = p->getRadius();
        for (int k = 0; k < 3; ++k)
            if (in.domain_max[k] - in.domain_min[k] < 4.0 * rmax) {
                in.domain_min[k] -= 2.0 * rmax;
                in.domain_max[k] += 2.0 * rmax;
            }
        const unsigned ns = this->speciesHandler.getSize();
        in.n_species = (int)ns;
        std::vector<dem_deletion_boundary> planes;
        deletions_.clear();
        for (BaseBoundary* b : this->boundaryHandler) {
            if (dynamic_cast<DeletionBoundary*>(b)) {
                planes.push_back(deletionPlane(b));
                deletions_.push_back(b);
                continue;
            }
            auto* pb = dynamic_cast<PeriodicBoundary*>(b);
            if (!pb) logger(ERROR, "GpuTimeStep: boundary % is not supported", b->getName());
            const Vec3D nrm = pb->getNormal();
            const int k = nrm.X != 0 ? 0 : (nrm.Y != 0 ? 1 : 2);
            if ((k == 0 && (nrm.Y != 0 || nrm.Z != 0)) || (k == 1 && nrm.Z != 0))
                logger(ERROR, "GpuTimeStep: periodic boundaries must be normal to a coordinate axis");
            // PeriodicBoundary::set stores a unit normal (+-1 along axis k) and
            // the planes x . normal = distanceLeft / distanceRight
            const double c = nrm.getComponent(k);
            const double a = pb->getDistanceLeft() * c, b2 = pb->getDistanceRight() * c;
            in.periodic_mask |= 1u << k;
            in.periodic_min[k] = a < b2 ? a : b2;
            in.periodic_max[k] = a < b2 ? b2 : a;
        }
        check(dem_create(&cfg, &in, &h_), "dem_create");
        std::vector<dem_species_pair> table((size_t)ns * ns);
        for (unsigned a = 0; a < ns; ++a)
            for (unsigned b = 0; b < ns; ++b) {
                BaseSpecies* s = a == b ? static_cast<BaseSpecies*>(this->speciesHandler.getObject(a))
                                        : this->speciesHandler.getMixedObject(a, b);
                dem_species_pair p{};
                fillSpecies(s, p);
                table[(size_t)a * ns + b] = p;
            }
        check(dem_set_species(h_, table.data(), (int)table.size()), "dem_set_species");
        std::vector<dem_wall> walls;
        walls_.clear();
        for (BaseWall* w : this->wallHandler) {
            dem_wall d{};
            d.species = (int)w->getIndSpecies();
            const Quaternion q = w->getOrientation();
            for (int k = 0; k < 4; ++k) d.orientation[k] = q.getComponent(k);
            copy3(d.position, w->getPosition());
            copy3(d.velocity, w->getVelocity());
            copy3(d.angular_velocity, w->getAngularVelocity());
            if (dynamic_cast<AxisymmetricIntersectionOfWalls*>(w)) {
                d.type = DEM_WALL_AXISYMMETRIC;
                fillFaces(w, d);
            } else if (dynamic_cast<IntersectionOfWalls*>(w)) {
                d.type = DEM_WALL_INTERSECTION;
                fillFaces(w, d);
            } else if (dynamic_cast<InfiniteWall*>(w)) {
                d.type = DEM_WALL_INFINITE;
            } else if (auto* tw = dynamic_cast<TriangleWall*>(w)) {
                d.type = DEM_WALL_TRIANGLE;
                d.n_faces = 3;
                d.group = (int)tw->getGroupId();
                for (int v = 0; v < 3; ++v) copy3(d.faces[v], tw->getVertex(v));
            } else {
                logger(ERROR, "GpuTimeStep: wall % is not supported", w->getName());
            }
            walls.push_back(d);
            walls_.push_back(w);
        }
        check(dem_set_walls(h_, walls.data(), (int)walls.size()), "dem_set_walls");
        check(dem_set_deletion_boundaries(h_, planes.data(), (int)planes.size()), "dem_set_deletion_boundaries");
        real_.clear();
        for (BaseParticle* p : this->particleHandler)
            if (isReal(p)) real_.push_back(p);
        const size_t n = real_.size();
        live_ = n;
        byId_.clear();
        for (BaseParticle* p : real_) {
            if (p->getId() >= byId_.size()) byId_.resize(p->getId() + 1, nullptr);
            byId_[p->getId()] = p;
        }
        inst_.assign(n, 0);
        x_.assign(3 * n, 0.0); v_.assign(3 * n, 0.0); w_.assign(3 * n, 0.0); q_.assign(4 * n, 0.0);
        f_.assign(3 * n, 0.0); t_.assign(3 * n, 0.0);
        std::vector<double> r(n), im(n), ii(n);
        std::vector<int32_t> sp(n), id(n);
        for (size_t i = 0; i < n; ++i) {
            const BaseParticle* p = real_[i];
            copy3(&x_[3 * i], p->getPosition());
            copy3(&v_[3 * i], p->getVelocity());
            copy3(&w_[3 * i], p->getAngularVelocity());
            for (int k = 0; k < 4; ++k) q_[4 * i + k] = p->getOrientation().getComponent(k);
            r[i] = p->getRadius();
            im[i] = p->getInvMass();
            ii[i] = p->getInvInertia().XX;
            sp[i] = (int32_t)p->getIndSpecies();
            id[i] = (int32_t)p->getId();
        }
        dem_particles_soa s{(int64_t)n, x_.data(), v_.data(), w_.data(), q_.data(), r.data(), im.data(), ii.data(),
                            sp.data(), id.data(), nullptr};
        check(dem_upload_particles(h_, &s), "dem_upload_particles");
    }
};

using GpuDPMBase = GpuTimeStep<DPMBase>;
using GpuMercury2D = GpuTimeStep<Mercury2D>;
using GpuMercury3D = GpuTimeStep<Mercury3D>;
