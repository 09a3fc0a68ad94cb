// gpu_binding_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The checker's reference-API driver (ref_driver.h) on the engine's drop-in
// base class: RefDriverT<GpuMercury3D> is the same Mercury3D subclass that
// oracle/ref_drivers/mdpm_ref_driver.cpp runs on the reference's Mercury3D,
// with only its base class changed. Built by oracle/ref.mk (target gpu) into
// oracle/_ref/libmdpm_gpu_binding.so.
#include "GpuTimeStep.h"
#include "ref_driver.h"

namespace {
using GpuRefDriver = RefDriverT<GpuMercury3D>;
} // namespace

extern "C" {

// mdpm_ref_solve_ene with the drop-in base class: DPMBase::solve() over
// `nsteps` time steps with the .ene file as the only output (prefix.ene, a
// line every `save_count` steps and one at the end), the steps on CUDA
// device `device`; the host copy of the particles is refreshed every
// `sync_interval` steps.
int mdpm_gpu_solve_ene(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                       const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                       int nsteps, int save_count, int device, int sync_interval, const char* prefix)
{
    GpuRefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.setGpuDevice(device);
    d.setGpuSyncInterval((unsigned)sync_interval);
    d.setTimeMax((nsteps - 0.5) * cfg->time_step);
    d.solve_writing_ene(prefix, (unsigned)save_count);
    return 0;
}

// The same run, returning the final particle state the host holds after
// solve() (caller order = upload order; position 3n, velocity 3n,
// angular_velocity 3n).
// the between-steps change of the next mdpm_gpu_solve_state (step < 0: none),
// made by the driver's actionsAfterTimeStep as a MercuryDPM driver makes it
void mdpm_gpu_set_event(long long step, int wall, const dem_deletion_boundary* b, int n)
{
    g_event_step = step;
    g_event_wall = wall;
    g_event_deletions.assign(b, b + n);
}

int mdpm_gpu_solve_state(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species,
                         const double* density, const dem_wall* walls, int nwalls, const dem_particles_soa* in,
                         int nsteps, int device, int sync_interval, dem_particles_soa* out, double* host)
{
    GpuRefDriver d;
    setup(d, cfg, inst, species, density, walls, nwalls, in, 1);
    d.setGpuDevice(device);
    d.setGpuSyncInterval((unsigned)sync_interval);
    d.setTimeMax((nsteps - 0.5) * cfg->time_step);
    d.after_step = [&d]() { apply_event(d, (long long)d.getNumberOfTimeSteps() + 1); };
    d.solve_writing_ene("/dev/null", 1u << 30);
    if (host) { // what the driver's InteractionHandler holds: elastic energy, interactions
        host[0] = d.getElasticEnergy();
        host[1] = (double)d.interactionHandler.getNumberOfObjects();
    }
    if (out->instance)
        for (int64_t i = 0; i < in->n; ++i) out->instance[i] = -1; // deleted particles left the handler
    for (int64_t r = 0; r < (int64_t)d.particleHandler.getSize(); ++r) {
        const BaseParticle* p = d.particleHandler.getObject((unsigned)r);
        const int64_t i = (int64_t)p->getId();
        if (i < 0 || i >= in->n) continue;
        if (out->instance) out->instance[i] = 0;
        const Vec3D x = p->getPosition(), v = p->getVelocity(), w = p->getAngularVelocity();
        for (int k = 0; k < 3; ++k) {
            out->position[3 * i + k] = x.getComponent(k);
            out->velocity[3 * i + k] = v.getComponent(k);
            out->angular_velocity[3 * i + k] = w.getComponent(k);
        }
    }
    return 0;
}

} // extern "C"
