/*
 * dem_b200.h -- C ABI of the B200 DEM time-step engine.
 *
 * The engine replaces the serial force/broad-phase loop of a MercuryDPM
 * driver (DPMBase::computeOneTimeStep, Kernel/DPMBase.cc:4315-4389) with
 * device-resident state and sm_100a kernels. A driver keeps its
 * Mercury3D/DPMBase set-up code (species, particles, walls, periodic
 * boundaries), hands the result to the engine once through this interface,
 * and advances it in batches of time steps.
 *
 * Conventions
 *  - Every entry point returns an int status (DEM_OK == 0); no exceptions
 *    cross the ABI. dem_last_error() gives the message of the last failure.
 *  - The caller owns every host buffer; the engine owns all device memory.
 *  - One host thread per handle. Calls on one handle are serialised on the
 *    handle's own CUDA stream.
 *  - Arrays are structure-of-arrays, FP64, indexed by the caller's particle
 *    order at upload (the engine reorders internally and restores the
 *    caller's order on download).
 *  - Units and sign conventions are MercuryDPM's: the force stored on a
 *    particle-particle contact acts on the particle with the lower id (P),
 *    its normal points from I to P (Kernel/Particles/BaseParticle.cc:688-710);
 *    for a wall contact P is the particle and the normal is minus the wall's
 *    outward normal (Kernel/Walls/BaseWall.cc:367-437).
 */
#ifndef DEM_B200_H
#define DEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DEM_OK             0
#define DEM_ERR_CAPACITY   1  /* neighbour-list or cell capacity exceeded          */
#define DEM_ERR_TIMEOUT    2  /* a bounded device wait gave up                      */
#define DEM_ERR_NAN        3  /* non-finite force or position detected              */
#define DEM_ERR_BAD_INPUT  4  /* invalid argument (sizes, indices, parameters)      */
#define DEM_ERR_CUDA       5  /* CUDA runtime failure                               */
#define DEM_ERR_STATE      6  /* call out of order (e.g. step before upload)        */
#define DEM_ERR_DOMAIN     7  /* a particle left the instance's bounding box        */

/* ---- contact laws (the Species typedef headers in Kernel/Species) ----- */
#define DEM_NORMAL_LINEAR_VISCOELASTIC   0 /* LinearViscoelasticInteraction.cc:105-135  */
#define DEM_NORMAL_HERTZIAN_VISCOELASTIC 1 /* HertzianViscoelasticInteraction.cc:106-141 */

#define DEM_FRICTION_NONE                0
#define DEM_FRICTION_SLIDING             1 /* SlidingFrictionInteraction.cc:106-193      */
#define DEM_FRICTION_ROLLING_TORSION     2 /* FrictionInteraction.cc:108-232             */
#define DEM_FRICTION_MINDLIN             3 /* MindlinInteraction.cc:279-344              */
#define DEM_FRICTION_MINDLIN_ROLLING_TORSION 4 /* MindlinRollingTorsionInteraction.cc:109-208 */

/* ---- wall types ------------------------------------------------------- */
#define DEM_WALL_INFINITE        0 /* InfiniteWall.cc:151-175                       */
#define DEM_WALL_AXISYMMETRIC    1 /* AxisymmetricIntersectionOfWalls.cc:93-124     */
#define DEM_WALL_INTERSECTION    2 /* IntersectionOfWalls.cc:532-547, 567-712       */
#define DEM_WALL_TRIANGLE        3 /* TriangleWall.cc:57-104, 218-262 (+ the triangle-wall
                                      correction, DPMBase.cc:3443-3486, BaseWall.cc:375-409) */

#define DEM_MAX_LEVELS      4
#define DEM_MAX_TRIANGLE_CONTACTS 8
#define DEM_MAX_WALL_FACES  8
#define DEM_MAX_WALLS_PER_INSTANCE 32
#define DEM_MAX_DELETION_PER_INSTANCE 2
#define DEM_MAX_INSERTION_PER_INSTANCE 4
#define DEM_MAX_PSD_POINTS 64

/* ---- insertion boundary kinds ----------------------------------------- */
#define DEM_INSERTION_CUBE  0 /* CubeInsertionBoundary::placeParticle (CubeInsertionBoundary.cc:173-184) */
#define DEM_INSERTION_CHUTE 1 /* ChuteInsertionBoundary::placeParticle (ChuteInsertionBoundary.cc:163-190) */

/* Parameters of one (mixed) species pair, as held by the reference's
 * Species<Normal,Friction,Adhesive> objects and the mixed-species triangle
 * (SpeciesHandler::getMixedObject, Kernel/SpeciesHandler.cc:901-937).
 * Values are the ones the reference species getters return, so the device
 * law evaluates the same expressions on the same numbers. */
typedef struct dem_species_pair {
    int32_t normal_law;            /* DEM_NORMAL_*                                   */
    int32_t friction_law;          /* DEM_FRICTION_*                                 */
    int32_t constant_restitution;  /* LinearViscoelasticNormalSpecies constantRestitution */
    int32_t reserved;
    double  stiffness;             /* linear k                                       */
    double  dissipation;           /* linear gamma; Hertz: dimensionless damping     */
    double  elastic_modulus;       /* Hertz effective elastic modulus                */
    double  shear_modulus;         /* Mindlin effective shear modulus                */
    double  sliding_stiffness, sliding_dissipation;
    double  sliding_mu, sliding_mu_static;
    double  rolling_stiffness, rolling_dissipation;
    double  rolling_mu, rolling_mu_static;
    double  torsion_stiffness, torsion_dissipation;
    double  torsion_mu, torsion_mu_static;
    double  interaction_distance;  /* mixed-species interaction distance (0: none)   */
} dem_species_pair;

/* A wall. Every wall keeps the reference's own representation: the
 * orientation quaternion (BaseInteractable::setOrientationViaNormal for an
 * InfiniteWall's normal, AxisymmetricIntersectionOfWalls::setAxis for an
 * axisymmetric wall's axis) and the position.
 *  - DEM_WALL_INFINITE: position is a point on the plane; the distance is
 *    Quaternion::getDistance (Kernel/Math/Quaternion.cc:658-670).
 *  - DEM_WALL_INTERSECTION / DEM_WALL_AXISYMMETRIC: faces[k] =
 *    (normal xyz, point xyz) exactly as passed to
 *    IntersectionOfWalls::addObject(normal, point), in the wall's frame
 *    (IntersectionOfWalls: the frame given by position and orientation;
 *    axisymmetric: (r, 0, a) about the axis through position). The engine
 *    derives the faces' quaternions, edges and corners as the reference does.
 *  - DEM_WALL_TRIANGLE: faces[0..2][0..2] = the vertices A, B, C in lab
 *    coordinates and position = the wall's position, as
 *    TriangleWall::setVertices(A, B, C, position) takes them (setVertices(A, B, C)
 *    is position = (A + B + C) / 3); the engine keeps A - position, B - position,
 *    C - position (vertexInLabFrame_) and rotates them with the orientation.
 *    n_faces is 3. group is BaseObject::groupId: triangles of one group > 0
 *    keep only the contact of larger overlap when their contacts are not both
 *    face contacts (BaseWall::getInteractionWith); a particle with two or more
 *    triangle contacts gets them weighted by overlap (DPMBase::computeAllForces).
 *    At most DEM_MAX_TRIANGLE_CONTACTS triangle contacts per particle.
 * Walls move every time step as BaseInteractable::integrateBeforeForceComputation
 * does without prescribed motion: position += velocity dt, orientation
 * rotated by angular_velocity dt. Wall indices in contacts are indices into
 * the array given to dem_set_walls. */
typedef struct dem_wall {
    int32_t type;                  /* DEM_WALL_*                                     */
    int32_t species;               /* species index of the wall                      */
    int32_t instance;              /* owning instance (0 for a single simulation)    */
    int32_t n_faces;               /* intersection walls: number of faces            */
    int32_t group;                 /* triangle walls: group id (0: none)             */
    int32_t reserved;
    double  position[3];
    double  orientation[4];        /* quaternion q0..q3                              */
    double  velocity[3];
    double  angular_velocity[3];
    double  faces[DEM_MAX_WALL_FACES][6];
} dem_wall;

/* Host-side particle arrays (structure of arrays, caller order).
 * position/velocity/angular_velocity: 3*n doubles, xyz interleaved per particle.
 * orientation: 4*n doubles (q0..q3) or NULL (identity).
 * inv_mass/inv_inertia: 0 for fixed particles (BaseParticle::fixParticle).
 * inv_inertia is the isotropic diagonal of BaseParticle::invInertia_
 * (Kernel/Particles/BaseParticle.cc:874-883). id is the reference's
 * BaseParticle::getId(); it orders each pair (lower id is P). */
typedef struct dem_particles_soa {
    int64_t  n;
    double  *position;
    double  *velocity;
    double  *angular_velocity;
    double  *orientation;
    double  *radius;
    double  *inv_mass;
    double  *inv_inertia;
    int32_t *species;
    int32_t *id;
    int32_t *instance;             /* NULL: all in instance 0                        */
} dem_particles_soa;

/* Contact list with history, one row per live contact, for download,
 * restart and oracle injection (the content of InteractionHandler,
 * Kernel/InteractionHandler.cc:146-174, 433-500).
 * For particle-wall contacts id_i is the wall index and is_wall is 1.
 * springs: 9 doubles per contact: sliding(3), rolling(3), torsion(3).
 * force/contact_point: 3 doubles per contact (may be NULL on upload). */
typedef struct dem_contacts_soa {
    int64_t  n;
    int32_t *id_p;
    int32_t *id_i;
    int32_t *is_wall;
    int32_t *periodic;             /* 1: the pair meets across a periodic boundary   */
    double  *springs;
    double  *force;
    double  *overlap;
} dem_contacts_soa;

/* Per-instance description. A single simulation is one instance. */
typedef struct dem_instance_desc {
    double   domain_min[3];        /* bounding box of the cell grid (DPMBase::setDomain) */
    double   domain_max[3];
    double   gravity[3];           /* DPMBase::setGravity                            */
    uint32_t periodic_mask;        /* bit d: dimension d is periodic                 */
    int32_t  species_offset;       /* first species of this instance                 */
    int32_t  n_species;            /* species table of this instance is n_species^2  */
    int32_t  reserved;
    double   periodic_min[3];      /* PeriodicBoundary left/right positions          */
    double   periodic_max[3];
} dem_instance_desc;

typedef struct dem_config {
    double   time_step;            /* DPMBase::setTimeStep                           */
    double   background_drag;      /* DPMBase::setBackgroundDrag                     */
    int32_t  rotation;             /* DPMBase::setRotation (1: integrate omega, q)   */
    int32_t  device;               /* CUDA device ordinal                            */
    int32_t  max_neighbors;        /* neighbour-list capacity per particle (0: auto) */
    int32_t  use_graphs;           /* capture the step loop in CUDA graphs           */
    double   skin;                 /* Verlet skin distance (0: 0.4 x smallest radius)*/
    int32_t  n_instances;          /* >= 1                                           */
    int32_t  max_contacts;         /* contact capacity: mean contacts per particle in
                                    * one evaluation (pairs once, plus wall contacts),
                                    * which sizes the per-contact spring storage
                                    * (0: auto, min(max_neighbors,16) + min(walls,4)) */
} dem_config;

/* Global balances (DPMBase::getKineticEnergy ... getCentreOfMass,
 * Kernel/DPMBase.cc:1528-1640; writeEneTimeStep :2100-2123). */
typedef struct dem_globals {
    double  kinetic_energy;
    double  rotational_energy;
    double  gravitational_energy;
    double  elastic_energy;
    double  momentum[3];
    double  angular_momentum[3];
    double  mass;
    double  centre_of_mass[3];
    int64_t n_contacts;
    int64_t n_wall_contacts;
    double  time;
    int64_t n_steps;
} dem_globals;

/* A DeletionBoundary (Kernel/Boundaries/DeletionBoundary.cc:109-126): a
 * particle of the instance whose position x has distance - x . normal < 0
 * after a drift is removed from the simulation. Removed particles keep their
 * slot: they stop interacting and moving, are left out of every balance and
 * coarse-graining sum, and dem_download_particles reports them with
 * instance -1 (position and velocity are then meaningless). */
typedef struct dem_deletion_boundary {
    int32_t instance;
    int32_t reserved;
    double  normal[3];
    double  distance;
} dem_deletion_boundary;

/* An InsertionBoundary of the kind DEM_INSERTION_CUBE (CubeInsertionBoundary)
 * or DEM_INSERTION_CHUTE (ChuteInsertionBoundary). Every time step, after the drift and before the
 * forces (DPMBase::computeOneTimeStep, Kernel/DPMBase.cc:4348-4352),
 * InsertionBoundary::checkBoundaryBeforeTimeStep (Kernel/Boundaries/
 * InsertionBoundary.cc:184-296) places new particles until max_failed
 * successive placements have failed or the inserted volume reaches
 * volume_flow_rate x (time + dt) + initial_volume (insertParticle, :150-176):
 *  - a new particle (InsertionBoundary::generateParticle, :103-142) takes
 *    one draw of the instance's random number generator (the species choice
 *    of a single template) and its radius from the cumulative number
 *    distribution psd_* with the PSD's own generator (PSD::drawSample,
 *    Kernel/Math/PSD.cc:114-128); it is drawn again only after it was placed;
 *  - a placement of a cube boundary draws the position in [pos_min, pos_max]
 *    and the velocity in [vel_min, vel_max], x, y, z each
 *    (CubeInsertionBoundary::placeParticle, Kernel/Boundaries/
 *    CubeInsertionBoundary.cc:173-184); one of a chute boundary puts the
 *    particle at x = pos_min.x + r and draws y in [pos_min.y - r, pos_max.y + r],
 *    z in [pos_min.z - r, pos_max.z + r + fixed_particle_radius] and the
 *    velocity inflow_velocity (1 + U(-variance, variance), U(-variance, variance),
 *    U(-variance, variance)) (ChuteInsertionBoundary::placeParticle,
 *    ChuteInsertionBoundary.cc:163-190); a placement succeeds when
 *    the particle touches no wall and no particle, its periodic images
 *    included (DPMBase::checkParticleForInteractionLocalPeriodic and
 *    checkParticleForInteractionLocal, DPMBase.cc:4868-4958);
 *  - mass and inertia are BaseParticle::computeMass's (Kernel/Particles/
 *    BaseParticle.cc:874-883) for the density; the angular velocity is zero
 *    and the orientation the identity.
 * The instance's generator (DPMBase::random) is in the state
 * RNG::setRandomSeed(seed) leaves it in (Kernel/Math/RNG.cc: the lagged
 * Fibonacci generator 607/273 seeded by the linear congruential one) when
 * the particles are uploaded, and carries on from step to step; a boundary's
 * PSD generator starts from psd_seed (the PSD's default is 0).
 * Inserted particles take the free rows of the upload: rows of the
 * boundary's instance with radius 0, in row order, each keeping its row's
 * id (give free rows the ids the reference's ParticleHandler hands out:
 * consecutive after the largest id in use). A free row is reported with
 * instance -1 until a particle is placed in it; with none left, dem_step
 * returns DEM_ERR_CAPACITY. */
typedef struct dem_insertion_boundary {
    int32_t  kind;                 /* DEM_INSERTION_*                                 */
    int32_t  reserved;
    int32_t  instance;
    int32_t  species;              /* the template particle's species (index in the instance) */
    int32_t  max_failed;           /* InsertionBoundary::maxFailed_                   */
    int32_t  n_psd;                /* points of the PSD: 2 .. DEM_MAX_PSD_POINTS      */
    double   pos_min[3];           /* CubeInsertionBoundary::setGeometry              */
    double   pos_max[3];
    double   vel_min[3];
    double   vel_max[3];
    double   density;              /* ParticleSpecies::getDensity of the species      */
    double   volume_flow_rate;     /* setVolumeFlowRate; +infinity (the default): none */
    double   initial_volume;       /* setInitialVolume                                */
    double   fixed_particle_radius;    /* chute: ChuteInsertionBoundary::set's fixedParticleRadius */
    double   inflow_velocity;          /* chute: inflowVelocity                           */
    double   inflow_velocity_variance; /* chute: inflowVelocityVariance                   */
    double   psd_radius[DEM_MAX_PSD_POINTS];      /* PSD::getParticleSizeDistribution(): radii    */
    double   psd_probability[DEM_MAX_PSD_POINTS]; /* and cumulative probabilities, from 0 to 1    */
    uint64_t psd_seed;             /* PSD::setRandomSeed                              */
} dem_insertion_boundary;

/* The chute's compact inflow fill, Chute::addFlowParticlesCompactly with
 * Chute::createFlowParticle (Kernel/Chute.cc:1083-1115), which a Chute
 * driver runs from setupInitialConditions: with r_in = (min_radius +
 * max_radius) / 2 it places particles until the instance holds
 * N = (unsigned)(particles + x_max y_max inflow_height / r_in^3 / 8) of them.
 * Each candidate draws its radius in [min_radius, max_radius], then z in
 * [z_min + r + fixed_particle_radius, inflow height], y in [y_min + r,
 * y_max - r] and x in [x_min + r, x_max - r] (the three coordinates are the
 * arguments of one Vec3D constructor, which the reference's compiler, g++,
 * evaluates last to first), at rest; it is kept when it touches no wall and
 * no particle (DPMBase::checkParticleForInteraction, periodic images
 * included), else the inflow height grows by 0.0001 max_radius. The draws
 * come from the instance's generator (seeded as for insertion boundaries,
 * dem_set_insertion_boundaries; the boundaries then continue from where the
 * fill left it). The fill runs inside dem_upload_particles, placing the
 * particles in the instance's free rows (radius 0, row order), before the
 * initial force evaluation. */
typedef struct dem_chute_fill {
    int32_t instance;
    int32_t species;               /* the flow particles' species (species 0 in Chute) */
    double  density;               /* its ParticleSpecies::getDensity                 */
    double  x_min, x_max;          /* getXMin, getXMax (= getChuteLength)             */
    double  y_min, y_max;          /* getYMin, getYMax (= getChuteWidth)              */
    double  z_min;                 /* getZMin                                         */
    double  inflow_height;         /* getInflowHeight when the fill starts            */
    double  min_radius, max_radius;/* get{Min,Max}InflowParticleRadius                */
    double  fixed_particle_radius; /* getFixedParticleRadius                          */
} dem_chute_fill;

/* Gaussian coarse-graining grid (CG<XZ|XYZ|O, Gauss, StandardFields>,
 * Kernel/CG/CG.hcc:233-528, Kernel/CG/Fields/StandardFields.cc:184-250).
 * The fields of StandardFields per grid point, in this order (29 doubles):
 *   0      volume fraction          sum V phi
 *   1      density                  sum m phi
 *   2-4    momentum                 sum m v phi
 *   5-10   momentum flux            sum m v(x)v phi     (xx xy xz yy yz zz)
 *   11-19  contact stress           sum F(x)branch psi  (row-major)
 *   20-22  interaction force density (contacts with fixed particles / walls)
 *   23-28  particle size density    sum r^k phi, k = 0..5
 * all divided by the volume of the averaged dimensions (CG::volumeAverageVariables).
 * Points are ordered (i*nY + j)*nZ + k over the resolved dimensions (unresolved: 1). */
#define DEM_CG_NFIELDS 29
#define DEM_CG_O   0
#define DEM_CG_XZ  1
#define DEM_CG_XYZ 2
typedef struct dem_cg_grid {
    int32_t coordinates;           /* DEM_CG_*                                       */
    int32_t instance;
    int32_t n[3];                  /* points per dimension (unused dims: 1)          */
    int32_t reserved;
    double  min[3];                /* CG domain (CG::setMin/setMax)                  */
    double  max[3];
    double  width;                 /* Gaussian standard deviation (Gauss::setWidth)  */
    double  cutoff_factor;         /* cutoff = cutoff_factor * width (reference: 3)  */
} dem_cg_grid;

/* Launch shapes of the time step's force kernels (dem_autotune). They change
 * how the work is spread over the GPU, never the arithmetic: results are
 * bit-identical under every shape. */
typedef struct dem_tuning {
    int32_t detect_block;            /* threads per block of the contact predicate: 64, 128 or 256 */
    int32_t contacts_blocks_per_sm;  /* resident blocks (of 128) per SM of the contact-law kernel,
                                        3..6, with the register budget they leave (168 .. 85) */
    int32_t sum_block;               /* threads per block of the sum/integration kernel: 64, 128, 256 */
    int32_t reserved;
    double  ms_before;               /* dem_autotune: one force evaluation with the shapes it found  */
    double  ms_after;                /* and with the ones it chose (never slower)                    */
} dem_tuning;

typedef struct dem_handle dem_handle;

/* DPMBase construction + setTimeStep/setGravity/setDomain. */
int  dem_create(const dem_config *config, const dem_instance_desc *instances,
                dem_handle **out);
/* Species table: n_species^2 entries per instance, row-major (i*n+j), the
 * mixed entries symmetric (SpeciesHandler::getMixedObject). */
int  dem_set_species(dem_handle *h, const dem_species_pair *table, int n_entries);
/* WallHandler contents (before dem_upload_particles). */
int  dem_set_walls(dem_handle *h, const dem_wall *walls, int n);
/* PeriodicBoundary objects of one instance's BoundaryHandler
 * (PeriodicBoundary::set, Kernel/Boundaries/PeriodicBoundary.cc:84-108): the
 * directions in mask (bit k = axis k) become periodic between lo[k] and
 * hi[k], the others take the instance's domain. The same fields as
 * dem_instance_desc's periodic_*; before dem_upload_particles. */
int  dem_set_periodic(dem_handle *h, int instance, const double lo[3], const double hi[3], uint32_t mask);
/* DeletionBoundary objects of BoundaryHandler, at most
 * DEM_MAX_DELETION_PER_INSTANCE per instance. Before dem_upload_particles, or
 * between dem_step calls (BoundaryHandler::copyAndAddObject during a run, as
 * Drivers/Calibration/CalibrationHeap.cpp:128-131 does): the set replaces the
 * previous one and applies from the next time step. */
int  dem_set_deletion_boundaries(dem_handle *h, const dem_deletion_boundary *b, int n);
/* WallHandler::removeObject / removeLastObject (Kernel/BaseHandler.h:131-136),
 * wall = index in the dem_set_walls array: no contacts with the wall from the
 * next time step on, its contacts' history dropped (as the removed wall's
 * interactions are). Before the upload or between dem_step calls; not for
 * triangle walls. */
int  dem_remove_wall(dem_handle *h, int wall);
/* InsertionBoundary objects of BoundaryHandler (CubeInsertionBoundary, above),
 * at most DEM_MAX_INSERTION_PER_INSTANCE per instance, run in array order
 * after the deletion boundaries' checks. seeds[i] is instance i's
 * RNG::setRandomSeed value (NULL: 0 for every instance, DPMBase's own,
 * DPMBase.cc:279). Before dem_upload_particles, which sizes the cell grid for
 * the PSD's radii, reserves the free rows and starts the generators. */
int  dem_set_insertion_boundaries(dem_handle *h, const dem_insertion_boundary *b, int n,
                                  const uint64_t *seeds);
/* Chute fills (dem_chute_fill, at most one per instance) for the next upload. */
int  dem_set_chute_fills(dem_handle *h, const dem_chute_fill *f, int n);
/* Per fill of the last upload: the inflow height it ended with and the
 * particles it placed (Chute::getInflowHeight, the growth of ParticleHandler). */
int  dem_get_chute_fill_results(dem_handle *h, double *inflow_height, int64_t *added, int n);
/* Per boundary (the order given): particles placed so far and their volume
 * (InsertionBoundary::getNumberOfParticlesInserted / getVolumeOfParticlesInserted). */
int  dem_get_insertion_counts(dem_handle *h, int64_t *inserted, double *volume, int n);
/* The first n values of RNG::getRandomNumber(0, 1) after RNG::setRandomSeed(seed)
 * (Kernel/Math/RNG.cc), from the generator the insertion kernel runs, here on
 * the host: a check of the restatement that needs no device. */
int  dem_rng_draws(uint64_t seed, int n, double *out);
/* The first n radii PSD::drawSample (Kernel/Math/PSD.cc:114-128) gives for
 * the boundary's PSD and psd_seed, from the kernel's code run on the host. */
int  dem_psd_draws(const dem_insertion_boundary *b, int n, double *out);
/* ParticleHandler contents; triggers the first force evaluation on the next
 * dem_step (the one DPMBase::initialiseSolve performs, DPMBase.cc:4180). */
int  dem_upload_particles(dem_handle *h, const dem_particles_soa *p);
/* Inject contact history (restart / oracle states). Call after upload. */
int  dem_upload_contacts(dem_handle *h, const dem_contacts_soa *c);
/* Advance n time steps (n >= 0; n == 0 only performs a pending initial
 * force evaluation). Equivalent to n calls of DPMBase::computeOneTimeStep
 * without output. Returns DEM_ERR_* on a device-side status. */
int  dem_step(dem_handle *h, int nsteps);
int  dem_download_particles(dem_handle *h, dem_particles_soa *p);
/* Total force and torque on every particle from the last force evaluation
 * (3*n doubles each, caller order). */
int  dem_download_forces(dem_handle *h, double *force, double *torque);
/* Current wall states (n must equal the count given to dem_set_walls; the
 * caller's order), after the motion of the steps taken so far
 * (BaseWall::getPosition / getOrientation). */
int  dem_download_walls(dem_handle *h, dem_wall *walls, int n);
/* Live contacts (one row per contact as the reference keeps them).
 * capacity: rows available in c; *count receives the number of contacts
 * (rows beyond capacity are not written). */
int  dem_download_contacts(dem_handle *h, dem_contacts_soa *c, int64_t capacity,
                           int64_t *count);
/* Contact point, unit normal (from I towards P; a wall's normal points into
 * the particle) and friction force (the tangential part of the contact force
 * as the law computed it) of the same contacts, in the order
 * dem_download_contacts reports them: what BaseInteraction::getContactPoint /
 * getNormal / getTangentialForce give the .fstat output
 * (BaseInteraction::writeToFStat, BaseInteraction.cc:487-530). Any of the
 * three arrays (3 doubles per contact) may be null. */
int  dem_download_contact_geometry(dem_handle *h, double *contact_point, double *normal, double *tangential_force,
                                   int64_t capacity, int64_t *count);
int  dem_reduce(dem_handle *h, int instance, dem_globals *out);
/* dem_reduce for the instances first .. first+count-1 of a batch in one pass
 * (the per-instance kinetic-energy traces and centres of mass of a batch of
 * calibration runs). Particle sums run in a fixed order; the elastic energy
 * and contact counts are accumulated with atomics, so their last bits may
 * vary between runs. */
int  dem_reduce_batch(dem_handle *h, int first, int count, dem_globals *out);
/* The batch form of the API: n_instances independent simulations in one
 * handle (dem_create with config->n_instances = n_instances; particles name
 * their instance in dem_particles_soa.instance, which is the instance-offset
 * table of the batch), and a run of nsteps followed by the balances of every
 * instance (out: n_instances entries). */
int  dem_batch_create(const dem_config *config, int n_instances, const dem_instance_desc *instances,
                      dem_handle **out);
int  dem_batch_run(dem_handle *h, int nsteps, dem_globals *out);
/* The balances of dem_reduce, computed without allocating any device memory.
 * It has no counterpart in the reference. It is for callers that may not
 * allocate GPU memory at the point where they need the balances, e.g. a
 * coupled solver that has reserved the whole device memory budget up front,
 * or a monitoring hook run between time steps of a host application that
 * forbids allocation there. dem_reduce allocates a small temporary buffer for
 * its per-block partial sums; this entry point keeps them in a static device
 * array of 1 MiB instead (held by every GPU that loads the library until the
 * process exits) and therefore accepts at most 2,097,152 particles and
 * 2,097,152 contact records (DEM_ERR_CAPACITY above that). The first call on
 * a device looks up the array's device address; make that first call before
 * any stream capture. The address is kept for the life of the process, so a
 * cudaDeviceReset of that device (which also invalidates every handle on it)
 * ends this entry point's use in the process. All calls share the array: calls that overlap on the
 * GPU (several handles on concurrent streams of one device) race. Results are
 * the same sums, in the same order, as dem_reduce. */
int  dem_reduce_noalloc(dem_handle *h, int instance, dem_globals *out);
int  dem_cg_eval(dem_handle *h, const dem_cg_grid *grid, double *fields_out);
/* Device time of the last dem_step call in milliseconds (CUDA events on the
 * handle's stream) and how many kernels it launched. */
int  dem_last_step_stats(dem_handle *h, double *ms, int64_t *kernel_launches,
                         int64_t *rebuilds);
int  dem_get_info(dem_handle *h, int64_t *n_particles, int64_t *max_neighbors,
                  int64_t *n_cells);
/* Device memory held by the handle's particle, list and contact arrays, and
 * the contact capacity (items of one evaluation) they were sized for. */
int  dem_get_memory(dem_handle *h, int64_t *device_bytes, int64_t *contact_capacity);
/* Neighbour-list entries, live particle contacts and wall contacts of the
 * current state (the sizes the per-step byte count is made of). */
int  dem_get_counts(dem_handle *h, int64_t *list_entries, int64_t *contacts,
                    int64_t *wall_contacts);
/* Profiling aid (no reference counterpart): launches the time-step force
 * kernel `reps` times on the current state, writing into the spare state and
 * history buffers without committing them, and returns the mean device time
 * of one launch in milliseconds (CUDA events on the handle's stream). The
 * simulation state is unchanged. */
int  dem_time_force_kernel(dem_handle *h, int reps, double *ms_per_launch);
/* Self-test of the bounded device waits (no reference counterpart): launches,
 * like the rebuild, one cooperative grid whose blocks meet at a barrier that
 * can never complete, so that every wait gives up after `polls` polls and
 * reports DEM_ERR_TIMEOUT; *status receives the status word the kernel wrote
 * (1 << DEM_ERR_TIMEOUT expected). The handle stays usable afterwards. */
int  dem_selftest_wait_expiry(dem_handle *h, int64_t polls, uint32_t *status);
/* Autotuner (the reference's HGridOptimiser, Kernel/HGridOptimiser.cc, picks
 * cell sizes offline from a cost model; the engine's cells follow the
 * reference's HGrid levels, and what is tuned instead are its kernels' launch
 * shapes, measured on the live state): times each force kernel's variants
 * (`reps` force evaluations each, best of three rounds, written to spare
 * buffers so the simulation state is unchanged), one kernel at a time, keeps
 * the fastest shape of each and recaptures the step graphs. Needs a force
 * evaluation (after the first dem_step). */
int  dem_autotune(dem_handle *h, int reps, dem_tuning *out);
/* Applies shapes found earlier (e.g. cached per workload class). */
int  dem_set_tuning(dem_handle *h, const dem_tuning *t);
int  dem_get_tuning(dem_handle *h, dem_tuning *out);
const char *dem_last_error(dem_handle *h);
void dem_destroy(dem_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* DEM_B200_H */
