/*
 * fopis_gpu.h — C ABI of libfopis_gpu.so, the B200 (sm_100a) electrostatic
 * particle-in-cell timestep of FOPIS ("TDPIC"), and its electromagnetic (FDTD)
 * variant.
 *
 * The reference has no plugin or FFI layer: its ES path is the RootGrid phase
 * methods that RootGrid::mainLoopES calls in order (src/Grid/RootGrid/RootGrid.cpp:82-143)
 * plus the start-up in Initializer::initTDPIC (src/Misc/Initialize.cpp:16-107);
 * RootGrid::mainLoopEM (RootGrid.cpp:145-191) is the EM path.
 * Each entry point below replaces one of those methods; the citation beside it
 * names the reference function whose behaviour it keeps.
 *
 * Conventions (all inherited from the reference):
 *   - Normalised units: length = dx, time = dt, mass = m_e, charge = e
 *     (src/Misc/Initialize.cpp:33-36). Positions are in cells, velocities in
 *     cells/step.
 *   - Node arrays carry one glue layer: (nx+2)(ny+2)(nz+2) doubles in C order
 *     [i][j][k], k fastest (src/Grid/Grid.cpp:148-196). A particle at x sits in
 *     node cell i = floor(x)+1 (include/position.hpp:59-69).
 *   - nx, ny, nz are the reference's node counts (Environment::nx). On a
 *     Dirichlet/Neumann axis nx nodes span nx-1 cells; on a periodic axis nx
 *     nodes span nx cells.
 *   - boundary is the 6-letter string "x-x+y-y+z-z+" of D/N/P
 *     (src/Misc/Environment.cpp:51-60).
 *
 * Every function returns 0 (FOPIS_OK) or a negative fopis_status. No C++
 * exception crosses the ABI. A context is used by one host thread at a time;
 * all of its work runs on its own CUDA stream. Host pointers are borrowed for
 * the duration of the call only.
 */
#ifndef FOPIS_GPU_H
#define FOPIS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FOPIS_MAX_SPECIES 8
#define FOPIS_MAX_OBJECTS 8

typedef enum fopis_status {
    FOPIS_OK = 0,
    FOPIS_ERR_ARG = -1,            /* bad argument (std::invalid_argument in the reference) */
    FOPIS_ERR_CUDA = -2,           /* CUDA runtime error */
    FOPIS_ERR_NOMEM = -3,          /* device allocation failed */
    FOPIS_ERR_STATE = -4,          /* call out of order (e.g. step before load) */
    FOPIS_ERR_NOT_CONVERGED = -5,  /* Poisson solve hit max_vcycles; phi kept */
    FOPIS_ERR_DEVICE = -6,         /* a kernel latched an error bit in the device status word */
    FOPIS_ERR_CAPACITY = -7,       /* particle / absorbed-list capacity exceeded */
    FOPIS_ERR_NO_CUDA = -8         /* no usable CUDA device */
} fopis_status;

/* Device status bits (fopis_get_stats().device_status). */
#define FOPIS_DEV_PARTICLE_OVERFLOW   0x1   /* appended particles exceeded capacity */
#define FOPIS_DEV_ABSORB_OVERFLOW     0x2   /* absorbed list exceeded capacity */
#define FOPIS_DEV_BAD_CMAT_NODE       0x4   /* absorption/emission hit a node that is not a surface node
                                               (Spacecraft::getCmatNumber throws, Spacecraft.cpp:233-234) */
#define FOPIS_DEV_SURFACE_NOT_FOUND   0x8   /* absorbed particle without a crossing face (Spacecraft.cpp:573-582) */
#define FOPIS_DEV_INJECT_REJECTS      0x10  /* injection rejection sampling hit its attempt cap */
#define FOPIS_DEV_NONFINITE           0x20  /* NaN/Inf met in a reduction */
#define FOPIS_DEV_RHO_OVERFLOW        0x40  /* a node's int64 fixed-point charge sum passed 2^64
                                               (more than 2^13 full particle weights on one node) */

typedef enum fopis_species_kind {
    FOPIS_SPECIES_AMBIENT = 0,        /* AmbientParticleType */
    FOPIS_SPECIES_PHOTOELECTRON = 1,  /* PhotoElectronParticleType */
    FOPIS_SPECIES_SECONDARY = 2       /* SecondaryParticleType (src/Particle/SecondaryParticleType.cpp):
                                         emitted where other species hit a body; thermal_velocity
                                         is the true-secondary emission speed sqrt(2T/m) */
} fopis_species_kind;

/* One particle species; fields mirror ParticleType (include/particle_type.hpp:13-120). */
typedef struct fopis_species {
    int kind;                   /* fopis_species_kind */
    int particle_per_cell;      /* ParticleType::particle_per_cell */
    double charge;              /* ParticleType::charge, in e */
    double mass;                /* ParticleType::mass, in m_e */
    double size;                /* ParticleType::size = int(dx^3 n / ppc) (ParticleType.cpp:33-36) */
    double thermal_velocity;    /* calcThermalVelocity() = sqrt(2T/m), normalised (ParticleType.cpp:49-51) */
    double deviation;           /* calcDeviation() = sqrt(T/m), normalised (ParticleType.cpp:53-55) */
    double drift[3];            /* AmbientParticleType::drift_velocity, normalised */
    int injection_axis[6];      /* AmbientParticleType::injection_axis (-x,+x,-y,+y,-z,+z) */
    double flux[6];             /* AmbientParticleType::calcFlux() (AmbientParticleType.cpp:8-57) */
    double emission_amount;     /* photoelectrons per lit surface node per step:
                                   dx^2 * getEmissionAmount() (Spacecraft.cpp:876-877) */
} fopis_species;

typedef enum fopis_precision {
    FOPIS_MIXED = 0,   /* int32 cell + FP32 offset/velocity particles, int64 fixed-point rho,
                          FP32 smoother inside FP64 iterative refinement */
    FOPIS_FP64 = 1     /* int32 cell + FP64 offset/velocity particles, FP64 E gather and push,
                          FP64 CIC deposit (atomic sums), phi from the same FP64 residual
                          refinement to the requested tolerance; the reference run for
                          the mixed mode's error */
} fopis_precision;

typedef enum fopis_guess_mode {
    FOPIS_GUESS_ZERO = 0,      /* every solve starts from phi = 0 */
    FOPIS_GUESS_WARM = 1,      /* start from the previous phi (the reference's behaviour) */
    FOPIS_GUESS_LEARNED = 2,   /* FOPIS_GUESS_HISTORY with the first solve seeded by the U-Net's
                                  predicted increment, with fallback */
    FOPIS_GUESS_HISTORY = 3    /* per-solve history: the first solve of a step starts from the
                                  previous step's first solve, the second from the first plus
                                  the previous step's conductor response */
} fopis_guess_mode;

/* Simulation parameters: the normalised content of input.json after
 * Initializer::loadEnvironment / loadParticleType / loadStaticField. */
typedef struct fopis_params {
    int nx, ny, nz;              /* Environment::nx,ny,nz (one rank: cell_x = nx) */
    char boundary[8];            /* Environment::boundary, e.g. "DDDDDD" */
    double eps0;                 /* Normalizer::eps0 */
    double static_bfield[3];     /* StaticField::static_bfield, normalised (Initialize.cpp:312-319) */
    double shine_vector[3];      /* StaticField::shine_vector */
    int nspecies;                /* Environment::num_of_particle_types; order ambient -> photo */
    fopis_species species[FOPIS_MAX_SPECIES];
    double poisson_tol;          /* ||f - A phi||_2 <= tol ||f||_2 ; 0 -> 1e-8 */
    int max_vcycles;             /* V-cycle cap per solve; 0 -> 100 */
    int guess_mode;              /* fopis_guess_mode */
    int sort_interval;           /* counting-sort period in steps; 0 -> 8 */
    int remove_interval;         /* removeInvalidParticles period (RootGrid.cpp:136-140); 0 -> 50 */
    double capacity_factor;      /* particle capacity / initial count; 0 -> 1.5 */
    int precision;               /* fopis_precision */
    int solver;                  /* fopis_solver: Environment::solver_type */
    uint64_t seed;               /* Philox key for loading, injection and emission */
    double energy_ev;            /* Normalizer::unnormalizeEnergy(1, "eV") = m_e dx^2 / (e dt^2): eV per
                                    normalised energy unit (secondary-emission yields); 0 without them */
    double mu0;                  /* Normalizer::mu0 = mu0 e^2 / (m_e dx) (include/normalizer.hpp:219-221);
                                    used by the EM solver only. Normalizer::c = 1/sqrt(eps0 mu0) must not
                                    exceed 1 (Environment::checkCFLCondition, Environment.cpp:193-203) */
} fopis_params;

typedef enum fopis_solver {
    FOPIS_SOLVER_ES = 0,   /* RootGrid::mainLoopES: Poisson solve each step */
    FOPIS_SOLVER_EM = 1    /* RootGrid::mainLoopEM (RootGrid.cpp:145-191): FDTD on a Yee grid with
                              damping layers of the grid's own size beyond every non-periodic face,
                              charge-conserving (zigzag) edge currents */
} fopis_solver;

/* A voxel conductor; replaces the ObjectDataFromFile + Spacecraft construction
 * (src/Spacecraft/ObjectUtils.cpp:9-333, Spacecraft.cpp:16-152). */
typedef struct fopis_object_desc {
    int n_cmat;                  /* surface node count = capacity-matrix size */
    const int32_t* cmat_nodes;   /* [n_cmat][3] glue-layout node indices; row c = cmat number c */
    int n_cells;                 /* inner (body) cells */
    const int32_t* cells;        /* [n_cells][3] glue-layout cell indices */
    int is_potential_fixed;      /* ObjectInfo_t::is_potential_fixed */
    double fixed_potential;      /* normalised */
    double initial_potential_offset; /* normalised (Spacecraft::initializeChargeMapOffset) */
    int emit_species;            /* photoelectron species emitted from the lit face, -1 = none */
    int secondary_species;       /* secondary-electron species emitted where particles hit the body,
                                    -1 = none (Spacecraft::hasSecondaryParticles, SecondaryEmission.cpp:5-12) */
    int dielectric;              /* surface_type "dielectric" (Spacecraft::isDielectricSurface) */
    const double* capacitance;   /* [n_cmat] normalised node capacitance of a dielectric surface, the mean
                                    over the node's faces of normalizeCapacitance(4 pi eps0 eps_r) of the
                                    face's material (Spacecraft.cpp:117-149); 0 where none */
} fopis_object_desc;

/* Field selectors for fopis_get_field / fopis_set_field. */
typedef enum fopis_field {
    FOPIS_FIELD_PHI = 0,     /* Field::phi */
    FOPIS_FIELD_RHO0 = 1,    /* Field::rho[0] (total, after redistribution) */
    FOPIS_FIELD_EXREF = 2,   /* Field::exref (nodal E) */
    FOPIS_FIELD_EYREF = 3,
    FOPIS_FIELD_EZREF = 4,
    FOPIS_FIELD_BXREF = 5,   /* Field::bxref (nodal B, EM) */
    FOPIS_FIELD_BYREF = 6,
    FOPIS_FIELD_BZREF = 7,
    FOPIS_FIELD_JXREF = 8,   /* Field::jxref (nodal current, EM; RootGrid::updateReferenceCurrent,
                                RootGridField.cpp:1256-1285) */
    FOPIS_FIELD_JYREF = 9,
    FOPIS_FIELD_JZREF = 10,
    FOPIS_FIELD_RHO_SPECIES = 16, /* + species id: Field::rho[1 + s] */
    /* EM Yee arrays in their own extents (fopis_field_shape): */
    FOPIS_FIELD_EX = 32,     /* Field::ex .. ez, edges, damping layers included */
    FOPIS_FIELD_EY = 33,
    FOPIS_FIELD_EZ = 34,
    FOPIS_FIELD_BX = 35,     /* Field::bx .. bz, faces, damping layers included */
    FOPIS_FIELD_BY = 36,
    FOPIS_FIELD_BZ = 37,
    FOPIS_FIELD_JX = 38,     /* Field::jx .. jz, edges of the glue grid */
    FOPIS_FIELD_JY = 39,
    FOPIS_FIELD_JZ = 40
} fopis_field;

typedef struct fopis_stats {
    int64_t timestep;            /* steps taken by this context */
    int vcycles_last;            /* V-cycles of the last solve */
    int vcycles_step;            /* V-cycles summed over the solves of the last step */
    int solves_step;             /* solves in the last step (2 with conductors) */
    int converged;               /* last solve reached the tolerance */
    double residual_last;        /* ||r||_2/||f||_2 of the last solve */
    double residual_initial;     /* same, before the first V-cycle of the last solve */
    int64_t num_particles[FOPIS_MAX_SPECIES];   /* slots in use per species: the valid particles plus the
                                                   slots of particles removed since the last sort */
    int64_t capacity[FOPIS_MAX_SPECIES];
    int64_t absorbed_step;       /* particles absorbed by conductors in the last step */
    int64_t injected_step;
    int64_t emitted_step;
    uint32_t device_status;      /* FOPIS_DEV_* bits */
    int learned_used;            /* the learned guess seeded the last step's solves */
    double ms_phase[8];          /* last step, ES: push, emit, inject, absorb, rho + first solve, second
                                    solve, efield, sort; EM: velocity (0 when the particle pass gives
                                    it), emit, position with the currents + inject, 0, rho, E update,
                                    B update, sort */
    int64_t kernel_launches;     /* kernels this context has launched since creation */
    int solve_mode;              /* 0: host-driven V-cycle loop; 1: one CUDA graph with a device-side
                                    loop; 2: the same graph with programmatic dependent launches */
    int pad;
    double residual_pointwise;   /* last solve, RootGrid::checkPhiResidual's measure
                                    (RootGridField.cpp:267-317): max over unknown nodes with a
                                    nonzero source of |L phi + rho/eps0| / |rho/eps0| (mean-free
                                    source when every axis is periodic) */
    int64_t valid_particles[FOPIS_MAX_SPECIES];  /* valid particles after the last fused step (those the
                                                    push kept plus the injected and emitted ones) or the
                                                    last sort */
    int64_t pushed_step[FOPIS_MAX_SPECIES];      /* valid particles the last fused step's push moved */
} fopis_stats;

/* ---- lifetime ----------------------------------------------------------- */

/* Replaces RootGrid::RootGrid field set-up (RootGrid.cpp:7-40, Grid.cpp:148-196).
 * device < 0 selects the current device. */
int fopis_create(const fopis_params* params, int device, void** ctx);
void fopis_destroy(void* ctx);
const char* fopis_last_error(void* ctx);
const char* fopis_version(void);

/* ---- conductors --------------------------------------------------------- */

/* Replaces RootGrid::initializeObjects (RootGridObject.cpp:6-75). */
int fopis_add_object(void* ctx, const fopis_object_desc* desc, int* object_id);
/* Replaces RootGrid::initializeObjectsCmatrix (RootGridObject.cpp:77-148): one
 * Poisson solve per surface node for B, then C = B^-1 (Cmatrix.hpp:31-34),
 * then Spacecraft::initializeChargeMapOffset (Spacecraft.cpp:160-183). */
int fopis_build_capacity_matrix(void* ctx, int object_id);
/* IO::loadCmatrixData / writeCmatrixData (IO.cpp:28-120): C row-major [i][j] = capacity_matrix(i, j). */
int fopis_set_capacity_matrix(void* ctx, int object_id, const double* C, int n);
int fopis_get_capacity_matrix(void* ctx, int object_id, double* C, int n);
/* Spacecraft::getLogEntry values (Spacecraft.cpp:1011-1044), normalised:
 * potential, total charge, current per species (charge per step). */
int fopis_get_object(void* ctx, int object_id, double* potential, double* charge,
                     double* current_per_species);
/* Spacecraft::charge_map [nspecies][n_cmat], normalised charge. */
int fopis_get_charge_map(void* ctx, int object_id, double* charge_map, int n);
/* Restores it (RootGrid::loadResumeObjectData, RootGridIO.cpp:273-280); n as above. */
int fopis_set_charge_map(void* ctx, int object_id, const double* charge_map, int n);

/* ---- particles ---------------------------------------------------------- */

/* Loads particles of one species from the reference's 56-byte Particle record
 * {double x,y,z,vx,vy,vz; int typeId,isValid} (include/particle.hpp:14-20).
 * Invalid records are skipped. Appends to what the species already holds. */
int fopis_load_particles(void* ctx, int species, const void* particles56, int64_t n);
/* Copies the valid particles of one species out in the 56-byte record layout.
 * *n_out receives the count; at most cap records are written. */
int fopis_get_particles(void* ctx, int species, void* particles56, int64_t cap, int64_t* n_out);
/* Raw split-precision state of the valid particles (mixed precision only): the
 * particle's node cell packed as (i << 20) | (j << 10) | k in glue-layout indices
 * (i = floor(x)+1, include/position.hpp:59-69), the in-cell offsets x-(i-1) and
 * the velocities. */
int fopis_get_particles_raw(void* ctx, int species, int32_t* cell, float* ox, float* oy,
                            float* oz, float* vx, float* vy, float* vz, int64_t cap, int64_t* n_out);
/* Uniform ambient loading of RootGrid::RootGrid (RootGrid.cpp:45-79) on the device:
 * Philox-keyed positions and Maxwellian velocities, conductor interiors removed
 * (Spacecraft::removeInnerParticle, Spacecraft.cpp:508-510). */
int fopis_generate_ambient(void* ctx);
/* Counting sort of every species by cell; drops invalid particles
 * (Grid::removeInvalidParticles, GridParticleTreatment.cpp:93-102, and more). */
int fopis_sort_particles(void* ctx);

/* ---- the ES step and its phases (RootGrid::mainLoopES order) ------------ */

/* Grid::initialize (Grid.cpp:23-36): updateRho, solvePoisson, updateEfield, and in
 * the EM mode updateBfield. */
int fopis_initialize(void* ctx);
/* n calls of RootGrid::mainLoopES (RootGrid.cpp:82-143), fused: the push kernel
 * gathers, pushes, moves, applies boundaries and deposits in one pass. With
 * solver FOPIS_SOLVER_EM, n calls of RootGrid::mainLoopEM (RootGrid.cpp:145-191). */
int fopis_step(void* ctx, int n);
/* Phase entry points, for parity checks between phases. */
int fopis_update_velocity(void* ctx);        /* Grid::updateParticleVelocityES (GridParticleTreatmentES.cpp:13-88);
                                                EM: updateParticleVelocityEM (GridParticleTreatmentEM.cpp:13-105) */
int fopis_emit_particles(void* ctx);         /* RootGrid::emitParticlesFromObjects (RootGridObject.cpp:175-181) */
/* Spacecraft::incident_events (SecondaryEmission.cpp:14-33): the hits recorded by the last
 * absorption, consumed by the next emission. One record of FOPIS_INCIDENT_DOUBLES doubles:
 * object, incident species, surface axis (0 x, 1 y, 2 z), remaining time (the move ratio
 * since the crossing), crossing point x, y, z, velocity vx, vy, vz. get copies at most cap
 * records out (*n gets the count); set replaces the pending list (n <= the absorbed-list
 * capacity). */
#define FOPIS_INCIDENT_DOUBLES 10
int fopis_get_incidents(void* ctx, double* records, int64_t cap, int64_t* n);
int fopis_set_incidents(void* ctx, const double* records, int64_t n);
int fopis_update_position(void* ctx);        /* RootGrid::updateParticlePositionES (GridParticleTreatmentES.cpp:90-181);
                                                EM: updateParticlePositionEM with the edge currents
                                                (GridParticleTreatmentEM.cpp:107-201) */
int fopis_inject_particles(void* ctx);       /* RootGrid::injectParticlesFromBoundary (RootGridParticle.cpp:3-130) */
int fopis_update_rho(void* ctx);             /* RootGrid::updateRho (RootGridField.cpp:1153-1252), incl. the
                                                first solve and Spacecraft::redistributeCharge when objects exist */
int fopis_solve_poisson(void* ctx);          /* RootGrid::solvePoisson (RootGridField.cpp:41-63) */
int fopis_update_efield(void* ctx);          /* ES: RootGrid::updateEfield + updateReferenceEfield (RootGridField.cpp:456-582);
                                                EM: RootGrid::updateEfieldFDTD (damping form, :584-710) */
int fopis_update_reference_fields(void* ctx);  /* ES: the nodal E from phi (updateReferenceEfield on the edges of
                                                updateEfield); EM: RootGrid::updateReferenceEfield and
                                                updateReferenceBfield on the current Yee arrays (RootGridField.cpp:
                                                489-582, 1102-1127), as Grid::initializeForLoad (Grid.cpp:38-50) */
int fopis_update_bfield(void* ctx);          /* EM: RootGrid::updateBfield (damping form, RootGridField.cpp:589-820)
                                                and updateReferenceBfield (:1102-1127); FOPIS_ERR_STATE in ES */
int fopis_remove_invalid_particles(void* ctx); /* Grid::removeInvalidParticles */
/* Ends a step driven through the phase entry points: ++Environment::timestep
 * (src/main.cpp:33), which keys the Philox draws of injection and emission. */
int fopis_advance_timestep(void* ctx);
/* Environment::timestep of the next step, as Environment::loadInfo restores it
 * (src/Misc/Environment.cpp:379-420); the Philox keys of injection and emission
 * continue from it. */
int fopis_set_timestep(void* ctx, int64_t timestep);
/* The fractional injection carry of RootGrid::injectParticlesFromBoundary
 * (RootGridParticle.cpp:3-130), [nspecies][6 faces]: saved with a resume so that
 * a continued run injects the same counts. */
int fopis_get_injection_carry(void* ctx, double* carry, int n);
int fopis_set_injection_carry(void* ctx, const double* carry, int n);

/* ---- fields and diagnostics --------------------------------------------- */

/* Copies a field out in the reference's C order [i][j][k] over its own extent:
 * n = (nx+2)(ny+2)(nz+2) for node fields, the product of fopis_field_shape's
 * extents for the EM Yee arrays (FOPIS_FIELD_EX .. JZ). */
int fopis_get_field(void* ctx, int which, double* out, size_t n);
/* Overwrites PHI or RHO0 (for solver-only use and warm starts) or, in the EM
 * mode, one Yee array or edge current (EX .. JZ: initial fields of a run or a
 * resume; the next position update recomputes J). */
int fopis_set_field(void* ctx, int which, const double* in, size_t n);
/* First index (the multi_array index base: below 0 on axes with damping
 * layers) and extent per axis of a field. */
int fopis_field_shape(void* ctx, int which, int lo[3], int n[3]);
/* Field::getBfieldEnergy (src/Grid/Field.cpp:215-234), normalised; 0 in ES. */
int fopis_get_bfield_energy(void* ctx, double* energy);
/* Grid::getParticleEnergy (GridParticleTreatment.cpp:104-118) and
 * Field::getEfieldEnergy (Field.cpp:194-213), normalised. */
int fopis_get_energy(void* ctx, double* particle_energy, double* efield_energy);
int fopis_get_stats(void* ctx, fopis_stats* stats);
/* The cudaStream_t all of the context's work runs on (for callers that order
 * their own work or events against it). */
int fopis_get_stream(void* ctx, void** stream);
/* Sets the Poisson start mode (fopis_guess_mode). */
int fopis_set_guess_mode(void* ctx, int mode);

/* ---- learned initial guess (no reference counterpart) -------------------- */

/* Trains the U-Net online on the (rho^n, phi^{n-1}, phi^{n-2}) -> phi^n - phi^{n-1}
 * pairs that the plain solver produces during fopis_step. enable = 0 stops. */
int fopis_unet_set_training(void* ctx, int enable, double learning_rate);
/* Loss of the last training step and number of steps taken. */
int fopis_unet_get_state(void* ctx, double* last_loss, int64_t* train_steps);
/* The fallback policy of FOPIS_GUESS_LEARNED: running averages of the first
 * solve's V-cycles from the history start and from the learned guess, and
 * whether the learned guess is currently enabled (0 while falling back). */
int fopis_unet_get_policy(void* ctx, double* plain_vcycles, double* learned_vcycles, int* learned_enabled);
/* The last first solve: initial residual ||f - A phi||/||f|| from the history
 * start and from the learned guess (equal when the guess was not used), and
 * the device time of the network's forward pass (with the guess check) and of
 * its training step, in milliseconds. A guess that does not lower the initial
 * residual is discarded for that solve. */
int fopis_unet_get_last(void* ctx, double* warm_residual, double* guess_residual, double* ms_forward,
                        double* ms_train);
/* The network on caller fields (host arrays of N glue-layout nodes): features
 * of rho0, phi^{n-1}, phi^{n-2}; pred (optional) receives the predicted
 * increment phi^n - phi^{n-1} on the solver's unknowns (0 elsewhere). With
 * phi_target the loss mean((out - (phi_target - phi1)/sigma)^2) goes to loss
 * and, when grads is given, its gradient for every parameter
 * (fopis_unet_params order); no optimiser step is taken. */
int fopis_unet_eval(void* ctx, const double* rho0, const double* phi1, const double* phi2,
                    const double* phi_target, double* pred, float* grads, double* loss);
/* FP32 master parameters: copied to get and/or replaced from set (either may be
 * null); *count receives their number. Order per convolution l = 0..5:
 * W[27][cout][cin] (tap = (di+1)*9 + (dj+1)*3 + (dk+1)), b[cout]; then the
 * head w[16], b. Convolutions (cin, cout, level): (16,16,0) (16,32,1) (32,64,2)
 * (64,64,2) (64,32,1) (32,16,0). */
int fopis_unet_params(void* ctx, float* get, const float* set, int64_t* count);
/* One activation or gradient buffer of the last evaluation as FP32, solver
 * unknown order with channels last (index: x0 e0 d1 e1 d2 e2 e3 u1 a4 u0 a5
 * g5 du0 da1 g4 du1 de3 g3 g2 dd2 g1 dd1 g0 ge0, then 24 = prediction).
 * With host null only *count (values) is set. */
int fopis_unet_tensor(void* ctx, int which, float* host, int64_t cap, int64_t* count);

/* ---- device self-check (no reference counterpart) ----------------------- */

/* Runs the bounded mbarrier wait that guards every tensor-core pipeline stage
 * of the learned guess, alone, on `device`: a barrier expecting one arrival is
 * waited on for up to `polls` polls; with arrive = 0 nothing arrives, so the
 * wait runs out and *status receives 1 (the kernels' error report), with
 * arrive = 1 the phase completes and *status receives 0. Nothing asynchronous
 * is in flight, so the device stays usable either way. */
int fopis_check_bounded_wait(int device, uint32_t polls, int arrive, uint32_t* status);

/* ---- allocation-free variant (no reference counterpart) ------------------ */

/* Field::getEfieldEnergy's value (the quantity fopis_get_energy reports as
 * efield_energy) for a potential the caller owns, computed without allocating
 * any device memory. For callers that cannot call cudaMalloc once their run
 * loop has started: hosts that give the library only memory from their own
 * pool allocator, and real-time loops that forbid allocator calls because
 * cudaMalloc/cudaFree synchronise the device.
 * phi: device pointer, (nx+2)(ny+2)(nz+2) doubles in the glue layout;
 * energy: device pointer to one double, written as 0.5 eps0 sum(edge E^2);
 * stream: a cudaStream_t (NULL = legacy default stream); work is enqueued, not
 * waited for. Scratch is a 32 KB file-scope device array held by every CUDA
 * context that loads the library until that context ends, so nx*ny*nz may not
 * exceed 33,554,432 (FOPIS_ERR_ARG beyond). All calls share that array: calls
 * that overlap on the GPU race. The first call in a context (on a device)
 * looks the array's address up with cudaGetSymbolAddress, keyed by the
 * context's unique id, and should come before any stream capture. This entry
 * point has no counterpart in the reference. */
int fopis_efield_energy_noalloc(const double* phi, int nx, int ny, int nz, double eps0, double* energy,
                                void* stream);

/* ---- set-up helpers (host side, no device work) ------------------------- */

/* ObjectUtils::getObjectNodesFromObjFile (ObjectUtils.cpp:9-333): parses a
 * MagicaVoxel .obj into surface nodes (cmat order) and inner cells, both in
 * glue-layout indices for a single-rank domain of nx,ny,nz nodes. Arrays are
 * allocated with malloc; release them with fopis_free. */
int fopis_parse_obj(const char* path, int nx, int ny, int nz,
                    int32_t** cmat_nodes, int* n_cmat, int32_t** cells, int* n_cells);
/* The same file's face textures per surface node (ObjectDataFromFile::textures,
 * ObjectUtils.cpp:65-160): node c (cmat order) lists the texture index of every quad
 * covering it, tex[start[c] .. start[c+1]), start has n_cmat + 1 entries. The
 * texture index is the vt number of the quad's first vertex (f v/vt/vn ...). */
int fopis_parse_obj_textures(const char* path, int nx, int ny, int nz,
                             int32_t** start, int32_t** tex, int* n_cmat);
void fopis_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* FOPIS_GPU_H */
