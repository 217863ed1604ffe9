/*
 * zmpm.h -- C ABI of the B200 implicit APIC MPM substep.
 *
 * This is the drop-in boundary for the implicit (backward-Euler) APIC MPM
 * substep of ziran2019 (Lib/MPM over Lib/SPGrid).  The reference exposes that
 * substep as C++ template classes with no FFI; every entry point below names the
 * reference member function or plugin call it replaces (path:line inside the
 * reference project).
 *
 * Conventions
 *   - Every function returns an int status (ZMPM_OK == 0; negative values are
 *     errors, positive values are informational outcomes of a substep).
 *   - No C++ exception crosses this boundary.
 *   - One context == one simulation on one CUDA device, driven from one host
 *     thread (the reference is also single-caller, MpmSimulationBase.h:133-229).
 *   - Host arrays are row-major: positions [n][3], matrices [n][3][3].
 *   - Particles are addressed by the index they were added with; the library
 *     reorders its device copy internally and never changes those indices.
 */
#ifndef ZMPM_H
#define ZMPM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status -- */
enum zmpm_status_code {
    ZMPM_OK = 0,
    /* a particle moved more than one cell in the substep; the reference throws
       RestartException here (Lib/MPM/MpmSimulationBase.cpp:983-1002) */
    ZMPM_CFL_VIOLATION = 1,
    /* Newton stopped at max_iterations above tolerance; the reference only
       returns false (Lib/Ziran/Math/Nonlinear/NewtonsMethod.h:65) */
    ZMPM_NEWTON_NOT_CONVERGED = 2,
    ZMPM_NAN_DETECTED = 3,
    ZMPM_TIMEOUT = 4, /* a bounded device-side wait gave up */
    ZMPM_BAD_ARG = -1,
    ZMPM_OUT_OF_GRID = -2, /* a particle stencil leaves the configured grid */
    ZMPM_CUDA_ERROR = -3,
    ZMPM_NO_MEMORY = -4,
    ZMPM_NOT_READY = -5, /* a test hook was called before zmpm_begin_implicit */
    ZMPM_UNSUPPORTED = -6
};

/* ------------------------------------------------------------- enums -------- */
enum zmpm_precision {
    ZMPM_FP64 = 0, /* every array and every operation in double */
    ZMPM_MIXED = 1 /* state, residuals, reductions FP64; Hessian-vector product FP32 */
};

/* SPGrid page shape.  GridState<double,3> is 128 B, so a 4 KiB page holds
   2x4x4 nodes; GridState<float,3> is 64 B -> 4x4x4 nodes
   (Lib/MPM/MpmGrid.h:14-43, Lib/SPGrid/Core/SPGrid_Mask.h:31-37). */
enum zmpm_layout {
    ZMPM_LAYOUT_AUTO = 0, /* FP64 -> 2x4x4, MIXED -> 4x4x4 */
    ZMPM_LAYOUT_244 = 1,
    ZMPM_LAYOUT_444 = 2
};

/* Constitutive models (F-based force helper plugins). */
enum zmpm_model {
    ZMPM_MODEL_NONE = 0,
    /* NeoHookeanBorden: Lib/Ziran/Physics/ConstitutiveModel/NeoHookeanBorden.cpp:16-111 */
    ZMPM_MODEL_NEOHOOKEAN_BORDEN = 1,
    /* StvkWithHenckyIsotropic: Lib/Ziran/Physics/ConstitutiveModel/StvkWithHenckyIsotropic.h:114-173 */
    ZMPM_MODEL_STVK_HENCKY_ISOTROPIC = 2,
    /* Fixed corotated (Stomakhin et al. 2012).  Not present in the reference;
       written in the reference's SVD-isotropic plugin form. */
    ZMPM_MODEL_FIXED_COROTATED = 3
};

/* Plasticity return maps (PlasticityApplier plugins). */
enum zmpm_plasticity {
    ZMPM_PLASTIC_NONE = 0,
    /* VonMisesStvkHencky::projectStrain, Lib/Ziran/Physics/PlasticityApplier.cpp:462-502 */
    ZMPM_PLASTIC_VON_MISES = 1,
    /* DruckerPragerStvkHencky::projectStrain (PlasticityApplier.cpp:272-317; Klar
       et al. 2016, sand) on StvkWithHenckyIsotropic particles: Hencky strain of
       the SVD shifted by the cohesion, projection to the cone tip when the trace
       (with the volume-correction log Jp) is >= 0, else onto the cone. */
    ZMPM_PLASTIC_DRUCKER_PRAGER = 2,
    /* NonAssociativeCamClay::projectStrain (PlasticityApplier.cpp:112-227, the
       branch it runs: Compare_With_Physbam, :35-110) on NeoHookeanBorden
       particles: projection of (p, s) onto the Cam-Clay ellipse with tips, and
       the "fake hardening" update of log Jp. */
    ZMPM_PLASTIC_CAM_CLAY = 3
};

/* Damage models applied after P2G (FractureSimulation::particlesToGrid,
   Projects/fracture/FractureSimulation.h:149-160). */
enum zmpm_damage {
    ZMPM_DAMAGE_NONE = 0,
    /* Rankine ("naive") damage, FractureSimulation::solvePhaseFieldSystemNaive
       (FractureSimulation.h:509-554): principal Cauchy stress of the undegraded
       NeoHookeanBorden stress, c <- min(c, sigma_F / sigma_max) when
       sigma_max > sigma_F, g = c^2 (1 - k) + k, with sigma_max the largest
       principal stress (what the criterion and the variable's name call for;
       ZMPM_DAMAGE_RANKINE_REFERENCE follows the reference's eigenvalue order). */
    ZMPM_DAMAGE_RANKINE = 1,
    /* CD-MPM phase field, FractureSimulation::solvePhaseFieldSystem
       (FractureSimulation.h:257-456): after P2G, c is solved on the grid from
       the lumped-mass elliptic (or parabolic, parabolic_M > 0) phase-field
       system by Jacobi-preconditioned CG (Projects/fracture/ConjugateGradient.h:
       53-104), transferred back (phaseG2P, :458-507) with c <- max(min(c, c_new), 0);
       then PhaseField::Update_Phase_Field_Fp (PhaseField.h:70-76) from the
       positive NeoHookeanBorden energy and g = c^2 (1 - k) + k.  Every particle
       of the scene carries the phase field (the reference indexes it for all
       particles), added by zmpm_add_phase_field. */
    ZMPM_DAMAGE_PHASE_FIELD = 2,
    /* Rankine damage as the reference computes it: sigma_max is
       cauchy.eigenvalues()[0].real() of Eigen's general eigensolver
       (FractureSimulation.h:539-543), the first eigenvalue in the order of the
       real Schur form (Householder-Hessenberg reduction and Francis
       double-shift QR), which need not be the largest. */
    ZMPM_DAMAGE_RANKINE_REFERENCE = 3
};

/* Krylov solver of the Newton step (BackwardEuler.h:82-98). */
enum zmpm_linear_solver { ZMPM_MINRES = 0, ZMPM_CG = 1 };

/* Implicit integrator of a substep.  NEWTON: MpmSimulationBase::backwardEulerStep
   (MpmSimulationBase.cpp:610-657).  ADMM: AdmmSimulation::admmStep
   (Projects/admm/AdmmSimulationFoam.h:766-801), the local (per-particle F),
   global (MINRES on the grid) and dual steps of "Silly Rubber".  EXPLICIT: the
   symplectic branch of MpmSimulationBase::advanceOneTimeStep
   (MpmSimulationBase.cpp:264-281): Kirchhoff stress at the particles
   (forcesUpdateParticleState), P2G of mass, momentum and force
   (particlesToGridWithForceHelper<APIC, quadratic, !MLS>, :500-560),
   gridVelocityExplicitUpdate with collisions (:818-865), the colliders'
   state at t + dt, trialCollision (:298-311) when `trial_collision` is set,
   then G2P. */
enum zmpm_integrator { ZMPM_NEWTON = 0, ZMPM_ADMM = 1, ZMPM_EXPLICIT = 2 };

/* Collision objects (AnalyticCollisionObject, CollisionObject.h:42-195). */
enum zmpm_collider_shape { ZMPM_HALF_SPACE = 0, ZMPM_SPHERE = 1, ZMPM_BOX = 2 };
enum zmpm_collider_type { ZMPM_STICKY = 1, ZMPM_SLIP = 2, ZMPM_SEPARATE = 3, ZMPM_GHOST = 4 };

/* ----------------------------------------------------------- structs -------- */
typedef struct zmpm_ctx zmpm_ctx;

typedef struct zmpm_config {
    int32_t precision;   /* zmpm_precision */
    int32_t layout;      /* zmpm_layout */
    int32_t grid_log2;   /* grid covers [0, 2^grid_log2)^3 nodes; <= 12 (SPGrid 4096^3) */
    int32_t device;      /* CUDA device ordinal */
    double dx;
    double gravity[3];
    double apic_rpic_ratio; /* 1 = APIC (reference default, MpmSimulationBase.cpp:36) */
    double cfl;             /* only used for the half-cell statistic, as the reference */
} zmpm_config;

typedef struct zmpm_solver {
    int32_t linear_solver;          /* zmpm_linear_solver */
    int32_t newton_max_iterations;  /* reference default 3 (MpmSimulationBase.cpp:51) */
    double newton_tolerance;        /* reference default 1e-5, mass-weighted norm */
    int32_t krylov_max_iterations;  /* reference default 20 (BackwardEuler.h:56) */
    int32_t pad0;
    double krylov_tolerance;        /* absolute; MINRES default 1 (BackwardEuler.h:62) */
    double linear_solve_tolerance_scale; /* NewtonsMethod.h:38, default 1 */
    /* ADMM (integrator = ZMPM_ADMM); AdmmSimulationFoam.h:47-70 */
    int32_t integrator;             /* zmpm_integrator, default NEWTON */
    int32_t admm_iterations;        /* admm_max_iterations (class default 100; scenes 15-40) */
    double admm_rho_scale;          /* rho_scale, default 0.5 */
    double admm_local_tolerance;    /* local_tolerance of the per-particle Newton, default 1e-8 */
    double admm_global_tolerance;   /* global_tolerance: absolute MINRES tolerance, default 1e-6 */
    int32_t admm_global_max_iterations; /* global_max_iteration, default 10000 */
    int32_t trial_collision;        /* EXPLICIT: useTrialCollision (MpmSimulationBase.cpp:61, default 1) */
    int32_t mls_mpm;                /* EXPLICIT only: MLS-MPM force and velocity gradient (MpmSimulationBase.h:66,
                                       MpmSimulationBase.cpp:102-106, :527-541, :947-961), default 0 */
    int32_t pad1;
} zmpm_solver;

typedef struct zmpm_collider {
    int32_t shape; /* zmpm_collider_shape */
    int32_t type;  /* zmpm_collider_type */
    double friction;
    /* material-space level set: HALF_SPACE origin=a, outward normal=b;
       SPHERE center=a, radius=radius; BOX min corner=a, max corner=b */
    double a[3];
    double b[3];
    double radius;
    /* rigid motion x = R s X + t (CollisionObject.cpp:340-400); the reference's
       updateState callback is replaced by linear-in-time translation and scale:
       t(time) = translation + time*translation_velocity, s = scale + time*scale_velocity */
    double rotation[4]; /* quaternion w,x,y,z */
    double angular_velocity[3];
    double translation[3];
    double translation_velocity[3];
    double scale;
    double scale_velocity;
} zmpm_collider;

typedef struct zmpm_stats {
    int32_t newton_iterations;   /* Newton iterations that ran a linear solve */
    int32_t krylov_iterations;   /* summed over Newton iterations */
    int32_t hvp_count;           /* Hessian-vector products evaluated */
    int32_t cfl_violation;       /* 1 if a particle moved more than dx */
    int32_t newton_converged;    /* 1 if the Newton norm fell below tolerance */
    int32_t status_flags;        /* bit 0: NaN seen, bit 1: bounded wait gave up */
    int64_t num_particles;
    int64_t num_groups;          /* particle groups (one per touched page) */
    int64_t num_blocks;          /* pages in the page map */
    int64_t num_nodes;           /* grid nodes with m != 0 */
    int64_t num_collision_nodes;
    double newton_residual_initial;
    double newton_residual_final;
    double ms_total;             /* device time of the substep */
    double ms_hvp;               /* summed device time of the persistent linear-solve kernels
                                    that iterated (only with zmpm_set_profiling on); each
                                    Krylov iteration there is one Hessian-vector product
                                    with its node passes */
    int32_t hvp_timed;           /* Krylov iterations (= products) in ms_hvp */
    int32_t kernel_launches;     /* CUDA kernels this library launched for the substep */
    int32_t phase_field_iterations; /* CG iterations of the phase-field solve (its `iterations` return) */
    int32_t fp64_residual;       /* MIXED: 1 if the Newton residual went to FP64 after the FP32 one stalled */
    double phase_field_residual; /* final |r|_2 of the phase-field CG */
    int64_t rankine_first_not_max; /* ZMPM_DAMAGE_RANKINE_REFERENCE particles whose first eigenvalue
                                      (the reference's sigma_max) is not the largest one */
    int64_t svd_fp64_reevaluations; /* MIXED: particle constitutive updates of the Newton solve redone in
                                       FP64 because their FP32 singular values were near inversion
                                       (|sigma2| <= 0.2) or strongly stretched (sigma0 >= 5) */
} zmpm_stats;

/* Result of the binning pass (sortParticlesAndPolluteGrid,
   Lib/MPM/MpmSimulationBase.cpp:1032-1103); caller-allocated arrays sized from
   zmpm_bin_counts.  Any pointer may be NULL. */
typedef struct zmpm_bin_result {
    uint64_t* particle_sorter;       /* [P] sorted keys */
    int32_t* particle_order;         /* [P] */
    uint64_t* particle_base_offset;  /* [P] indexed by particle */
    int32_t* particle_group;         /* [G][2] first,last (inclusive) */
    uint64_t* block_offset;          /* [G] page index of each group */
    uint64_t* page_offsets;          /* [B] page map blocks, first-touch order */
} zmpm_bin_result;

/* ------------------------------------------------------------ lifecycle ----- */
/* replaces MpmSimulationBase ctor + initialize (MpmSimulationBase.cpp:33-144) */
int zmpm_create(const zmpm_config* cfg, zmpm_ctx** out);
int zmpm_destroy(zmpm_ctx* ctx);
const char* zmpm_last_error(const zmpm_ctx* ctx);
const char* zmpm_status_string(int status);

/* ----------------------------------------------------- scene / plugin API --- */
/* Appends particles (the sampling helpers' output, MpmInitializationHelper.h);
   F = I, C = 0.  *lower receives the handle's first index
   (MpmParticleHandleBase ctor, MpmParticleHandleBase.cpp:1-60). */
int zmpm_add_particles(zmpm_ctx* ctx, int64_t count, const double* x, const double* v,
    const double* mass, const double* volume, int64_t* lower);

/* MpmParticleHandleBase::addFBasedMpmForce (MpmParticleHandleBase.cpp:77-90):
   attaches a constitutive model built from (E, nu) to particles [lower, upper). */
int zmpm_add_fbased_force(zmpm_ctx* ctx, int64_t lower, int64_t upper, int32_t model,
    double youngs_modulus, double poisson_ratio);

/* Per-particle Lame parameters (each reference particle owns its model copy,
   MpmParticleHandleBase.cpp:470).  For NeoHookeanBorden lambda is converted to
   kappa = 0.666666 mu + lambda as NeoHookeanBorden.cpp:20 does. */
int zmpm_set_lame(zmpm_ctx* ctx, int64_t lower, int64_t upper, const double* mu,
    const double* lambda);

/* MpmParticleHandleBase::addPlasticity (MpmParticleHandleBase.cpp:331-348). */
int zmpm_add_plasticity(zmpm_ctx* ctx, int64_t lower, int64_t upper, int32_t kind,
    double yield_stress, double xi, double fail_stress);
/* DruckerPragerStvkHencky(friction_angle [degrees], beta, cohesion,
   volume_correction) (PlasticityApplier.cpp:247-261; defaults 30, 1, 0, 1) on
   StvkWithHenckyIsotropic particles [lower, upper); log Jp starts at 0. */
int zmpm_add_drucker_prager(zmpm_ctx* ctx, int64_t lower, int64_t upper, double friction_angle, double beta, double cohesion,
    int32_t volume_correction);
/* NonAssociativeCamClay(logJp, friction_angle [degrees], beta, xi, dim = 3,
   hardeningOn) (PlasticityApplier.cpp:10-20) on NeoHookeanBorden particles. */
int zmpm_add_cam_clay(zmpm_ctx* ctx, int64_t lower, int64_t upper, double log_jp, double friction_angle, double beta, double xi,
    int32_t hardening);
/* log Jp of Drucker-Prager and Cam-Clay particles (particle order; 0 otherwise). */
int zmpm_get_log_jp(zmpm_ctx* ctx, double* log_jp);

/* Damage on particles [lower, upper) that use NeoHookeanBorden: the phase
   field of MpmParticleHandleBase::addFBasedMpmForceWithPhaseField
   (MpmParticleHandleBase.cpp:92-118: c = 1, residual_phase) and
   FractureSimulation::sigmaF (FractureSimulation.h:52). */
int zmpm_add_damage(zmpm_ctx* ctx, int64_t lower, int64_t upper, int32_t kind, double sigma_f, double residual_phase);
/* Phase-field value c per particle (1 undamaged, 0 fully damaged). */
int zmpm_get_damage(zmpm_ctx* ctx, double* c);

/* CD-MPM phase field on NeoHookeanBorden particles [lower, upper):
   MpmParticleHandleBase::addFBasedMpmForceWithPhaseField(percentage, l0, model,
   allow_damage) (MpmParticleHandleBase.cpp:92-118): c = 1, H = 0, l0,
   1/sigma_c = 1 / psi((1 + percentage) I) (PhaseField::Get_Sigma_C_Based_On_Max_Deformation,
   PhaseField.h:58-68), pf_Fp = 1, H_max = +max, vol = V0, allow_damage; residual
   phase k (the reference fixes 0.001).  Sets the particles' damage kind to
   ZMPM_DAMAGE_PHASE_FIELD. */
int zmpm_add_phase_field(zmpm_ctx* ctx, int64_t lower, int64_t upper, double percentage, double l0, int32_t allow_damage,
    double residual_phase);
/* FractureSimulation members of the phase-field solve: parabolic_M (0: elliptic),
   lumping (default 1), delete_particle_threshold (default 0; particles with
   c < threshold are parked at (4, 4, 4) with V = 0, F = I, no further damage,
   FractureSimulation.h:172-207), and the CG's max_iterations (100) and absolute
   tolerance (1e-6), FractureSimulation.h:61-63, :444-446. */
int zmpm_set_phase_field_solver(zmpm_ctx* ctx, double parabolic_M, int32_t lumping, double delete_threshold, int32_t cg_max_iterations,
    double cg_tolerance);
/* Per-particle phase-field state (particle order); any pointer may be NULL. */
int zmpm_get_phase_field(zmpm_ctx* ctx, double* c, double* H, double* pf_Fp, double* vol);
/* Replaces 1/sigma_c per particle (the host side of randomizePhaseFieldSigmaC /
   voronoiSigmaC, MpmParticleHandleBase.cpp:120-200). */
int zmpm_set_phase_field_sigma_c(zmpm_ctx* ctx, const double* one_over_sigma_c);

/* MpmParticleHandleBase::addFElasticNonequilibratedBasedMpmForce
   (MpmParticleHandleBase.cpp:468-478) with the reference's only instantiated
   model, StvkWithHencky(E, nu) (StvkWithHencky.cpp:10-20): a second elastic
   strain Fe ("Fe_Nonequilibrated", starts at I) that G2P advects and relaxes by
   the viscous return map of FElasticNonequilibratedBasedMpmForceHelper::
   evolveStrain (FElasticNonequilibratedBasedMpmForceHelper.h:62-87).  Its
   energy enters the ADMM local step (AdmmSimulationFoam.h:575-612).  Every
   particle in [lower, upper) must already carry StvkWithHenckyIsotropic;
   StvkWithHencky has no stress differential (StvkWithHencky.cpp:185-190), so a
   Newton substep over such particles returns ZMPM_BAD_ARG. */
int zmpm_add_viscoelastic(zmpm_ctx* ctx, int64_t lower, int64_t upper, double youngs_modulus, double poisson_ratio,
    double viscosity_d, double viscosity_v);
/* Fe per particle, [P][3][3] in particle-index order (I where none is attached). */
int zmpm_get_viscoelastic_strain(zmpm_ctx* ctx, double* Fe);
int zmpm_set_viscoelastic_strain(zmpm_ctx* ctx, const double* Fe);

/* MpmSimulationBase::addCollisionObject (MpmSimulationBase.cpp:80-84). */
int zmpm_add_collision_object(zmpm_ctx* ctx, const zmpm_collider* obj, int32_t* id);
/* Replaces a collider description (the reference's updateState callback). */
int zmpm_set_collision_object(zmpm_ctx* ctx, int32_t id, const zmpm_collider* obj);

/* ---------------------------------------------------------- state I/O ------- */
/* Copy particle state to/from host arrays in particle-index order.  Any pointer
   may be NULL.  x,v: [P][3]; C,F: [P][3][3]. */
int zmpm_get_particles(zmpm_ctx* ctx, double* x, double* v, double* C, double* F);
int zmpm_set_particles(zmpm_ctx* ctx, const double* x, const double* v, const double* C,
    const double* F);
/* Plastic state per particle (VonMisesStvkHencky::yield_stress, broken). */
int zmpm_get_plastic_state(zmpm_ctx* ctx, double* yield_stress, int32_t* broken);
int64_t zmpm_num_particles(const zmpm_ctx* ctx);
double zmpm_time(const zmpm_ctx* ctx);

/* -------------------------------------------------------------- substep ----- */
/* MpmSimulationBase::advanceOneTimeStep, implicit branch
   (MpmSimulationBase.cpp:256-296): reinitialize (sort + page map) -> P2G ->
   backward-Euler Newton (MINRES/CG, matrix-free Hessian) -> G2P ->
   evolveStrain -> plasticity.  stats may be NULL. */
int zmpm_substep(zmpm_ctx* ctx, double dt, const zmpm_solver* solver, zmpm_stats* stats);

/* The implicit substep in the phases a reference subclass can override
   (MpmSimulationBase virtuals, Lib/MPM/MpmSimulationBase.h:133-229; the
   sequence of advanceOneTimeStep's implicit branch, MpmSimulationBase.cpp:
   282-295).  zmpm_substep(ctx, dt, s, st) equals
     zmpm_particles_to_grid(ctx, dt, s); zmpm_backward_euler_step(ctx, st);
     zmpm_grid_to_particles(ctx, 1, st);
   and a caller may run its own work between the calls (a fracture hook after
   particlesToGrid, its own plasticity after gridToParticles).  Newton and ADMM
   integrators only (ZMPM_UNSUPPORTED for ZMPM_EXPLICIT); a call out of order
   returns ZMPM_NOT_READY, and a particle or plugin edit between the calls ends
   the sequence.

   reinitialize + particlesToGrid (MpmSimulationBase.cpp:146-230, 437-486): the
   sort and page map, APIC P2G, the registered damage hook
   (FractureSimulation::particlesToGrid, FractureSimulation.h:149-160) and the
   Newton start (startBackwardEuler, :610-633) for step dt. */
int zmpm_particles_to_grid(zmpm_ctx* ctx, double dt, const zmpm_solver* solver);
/* backwardEulerStep (MpmSimulationBase.cpp:635-657), or AdmmSimulation's ADMM
   solve when solver->integrator is ZMPM_ADMM, on the grid of the last
   zmpm_particles_to_grid; fills the Newton fields of stats (may be NULL). */
int zmpm_backward_euler_step(zmpm_ctx* ctx, zmpm_stats* stats);
/* gridToParticles(dt) (MpmSimulationBase.cpp:879-1016): G2P, the particle
   advection and CFL check, evolveStrain, and with apply_plasticity != 0 the
   return maps of applyPlasticity (:1018-1030) in the same pass.  Ends the
   substep: the context's time advances by dt; ZMPM_CFL_VIOLATION as
   zmpm_substep. */
int zmpm_grid_to_particles(zmpm_ctx* ctx, int32_t apply_plasticity, zmpm_stats* stats);
/* MpmSimulationBase::applyPlasticity (MpmSimulationBase.cpp:1018-1030) alone:
   every particle's plasticity return map on its current F. */
int zmpm_apply_plasticity(zmpm_ctx* ctx);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
   caller can order its own work or CUDA events against the substep. */
int zmpm_get_stream(zmpm_ctx* ctx, void** stream);
/* Polls of a grid-wide barrier of the persistent Krylov kernel before the wait
   gives up (0: the default, 2^22, about a second).  A wait that gives up makes
   every CTA of the kernel return and the substep report ZMPM_TIMEOUT; the
   context stays usable.  (The reference runs on one host thread and has no
   device waits.) */
int zmpm_set_spin_limit(zmpm_ctx* ctx, int64_t polls);

/* on != 0: run the Newton loop host-driven (every kernel a plain launch, no
   CUDA graph) and bracket each linear solve's persistent kernel with CUDA
   events; zmpm_stats.ms_hvp reports their summed device time and hvp_timed
   the Krylov iterations they ran (the reference's ZIRAN_TIMER scopes,
   Lib/Ziran/CS/Util/Timer.h:34-58, as device timers).  ADMM substeps run
   their iteration loop host-driven too. */
int zmpm_set_profiling(zmpm_ctx* ctx, int32_t on);

/* ------------------------------------------------------------ adjoint ------ */
/* Reverse mode of one implicit substep (no reference counterpart: ziran2019 has
   no differentiation).  The context holds the state s_n; the call runs the
   substep forward from s_n (the context then holds s_{n+1}) and maps the
   gradients of a scalar loss with respect to s_{n+1} to gradients with respect
   to s_n in place: gx, gv [P][3], gC, gF [P][3][3] in particle-index order
   (NULL means zero).  gE [P] accumulates dL/dE_p, the Young's modulus at fixed
   Poisson ratio (mu and lambda scale with E).  The derivative is the hand-written
   adjoint of P2G, of the converged Newton solution through the implicit
   function theorem, of G2P (quadratic B-spline weights, their gradients and
   Hessians) and of the von Mises return map (VonMisesStvkHencky with xi = 0 on
   StvkWithHenckyIsotropic particles; the projection is differentiated as an
   isotropic function of the trial F, and dL/dE includes the yield radius'
   dependence on mu): the adjoint system (M + dt^2 K) lambda = g uses the
   substep's own symmetric Hessian, solved in FP64 by CG to the relative
   `adjoint_tolerance`.  Binning is held fixed (piecewise constant in x).
   Returns ZMPM_UNSUPPORTED for other plasticity (hardening, Drucker-Prager,
   Cam-Clay), damage, viscoelastic particles or the ADMM integrator. */
int zmpm_adjoint_substep(zmpm_ctx* ctx, double dt, const zmpm_solver* s, double adjoint_tolerance, double* gx, double* gv, double* gC,
    double* gF, double* gE, zmpm_stats* stats);

/* Device-resident checkpoints of the full particle state and time (for
   checkpointed adjoint rollouts).  slot >= 0; a slot is allocated on first
   save and kept until zmpm_destroy. */
int zmpm_checkpoint_save(zmpm_ctx* ctx, int32_t slot);
int zmpm_checkpoint_load(zmpm_ctx* ctx, int32_t slot);

/* MpmSimulationBase::evalMaxParticleSpeed (MpmSimulationBase.cpp:1143-1166):
   the largest particle speed and the particles' bounding box (any pointer may
   be NULL). */
int zmpm_max_particle_speed(zmpm_ctx* ctx, double* speed, double* min_corner, double* max_corner);
/* MpmSimulationBase::calculateDt (MpmSimulationBase.cpp:766-790): cfl dx / v,
   v the larger of the particle speed and the colliders' evalMaxSpeed
   (CollisionObject.cpp:159-196) over the particles' box grown by 4 dx; max_dt
   when nothing moves.  cfl is the config's.  The frame-boundary clamp of
   TimeStepping::nextDt is the caller's (the Python TimeStepping mirrors it). */
int zmpm_calculate_dt(zmpm_ctx* ctx, double max_dt, double* dt);

/* Restart files: the role of SimulationBase::write / read with
   MpmSimulationBase::writeState / readState (SimulationBase.h:146-187,
   MpmSimulationBase.cpp:725-761).  The library's own versioned binary format
   (every per-particle array by name, the colliders, the phase-field solver
   settings and the time), not the reference's DataManager stream, whose
   attribute order follows a hash map.  read_state replaces the context's
   particles; the context must have the file's dx and grid size. */
int zmpm_write_state(zmpm_ctx* ctx, const char* path);
int zmpm_read_state(zmpm_ctx* ctx, const char* path);

/* The reference's restart directory (SimulationBase::write, read and
   outputFileName, SimulationBase.h:146-199).  write_restart creates
   output_dir if needed and writes there restart_<frame>.dat
   (restart_<frame>_<substep>.dat when substep > 0; zmpm_write_state's
   format), then last_written.txt holding the frame and binary_ver.txt
   holding ZMPM_BINARY_VER.  read_restart reads binary_ver.txt (0 when it is
   missing) and fails with ZMPM_BAD_ARG when it is newer than
   ZMPM_BINARY_VER, stores last_written.txt's frame in *last_written_frame
   (-1 when missing; the reference warns when it is below `frame`, stale
   data), then reads the state file.  last_written_frame may be NULL. */
#define ZMPM_BINARY_VER 1
int zmpm_write_restart(zmpm_ctx* ctx, const char* output_dir, int32_t frame, int32_t substep);
int zmpm_read_restart(zmpm_ctx* ctx, const char* output_dir, int32_t frame, int32_t substep, int32_t* last_written_frame);

/* Particle output in Houdini's binary geometry point format (BGEO version 5,
   uncompressed, big-endian), as the reference writes it through Partio:
   writePartio (PartioIO.h:138-182) stores "position"; FractureSimulation's
   frame dump (FractureSimulation.h:110-146) adds "pf" and "sigmaC". */
enum zmpm_bgeo_fields {
    ZMPM_BGEO_POSITION = 0,     /* position only */
    ZMPM_BGEO_VELOCITY = 1,     /* + "v" (3 floats) */
    ZMPM_BGEO_PHASE_FIELD = 2   /* + "pf" and "sigmaC" (1 float each; 1 without a phase field) */
};
int zmpm_write_bgeo(zmpm_ctx* ctx, const char* path, int32_t fields);

/* Default solver settings of the reference (MpmSimulationBase.cpp:51,
   BackwardEuler.h:56-62, LinearSolver.h:24). */
void zmpm_default_solver(zmpm_solver* s, int32_t linear_solver, int32_t precision);

/* -------------------------------------------------------------- hooks ------- */
/* Binning only (sortParticlesAndPolluteGrid).  counts: [P, G, B]. */
int zmpm_bin(zmpm_ctx* ctx, int64_t* counts);
int zmpm_bin_fetch(zmpm_ctx* ctx, zmpm_bin_result* out);

/* Runs reinitialize + particlesToGrid + startBackwardEuler for time step dt
   (MpmSimulationBase.cpp:610-633) and stops, so the hooks below can evaluate
   the Newton objective.  num_nodes receives N. */
int zmpm_begin_implicit(zmpm_ctx* ctx, double dt, int64_t* num_nodes);
/* Grid after P2G in node-index order (getNumNodes numbering, MpmGrid.h:123-136):
   m [N], v [N][3], coord [N][3]. */
int zmpm_get_grid(zmpm_ctx* ctx, double* m, double* v, int32_t* coord);
/* Initial Newton guess dv [N][3] and collision projection flags [N]. */
int zmpm_get_initial_dv(zmpm_ctx* ctx, double* dv, int32_t* collided);
/* BackwardEulerLagrangianForceObjective::updateState + computeResidual +
   computeNorm (BackwardEuler.h:101-175): residual [N][3], norm may be NULL. */
int zmpm_residual(zmpm_ctx* ctx, const double* dv, double* residual, double* norm);
/* BackwardEulerLagrangianForceObjective::multiply (BackwardEuler.h:322-351),
   matrix-free (M + dt^2 K) x at the state of the last zmpm_residual call.
   fp32 != 0 evaluates the Hessian-vector product in FP32 (MIXED contexts). */
int zmpm_multiply(zmpm_ctx* ctx, const double* x, double* b, int32_t fp32);

/* --------------------------------------------------- allocation-free ----- */
/* Largest particle count zmpm_sort_keys_noalloc accepts. */
#define ZMPM_NOALLOC_MAX_PARTICLES 262144

/* This entry point has no counterpart in the reference.  It is for callers that
   cannot call cudaMalloc (a host that owns all device memory and forbids new
   allocations, or a loop that cannot take cudaMalloc's implicit device
   synchronisation): it computes the particle keys of the binning pass
   (sortParticlesAndPolluteGrid's key and sort) for n particles and sorts them,
   allocating nothing.
     x      device array [n][3] of positions (row-major, like the host arrays)
     keys   device array [n]; receives the sorted keys, bit-identical to
            zmpm_bin_result.particle_sorter of a context with the same
            precision, layout, grid_log2 and dx
     stream cudaStream_t to run on (NULL = the default stream)
   Scratch memory is one fixed device array inside the library (about 2.2 MB on
   every GPU that loads it, kept until exit); n above
   ZMPM_NOALLOC_MAX_PARTICLES is rejected with ZMPM_BAD_ARG.  The first call
   on each device looks up that array's device address and keeps it for the
   life of the process, so do not use this call after resetting the device
   (cudaDeviceReset).  Calls share the array: calls that overlap on the GPU
   race.  Returns ZMPM_OUT_OF_GRID if a particle's stencil leaves the grid or a
   coordinate is not finite.  The call synchronises `stream` and reads a status
   word back to the host before it returns, so it cannot be made inside a
   stream capture. */
int zmpm_sort_keys_noalloc(const double* x, int64_t n, double dx, int32_t precision, int32_t layout, int32_t grid_log2,
    uint64_t* keys, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ZMPM_H */
