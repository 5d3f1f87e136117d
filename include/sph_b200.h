/*
 * sph_b200.h -- C-ABI of libsph_b200, the B200 (sm_100a) weakly-compressible
 * SPH time step of SPH-2D.
 *
 * The reference host (Fortran 90, one MPI rank per subdomain) calls
 * argument-less subroutines that read and write module globals:
 *   find_particle_pair()                          Taylor_Green_Vortex/find_particle_pair.f90:21-163
 *   Define_freesurface_and_Normailized_derivates() Taylor_Green_Vortex/Define_freesurface_and_Normailized_derivates.f90:21-443
 *   Solver_Normalized_*()                         Taylor_Green_Vortex/Solver_Normalized_Modified_Linear_Riemann_Delta_SPS.f90:23-639
 *                                                 Taylor_Green_Vortex/Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS.f90
 *   single_step_compute(i_time_step)              Taylor_Green_Vortex/single_step_compute.f90:19-301
 *   time_iteration()  (Runge-Kutta branch)        Taylor_Green_Vortex/time_iteration.f90:781-1159
 *   Shift_particle_position(i_time_step)          Taylor_Green_Vortex/Shift_particle_position.f90:21-137
 *   Distribute_Period_Boundary_Particle(i)        Taylor_Green_Vortex/Distribute_Period_Boundary_Particle.f90:21-269
 * Each entry point below replaces one of them (cited per function).  The
 * Fortran shim passes its module arrays (column-major (n,2) = all x then all
 * y), the particle counts and an sph_config filled from information_module.
 *
 * Conventions
 *   - Every function returns int: 0 (SPH_OK) or a negative SPH_E_* code; the
 *     library never aborts the process and never traps on the device.
 *   - Host pointers are owned by the caller; the library copies from / to
 *     them and never keeps them.
 *   - Particle indices crossing the ABI are 1-based (Fortran) in pair lists.
 *   - One handle per host thread; a handle is not thread-safe.
 */
#ifndef SPH_B200_H
#define SPH_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SPH_OK            0
#define SPH_E_ARG        -1   /* null pointer, n <= 0, n > capacity, ...   */
#define SPH_E_CAPACITY   -2   /* pair / particle / cell capacity exceeded   */
#define SPH_E_NONFINITE  -3   /* NaN/Inf produced in the state               */
#define SPH_E_CUDA       -5   /* a CUDA runtime call failed                  */
#define SPH_E_TIMEOUT    -6   /* reserved: no kernel of this library waits on
                                 another block, launch or device, so no wait can
                                 time out; never returned                         */
#define SPH_E_CONFIG     -7   /* unsupported configuration value             */
#define SPH_E_DOMAIN     -8   /* a particle left the cell grid               */
#define SPH_E_SKIN       -9   /* a particle moved further than the cell skin */
#define SPH_E_NODEVICE  -10   /* no CUDA device / extension not usable       */

/* ---- enumerations ------------------------------------------------------ */
/* Kernel_function_model values of Moving_Square.../Compute_Kernel.f90:56-255 */
#define SPH_KERNEL_GAUSSIAN   4   /* improved Gaussian, support 3h           */
#define SPH_KERNEL_WENDLAND2  5   /* Wendland C2, support 2h                 */

/* Solver_* variants (which `call Solver_...` line is live) */
#define SPH_SOLVER_MODLR_DELTA_SPS  0 /* Solver_Normalized_Modified_Linear_Riemann_Delta_SPS (TGV default) */
#define SPH_SOLVER_MUSCL_DELTA_SPS  1 /* Solver_Normalized_MUSCL_Linear_Riemann_Delta_SPS                 */
#define SPH_SOLVER_MS_MODLR_DELTA   2 /* Moving_Square.../Solver_Normalized_Modified_Linear_Riemann_Delta (MS default) */
#define SPH_SOLVER_MS_HLLC_DELTA    3 /* Moving_Square.../Solver_Normalized_HLLC_Riemann_Delta                     */
#define SPH_SOLVER_DELTA_SPS        4 /* Taylor_Green_Vortex/Solver_Normalized_Delta_SPH_SPS (no Riemann state:
                                         pair-mean pressure and velocity, Antuono delta-SPH diffusion,
                                         no XSPH; its energy equation, which nothing else reads under the
                                         Tait EOS, is not integrated)                                   */

#define SPH_EOS_TAIT    0   /* Status_Equation.f90:56-66  p = B((rho/rho0)^7-1) + pb */
#define SPH_EOS_LINEAR  1   /* Status_Equation.f90:69-76  p = c0^2 (rho-rho0) + pb   */

#define SPH_PAIRS_ONE_FLUID   0 /* TGV find_particle_pair.f90:76  keep if i or j is fluid     */
#define SPH_PAIRS_NO_SAME_BND 1 /* MS  Find_particle_pair.f90:73-75 drop -2/-2, -3/-3, -201/-201 */

#define SPH_PREC_FP64   0   /* every field and pair term in FP64                     */
#define SPH_PREC_MIXED  1   /* FP32 pair arithmetic summed in FP64, FP64 state         */

#define SPH_INTEGRATOR_RK4_REUSE 0 /* time_iteration.f90:781-1159 (3 RHS/step after step 1) */
#define SPH_INTEGRATOR_EULER_PC  1 /* Moving_Square.../SPH_Time_Iteration.f90:304-334, Iteration_Method 2 (1 RHS/step) */

/* particle type labels (Information_Module.f90 of the moving-square case) */
#define SPH_TYPE_WATER     2
#define SPH_TYPE_PERIODIC  -101
#define SPH_TYPE_ILL       120
#define SPH_TYPE_FIX_GHOST  -3
#define SPH_TYPE_BODY       -4   /* Body_Particle_Label: an initial type (body force) */
#define SPH_TYPE_INLET    -201

/* ---- configuration (filled once from information_module) ------------- */
typedef struct sph_config {
    int    kernel_model;      /* SPH_KERNEL_*                                        */
    int    solver;            /* SPH_SOLVER_*                                        */
    int    eos;               /* SPH_EOS_*                                           */
    int    pair_rule;         /* SPH_PAIRS_*                                         */
    int    precision;         /* SPH_PREC_*                                          */
    int    renormalize;       /* 0: reference (inverse replaced by I), 1: true inverse */
    int    reference_literals;/* 1: default-real literals of the reference (PI, 1e-7..) */
    int    periodic;          /* 1: device-generated periodic images each step       */
    int    shifting;          /* 1: Shift_particle_position after each step          */
    int    integrator;        /* SPH_INTEGRATOR_*                                    */
    double kernel_scale;      /* kernel_scale (support = kernel_scale * h)           */
    double h;                 /* smooth_length (uniform)                             */
    double dx;                /* interior_dx (SPS filter width, shift cap unit)      */
    double rho0;              /* water_rho_0                                         */
    double c0sq;              /* square_c_0                                          */
    double background_p;      /* Background_Pressure                                 */
    double nu;                /* water_kinematic_viscosity (Morris Laplacian)        */
    double alpha, beta, fai;  /* Monaghan artificial viscosity alpha, beta, fai_coefficient */
    double delta;             /* delta-SPH density diffusion coefficient             */
    double delta_alpha;       /* Delta_alpha (artificial internal acceleration)      */
    double xsph_eps;          /* epsilon (XSPH)                                      */
    double shift_beta, shift_R, shift_max; /* shift_belta, shift_R, max_shift        */
    int    shift_n;           /* shift_n                                             */
    double fs_threshold;      /* volume fraction at or below which a particle is a surface candidate (0.65) */
    double box_lo[2], box_hi[2];   /* periodic box (Period_Boundary_*_Min/Max)       */
    double grid_lo[2], grid_hi[2]; /* extent every particle must stay inside         */
    double cell_skin;         /* extra cell width as a fraction of the support (>= 0) */
    int    laplacian;         /* laplacianTerm: 1 Morris, 0 Monaghan (moving-square solvers) */
    int    free_surface;      /* Has_FreeSurface_Or_Not: 1 detect free-surface particles, 0 none */
    /* MLS density re-initialisation (Reinitialize_particle_density), run after the
     * integrator update and before shifting of every mls_every-th step:
     * mls_order 0 off, 1 the Shepard-normalised mass sum over the step's last
     * pair list (sum m_j W_ij / sum W_ij V_j over same-type pairs), 3 linear or
     * 6 quadratic moving least squares (RefreshDensity_MLS_Order),
     * mls_every = MLS_time_step / RefreshDensity_time_step,
     * mls_alpha = slighted_modified_alpha (the moment matrix gets alpha^3 on its diagonal). */
    int    mls_order;
    int    mls_every;
    double mls_alpha;
    /* Fixed-ghost and body-ghost assignment of the moving-square driver
     * (Moving_Square.../Assign_boundary_particles.f90:611-941), run at the start of
     * every right-hand side when ghost_assign = 1; 0 leaves the ghost states to
     * the host.  Shepard interpolation (MLS_order_Boundary = 1) over the non-ghost
     * particles within kernel_scale * ghost_h_factor * h (ghost_h_factor = 1.2),
     * mirrored velocities by wall label (sph_set_boundary_labels), the body's
     * prescribed velocity (sph_set_body_motion). */
    int    ghost_assign;
    int    wall_bc;               /* ExternalBoundaryCondition: 1 free slip, 0 no slip  */
    double ghost_h_factor;
    double shock_release_time;    /* Shock_wave_release_time                           */
    double gravity[2];            /* Gravity_grad                                      */
} sph_config;

/* diagnostics returned by sph_step (reductions in FP64) */
typedef struct sph_diag {
    double kinetic_energy;    /* sum 0.5 m |v|^2 over water particles (Sampling_subroutine.f90:346-349) */
    double max_speed;         /* max |v| over water particles                       */
    long long pair_count;     /* pairs seen by the last RHS evaluation              */
    int    n_images;          /* periodic images generated at the last step start   */
    int    n_surface;         /* free-surface particles at the last RHS evaluation  */
    double body_force[6];     /* pressure x,y; viscous x,y; total x,y of the last RHS (FP64,
                                 Moving_Square.../Calculate_Body_Force.f90:53-142 and
                                 Single_step_compute.f90:228-243); zero without body particles */
} sph_diag;

/* per-pass device times (CUDA events) accumulated since the last reset, ms */
typedef struct sph_timings {
    double sort_ms, pass_a_ms, surface_ms, pass_c_ms, update_ms, images_ms, total_ms;
    long long rhs_evaluations, steps;
    long long kernel_launches;  /* libsph_b200 kernels launched (library sort/scan calls not counted) */
    double adjoint_ms;          /* reverse kernels of sph_adjoint_backward */
} sph_timings;

typedef struct sph_handle sph_handle;

/* Allocate device buffers for up to n_capacity host particles (plus their
 * periodic images) and validate the configuration.  No reference counterpart:
 * the reference sizes static module arrays at compile time
 * (Taylor_Green_Vortex/information_module.f90:96-97, 286-302). */
int sph_init(const sph_config* cfg, int n_capacity, sph_handle** out);
int sph_free(sph_handle* h);

/* Upload the host particle state.  Replaces the copy of the global arrays
 * into the subdomain arrays (Taylor_Green_Vortex/Devide_block_and_send_tasks.f90:670-701).
 * pos, vel: [2n] column-major; rho, mass: [n]; type: [n] labels;
 * sps_mass: [n] or NULL -- the mass array the SPS force indexes with the
 * neighbour's subdomain index (Solver_..._SPS.f90:489-490 reads the global
 * particle_mass(j)); NULL means the particle's own mass. */
int sph_set_state(sph_handle* h, int n, const double* pos, const double* vel,
                  const double* rho, const double* mass, const int* type,
                  const double* sps_mass);

/* Overwrite position, velocity and density of the n host particles between
 * steps (the host's boundary / wave-maker modules own and may modify these
 * arrays) while keeping the integrator history: the rates the next step reuses
 * as K1 stay attached to their particles.  No reference counterpart: the
 * Fortran host writes its module arrays directly. */
int sph_update_state(sph_handle* h, int n, const double* pos, const double* vel, const double* rho);

/* subdomain_particle_initial_type for the n host particles: particles whose
 * initial type is SPH_TYPE_BODY form the body of the body-force integral
 * (Moving_Square.../Calculate_Body_Force.f90:60).  Without this call no body
 * force is computed. */
int sph_set_initial_type(sph_handle* h, int n, const int* initial_type);

/* subdomain_Boundary_particle_type for the n host particles: -6 horizontal
 * wall, -7 corner ("center"), -8 vertical wall, -9 along the cylinder, 0
 * anything else (Moving_Square.../Initial_Particle_From_First_Step.f90:220-300).
 * Used by the ghost assignment.  A -9 ghost keeps its interpolated velocity, as
 * in the reference: its radius_free_slip call (Assign_boundary_particles.f90:905,
 * Function_Module.f90:929-960) reads and writes the global particle arrays,
 * at the subdomain index and at fix_ghost_name, not the ghost's own velocity. */
int sph_set_boundary_labels(sph_handle* h, int n, const int* labels);

/* Custom_velocity and Custom_accleration of Body_Motion_Solver
 * (Moving_Square.../Body_Motion_Solver.f90:150-195) for the following steps: the
 * body particles (initial type SPH_TYPE_BODY) are translated by vel * dt at the
 * start of every step, their ghosts take vel, and acc enters the pressure
 * extrapolation onto them.  A host with a non-constant motion calls this before
 * every sph_step(h, 1, ...). */
int sph_set_body_motion(sph_handle* h, const double vel[2], const double acc[2]);

/* Real_physical_time of the next step's start, before its dt increment
 * (SPH_Time_Iteration.f90:71-72); sph_set_state resets it to 0. */
int sph_set_time(sph_handle* h, double t);

/* Download the host particles (same order as set_state).  press is the
 * equation of state evaluated at the returned density.  Any pointer may be NULL. */
int sph_get_state(sph_handle* h, int n, double* pos, double* vel, double* rho, double* press);

/* ---- snapshot streaming and restart (Output_for_tecplot.f90,
 * Output_for_Restart_Calculation.f90: the host's output modules keep writing
 * the files; the library delivers the state without stalling the step) -----
 *
 * sph_snapshot_begin queues a copy of the current state (the layout of
 * sph_get_state) into the given host buffers and returns at once: the state is
 * copied on the device in the step's stream order, and the transfer to the host
 * runs on a separate copy stream while later sph_step calls proceed.  The
 * buffers must stay valid until the snapshot completes; with page-locked
 * (cudaHostAlloc'd) buffers the transfer overlaps the steps, with pageable ones
 * it completes before the call returns.  A new snapshot first waits for the
 * previous one.  sph_snapshot_query returns SPH_OK when the last snapshot is
 * complete (or none was taken) and SPH_PENDING while it is in flight;
 * sph_snapshot_wait blocks until it is complete. */
#define SPH_PENDING 1
int sph_snapshot_begin(sph_handle* h, int n, double* pos, double* vel, double* rho, double* press);
int sph_snapshot_query(sph_handle* h);
int sph_snapshot_wait(sph_handle* h);

/* Exact restart: the whole per-particle and per-run state a later step depends
 * on (positions, velocities, densities, masses, SPS masses, types, initial
 * types, wall labels, the rates carried to the next step, the step count, the
 * physical time and the body motion), so that a handle restored from it
 * continues bit-identically to the one saved.  Little-endian binary: a 64-byte
 * header (magic "SPHB200R", version 1, n, then the step count, the time and the
 * body velocity and acceleration as doubles) followed by per-particle arrays in
 * set_state order: pos, vel (x, y pairs), rho, mass, smass (double), type,
 * itype, labels (int32), carried drho, acc, avg (double; acc and avg as x, y
 * pairs).  sph_restart_load needs a handle of the same configuration with
 * capacity for n; it replaces sph_set_state, sph_set_initial_type,
 * sph_set_boundary_labels, sph_set_time and sph_set_body_motion. */
size_t sph_restart_size(int n);
int sph_restart_save(sph_handle* h, void* buf, size_t bytes);
int sph_restart_load(sph_handle* h, const void* buf, size_t bytes);

/* find_particle_pair (Taylor_Green_Vortex/find_particle_pair.f90:21-163) on the
 * current state.  Writes up to pair_cap pairs (1-based, i<j in host/image index
 * order; images are numbered n+1.. in generation order), their kernel value
 * w and gradient dwdx ([2*pair_cap] column-major, may be NULL).  *pair_number
 * receives the total count; SPH_E_CAPACITY if it exceeds pair_cap. */
int sph_find_particle_pair(sph_handle* h, long long pair_cap, int* pair_i, int* pair_j,
                           double* w, double* dwdx, long long* pair_number);

/* One right-hand-side evaluation, i.e. the body of single_step_compute
 * (Taylor_Green_Vortex/single_step_compute.f90:62-171): EOS, pair search,
 * Define_freesurface_and_Normailized_derivates and the configured Solver_*,
 * then assembly.  Outputs for the n host particles (any may be NULL):
 * drhodt [n], acc [2n] (particle_acceleration), avg_vel [2n] (average_velocity),
 * fs [n] free-surface flag, near [n] near-free-surface flag. */
int sph_rhs(sph_handle* h, double* drhodt, double* acc, double* avg_vel, int* fs, int* near_fs);

/* nsteps time steps of the configured integrator (time_iteration,
 * Taylor_Green_Vortex/time_iteration.f90:781-1073): periodic wrap and images,
 * the stage updates, shifting.  The state stays on the device.  out may be NULL. */
int sph_step(sph_handle* h, int nsteps, double dt, sph_diag* out);

/* Kinetic energy and max |v| of the water particles
 * (Taylor_Green_Vortex/Sampling_subroutine.f90:340-356), FP64 reduction. */
int sph_diagnostics(sph_handle* h, sph_diag* out);

/* Intermediate per-particle fields of the last sph_rhs / RHS evaluation, for
 * the n host particles, column-major blocks.  They are the module arrays the
 * reference fills in Define_freesurface_and_Normailized_derivates and the
 * solvers (Taylor_Green_Vortex/Public_variable_module.f90): */
#define SPH_FIELD_FRA_V  0  /* [n]  subdomain_fra_v                                   */
#define SPH_FIELD_BINV   1  /* [4n] Tensor_dyadic_inverse_matrix (11,12,21,22 blocks)  */
#define SPH_FIELD_TAU    2  /* [3n] tao_xx, tao_xy, tao_yy                            */
#define SPH_FIELD_GRADS  3  /* [8n] grad_rho x,y; grad_pressure x,y; grad u x,y; grad v x,y */
int sph_get_field(sph_handle* h, int field, double* out);

int sph_get_timings(sph_handle* h, sph_timings* out);
int sph_reset_timings(sph_handle* h);

/* find_particle_pair for callers that cannot allocate GPU memory.  No
 * counterpart in the reference.  Hosts whose GPU memory is owned and pooled by
 * another framework, or that run where allocation is not allowed, pass their
 * own device buffers: d_pos [2n] column-major and d_type [n] as inputs,
 * d_pair_i/d_pair_j [pair_cap], d_w [pair_cap] and d_dwdx [2*pair_cap] (may be
 * NULL) as outputs -- the same contents and order sph_find_particle_pair
 * returns for a non-periodic configuration -- and *pair_number (host) receives
 * the pair count.  stream is a cudaStream_t (NULL: the legacy default stream).
 * The search works in a fixed static device array (about 2.4 MiB per GPU that
 * loads the library, held until exit) and calls no cudaMalloc / cudaFree:
 * at most 65536 particles and 65536 background cells of edge kernel_scale*h
 * over grid_lo..grid_hi; larger inputs return SPH_E_CAPACITY.  At most 256
 * pairs (i, j > i) per particle: beyond that it returns SPH_E_CAPACITY with
 * *pair_number = -1.  pair_cap = 0 counts only (SPH_OK); a pair_cap below the
 * count fills the first pair_cap pairs and returns SPH_E_CAPACITY.  Calls share
 * that array: GPU work of two calls must not overlap.  The first call on a
 * device resolves the array's address (cudaGetSymbolAddress) and keeps it for
 * the life of that device context; make it before any stream capture, and do
 * not call this entry point on a device after cudaDeviceReset.
 * cfg->periodic is ignored (no images are generated). */
int sph_find_particle_pair_noalloc(const sph_config* cfg, int n, const double* d_pos, const int* d_type,
                                   long long pair_cap, int* d_pair_i, int* d_pair_j, double* d_w,
                                   double* d_dwdx, long long* pair_number, void* stream);

/* ---- discrete adjoint of the time step (no counterpart in the reference) --
 * A forward/backward pair with the contract of an autograd function, for a
 * Fortran host that has no automatic differentiation: sph_adjoint_forward
 * runs nsteps steps from the handle's current state, keeps checkpoints of the
 * state every checkpoint_every steps inside the handle (the saved context)
 * and returns the loss; sph_adjoint_backward takes dL/dloss and returns the
 * gradient of the loss with respect to the state the forward started from
 * and to the viscosity.  The backward pass re-runs each checkpoint segment,
 * rebuilds every step's pair set from the recomputed positions and holds it
 * fixed while the reverse kernels run (the pair set is piecewise constant in
 * the positions; the gradient is that of the taken branches of max/min and
 * of the artificial-viscosity switch).  The handle's state after the backward
 * pass is the forward's final state.
 *
 * Device memory: besides the checkpoints, the handle keeps, while a segment
 * is reversed, the stage states of each of its steps, their sorted states
 * and, where that leaves 1 GiB free, what pass A computed for each RHS the
 * re-run evaluated (per step of a segment: about 20 bytes times max_nbr plus
 * 200 bytes per particle slot for each such RHS, three for the Runge-Kutta
 * driver and one for the Euler predictor-corrector).  When memory is short it
 * keeps less and recomputes instead; the gradient is the same either way.
 *
 * Supported configurations (others return SPH_E_CONFIG), either kernel, with
 * or without renormalisation:
 *  - the normalised modified linear Riemann and MUSCL linear Riemann delta-SPH
 *    + SPS solvers and the plain delta-SPH method (SPH_SOLVER_MODLR_DELTA_SPS
 *    without XSPH, SPH_SOLVER_MUSCL_DELTA_SPS, SPH_SOLVER_DELTA_SPS) with the
 *    RK4 driver, with or without particle
 *    shifting (the limiter, the capped shift and its density correction are
 *    differentiated on the branch the forward took), with or without the
 *    density re-initialisation (mls_order 3 or 6, moving least squares, its
 *    Shepard fallback differentiated where the forward took it; mls_order 1,
 *    the Shepard density on the last RHS's pairs); with the
 *    re-initialisation every step of a checkpoint segment must keep its states,
 *    else sph_adjoint_forward returns SPH_E_CAPACITY (lower checkpoint_every);
 *  - the moving-square modified linear Riemann and HLLC solvers
 *    (SPH_SOLVER_MS_MODLR_DELTA, SPH_SOLVER_MS_HLLC_DELTA; Morris laplacian,
 *    XSPH velocities in the continuity flux; the HLLC state on the sampled
 *    region and wave speeds the forward took) with the Euler
 *    predictor-corrector driver, with the library's ghost assignment
 *    (ghost_assign = 1: the reverse runs through the Shepard interpolation onto
 *    the wall and body ghosts) or with caller-given ghost states, with or
 *    without particle shifting after the corrector (the capped shift of the
 *    corrector RHS over its pairs, ghosts included), with or without the
 *    density re-initialisation (mls_order 3 or 6, the moving-square variant:
 *    W V weights, the particle itself counted, the ghosts' density and mass as
 *    the corrector RHS assigned them; mls_order 1 on the corrector RHS's pairs).
 * The reverse kernels compute in FP64 for both precisions of the forward step.
 *
 * Body motion: with body_motion set, step k of the forward run (k = 0 ..
 * nsteps-1) moves the body with velocity (body_motion[4k], body_motion[4k+1])
 * and acceleration (body_motion[4k+2], body_motion[4k+3]) (Custom_velocity and
 * Custom_accleration of Body_Motion_Solver at time t0 + (k+1) dt); NULL keeps
 * the handle's sph_set_body_motion values for every step.  After the backward
 * pass sph_adjoint_motion_gradient returns dL/d(body_motion), from which the
 * gradient with respect to any parametrisation of the motion (an amplitude,
 * Fourier coefficients) follows by the chain rule on the host. */
#define SPH_LOSS_VELOCITY_MISFIT 0  /* sum over water particles of |v - v_target|^2 */
#define SPH_LOSS_KINETIC_ENERGY  1  /* sum over water particles of m |v|^2 / 2       */
#define SPH_LOSS_DRAG            2  /* sum over the steps of dt * F_x, F = the total body force
                                       of the step's last RHS (sph_diag.body_force[4]);
                                       needs a body (sph_set_initial_type)             */
#define SPH_ADJ_NPARAMS 1           /* g_params[0] = dL/dnu                          */

typedef struct sph_adj_config {
    int nsteps;             /* time steps of the forward run                          */
    int checkpoint_every;   /* steps between state checkpoints (>= 1)                 */
    int loss;               /* SPH_LOSS_*                                             */
    int reserved;
    double dt;
    const double* target_vel;  /* [2*n] column-major (u block, v block); copied; misfit only */
    const double* body_motion; /* [4*nsteps] per-step body velocity and acceleration; copied;
                                  NULL: the handle's constant body motion            */
} sph_adj_config;

int sph_adjoint_forward(sph_handle* h, const sph_adj_config* cfg, double* loss);

/* Any output pointer may be NULL.  g_vel0 and g_pos0 are [2*n] column-major,
 * g_rho0 is [n], g_params is [SPH_ADJ_NPARAMS].  Returns SPH_E_ARG when no
 * forward context is held. */
int sph_adjoint_backward(sph_handle* h, double dloss, double* g_vel0, double* g_rho0, double* g_pos0,
                         double* g_params);

/* dL/d(body_motion) of the last backward pass, [4*nsteps] in the layout of
 * sph_adj_config.body_motion (zero when the run has no body or no ghost
 * assignment).  Returns SPH_E_ARG when no backward pass has completed. */
int sph_adjoint_motion_gradient(sph_handle* h, double* g_motion);

/* Human-readable message for a status code (static storage). */
const char* sph_strerror(int code);

#ifdef __cplusplus
}
#endif
#endif /* SPH_B200_H */
