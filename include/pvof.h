/*
 * pvof.h -- C ABI of the B200 implementation of PARTIES' two-phase
 * (diffuse-interface Cahn-Hilliard) RK3 substep.
 *
 * Every entry point takes plain pointers and sizes; no CUDA or torch type
 * appears here.  A context owns the device copy of the solver state.  Host
 * arrays exchanged with pvof_upload_field / pvof_download_field use the
 * reference's field layout: one contiguous block per field, element (i,j,k)
 * at ((k-Ks)*nJ + (j-Js))*nI + (i-Is), i fastest, where
 *   ghosted ("flow") fields span i in [-G, NX+G), j in [-G, NY+G),
 *     k in [-G, NZ+G)            (PARTIES/src/Memory.c:36-89), and
 *   no-ghost ("ng_") fields span i in [0, NX), j in [0, NY), k in [0, NZ)
 *                                (PARTIES/src/Memory.c:270-323),
 * with NX = NXM+1, NY = NYM+1, NZ = NZM+1 (a half cell is added at the far end
 * of every direction, PARTIES/src/Grid.c:60-64) and G = ghost_nodes = 3.
 * In the 2D modes NZM = 1 and the device keeps the k = 0 plane only; upload
 * reads the k = 0 plane of the block and download writes it to every plane
 * of the G range (the reference keeps those planes identical).
 *
 * The 3D mode (PVOF_GEOM_3D, the reference built without TWOD_* flags) keeps
 * every plane.  It supports x and z periodic with walls in y and no solids,
 * and the whole-substep entry points: pvof_create/destroy, the field copies,
 * pvof_set_stage, pvof_initialize, pvof_substep, pvof_run_steps,
 * pvof_liquid_mass and the measurement calls (launch count, timers, L2
 * flush, clamp total, solver timing).  Other entry points return PVOF_EINVAL on a 3D
 * context.  In 3D the fields C_G, rho and mu are download-only (they are
 * functions of C_L), *_EXPLICIT and *_VISC_EXPLICIT equal their _OLD copies
 * after a substep, and CH_RHS_CUR equals CH_RHS_N.
 *
 * Routine entry points keep the reference's names with a pvof_ prefix.  The
 * reference passes the RK stage and dt through Parameters (which_stage, dt);
 * here they are set once per substep with pvof_set_stage().
 *
 * Errors: functions return 0 (or a non-negative count) on success and a
 * negative PVOF_E* code on failure; pvof_last_error() gives a message.  The
 * reference aborts through Display_throw_error (PARTIES/src/IO/Display.c:910);
 * the caller decides what to do with the code.  Iterative solvers always stop
 * at their iteration limits and report non-convergence in the statistics.
 */
#ifndef PVOF_H
#define PVOF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PVOF_ABI_VERSION 4

/* error codes */
#define PVOF_OK 0
#define PVOF_EINVAL (-1)     /* bad argument or unsupported configuration */
#define PVOF_ECUDA (-2)      /* CUDA runtime error */
#define PVOF_ENOMEM (-3)     /* device allocation failed */
#define PVOF_ENODEV (-4)     /* no CUDA device */
#define PVOF_EDIVERGED (-5)  /* the outer Poisson loop did not reach div < 1e-6 in 10 passes */

/* geometry (runtime form of the reference's TWOD_CARTESIAN / AXISYM_RZ flags,
 * PARTIES/src/Include/Boundary.h:36-38) */
#define PVOF_GEOM_3D 0
#define PVOF_GEOM_PLANAR 1
#define PVOF_GEOM_AXISYM 2

/* wall type per face (Boundary.h x/y/z boundary macros) */
#define PVOF_WALL_NOSLIP 0
#define PVOF_WALL_FREESLIP 1

/* faces */
#define PVOF_LEFT 0
#define PVOF_RIGHT 1
#define PVOF_BOTTOM 2
#define PVOF_TOP 3
#define PVOF_BACK 4
#define PVOF_FRONT 5

/* Grid and case description: the [geometry], [grid], [twod] sections of the
 * reference's parties.inp (PARTIES/src/IO/default.inp) plus the compile-time
 * boundary flags of Boundary.h. */
typedef struct pvof_grid_desc {
    int NXM, NYM, NZM;          /* physical cells per direction */
    int ghost_nodes;            /* must be 3 */
    int geometry;               /* PVOF_GEOM_* */
    int periodic[3];            /* XPERIODIC, YPERIODIC, ZPERIODIC */
    int wall[6];                /* PVOF_WALL_* per face (ignored on periodic axes) */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double slab_thickness;      /* twod_slab_thickness after Input.c defaults */
    double theta_span;          /* axisym_theta_span */
} pvof_grid_desc;

/* Physical and solver parameters: [flow], [vof], [particle] grav, [conc]
 * richardson and [lsolve] of parties.inp, plus the SURFACE_TENSION and
 * VOF_GRAVITY compile flags. */
typedef struct pvof_params {
    double Re, We;
    double rho1, rho2, mu1, mu2;
    double Cn, Pe_CH;
    double grav[3];
    double richardson;
    double dp_dx;
    int weno_order;
    int ch_iter_max;
    double ch_tol;
    int CG_MAXIT;
    double CG_ETOL;
    int P_CG_MAXIT;
    double P_CG_ETOL;
    int surface_tension;        /* SURFACE_TENSION */
    int gravity;                /* VOF_GRAVITY */
    /* resolved solids (used once pvof_set_particles has been called) */
    double contact_angle_deg;   /* [vof] contact_angle_deg (default 90) */
    int N_forcing_loops;        /* [particle] N_forcing_loops (default 2) */
    /* no counterpart in the reference: 1 selects the FP32 stencil form (WENO5
     * fluxes, chemical potential and surface-tension force in single
     * precision; fields, reductions and solvers stay FP64); 0 is the plain
     * FP64 path that matches the reference */
    int stencil_fp32;
    /* no counterpart in the reference: 1 starts the first pressure solve of a
     * substep from the correction of the same RK stage of the previous time
     * step instead of zero; 2 adds to it the change predicted by the network
     * set with pvof_set_pressure_network (the learned warm start); the solve
     * still stops at the same absolute residual, so the result moves within
     * that tolerance */
    int pressure_warm_start;
    /* no counterpart in the reference: 1 preconditions the pressure PCG with
     * the inverse of the constant-density Laplacian (an FFT along the periodic
     * x rows and a tridiagonal solve per wavenumber along y), scaled on both
     * sides by the square root of the Jacobi weights, instead of the Jacobi
     * diagonal; the solve still stops when sqrt(r^T D^-1 r), D the
     * Jacobi diagonal, is below P_CG_ETOL, so the result moves within that
     * tolerance.  Planar grids with x periodic, walls in y, a power-of-two x
     * cell count up to 1024 and at most 1024 y cells; in the 3D mode the
     * transforms run along x and z (power-of-two cell counts up to 1024) and
     * the tridiagonal solves along y; 0 is the reference's Jacobi-PCG */
    int pressure_preconditioner;
    /* no counterpart in the reference: 1 drops the 1e-14 that the momentum
     * CG adds to its step-length and direction-update denominators
     * (msolve_cg.c).  Once the preconditioned residual r^T D^-1 r falls near
     * 1e-14 that constant shortens every step, so the reference's solve stalls
     * above CG_ETOL and runs to CG_MAXIT; without it the solve stops at
     * CG_ETOL.  0 is the reference's iteration */
    int velocity_cg_unregularized;
} pvof_params;

/* Field identifiers for upload/download. */
enum pvof_field {
    PVOF_F_C_L = 0, PVOF_F_C_G, PVOF_F_C_S, PVOF_F_F,
    PVOF_F_RHO, PVOF_F_MU, PVOF_F_PSI_LG, PVOF_F_LAP_C,
    PVOF_F_CH_RHS_N, PVOF_F_CH_RHS_CUR,
    PVOF_F_U, PVOF_F_V, PVOF_F_W, PVOF_F_U_BC, PVOF_F_V_BC,
    PVOF_F_P, PVOF_F_DELTAP, PVOF_F_P_RHS,
    /* no-ghost momentum arrays (Velocity ng_*) */
    PVOF_F_U_EXPLICIT, PVOF_F_U_EXPLICIT_OLD, PVOF_F_U_IMPLICIT,
    PVOF_F_U_VISC_EXPLICIT, PVOF_F_U_VISC_EXPLICIT_OLD, PVOF_F_U_RHS,
    PVOF_F_V_EXPLICIT, PVOF_F_V_EXPLICIT_OLD, PVOF_F_V_IMPLICIT,
    PVOF_F_V_VISC_EXPLICIT, PVOF_F_V_VISC_EXPLICIT_OLD, PVOF_F_V_RHS,
    /* no-ghost surface-tension face forces */
    PVOF_F_FSIG_OLD_X, PVOF_F_FSIG_OLD_Y, PVOF_F_FSIG_NEW_X, PVOF_F_FSIG_NEW_Y,
    /* solid normals of the contact-line projection (VolumeFraction nx_IBM, ny_IBM) */
    PVOF_F_NX_IBM, PVOF_F_NY_IBM,
    /* the 3D mode's w momentum arrays and z surface-tension force (no-ghost) */
    PVOF_F_W_EXPLICIT, PVOF_F_W_EXPLICIT_OLD, PVOF_F_W_IMPLICIT,
    PVOF_F_W_VISC_EXPLICIT, PVOF_F_W_VISC_EXPLICIT_OLD, PVOF_F_W_RHS,
    PVOF_F_FSIG_OLD_Z, PVOF_F_FSIG_NEW_Z,
    PVOF_F_COUNT
};

/* Per-substep statistics (iteration counts and residuals the reference
 * prints through Display_progress). */
typedef struct pvof_stats {
    int ch_iters;          /* biharmonic CG iterations (VOF_DIFFUSE.c:1048) */
    double ch_rel_res;
    int u_iters, v_iters;  /* velocity PCG iterations (msolve_cg.c:716) */
    double u_rms, v_rms;
    int p_iters;           /* pressure PCG iterations of the last Poisson pass */
    int p_iters_total;     /* over all passes of the outer Poisson loop */
    double p_res;
    int poisson_passes;    /* outer loop count (Temporal_int.c:1052-1107) */
    double div_max;        /* Pressure_compute_velocity_divergence */
    double clamp_mass;     /* liquid mass changed by the C_L clamp over the physical cells
                              (VOF_DIFFUSE.c:1093-1127) */
    int w_iters;           /* w-velocity PCG iterations (3D mode; 0 in 2D) */
    double w_rms;
} pvof_stats;

typedef struct pvof_ctx pvof_ctx;

/* Library */
int pvof_abi_version(void);
const char *pvof_last_error(void);
int pvof_device_count(void);

/* Context: allocates the device state for one case on `device`.
 * Replaces the allocation done by Velocity_create / Pressure_create /
 * VoF_create (PARTIES/src/Cart3d.c:339-390) for the fields listed above. */
int pvof_create(const pvof_grid_desc *grid, const pvof_params *params, int device, pvof_ctx **out);
int pvof_destroy(pvof_ctx *ctx);

/* Host <-> device copies of one field in the reference block layout (see the
 * header comment); count = number of doubles in the host block, checked. */
int pvof_upload_field(pvof_ctx *ctx, int field, const double *host_block, size_t count);
int pvof_download_field(pvof_ctx *ctx, int field, double *host_block, size_t count);
/* number of doubles in the host block of `field` */
size_t pvof_field_block_count(const pvof_ctx *ctx, int field);
int pvof_synchronize(pvof_ctx *ctx);

/* Stage and time step of the following routine calls: the reference's
 * params->which_stage (0..2) and params->dt. */
int pvof_set_stage(pvof_ctx *ctx, int which_stage, double dt);

/* Start-up after the initial fields (F, u, v, p) are uploaded:
 * Velocity_update_boundaries of u and v, Pressure_apply_BCs and ghost update
 * of p, the VOF part of Cart3d_initialize_primitive_data
 * (PARTIES/src/Cart3d.c:1096-1130: boundary values of F, VOF_DIFFUSE_init,
 * density and viscosity, surface-tension bootstrap with f_old = f_new) and the
 * cell-centred velocity of the first substep.  Resets the time to 0. */
int pvof_initialize(pvof_ctx *ctx);

/* --- routines, reference name and file:line each replaces --------------- */
/* VOF_DIFFUSE.c:524-568 VOF_DIFFUSE_init (C_L from F, clamp, phase cache) */
int pvof_VOF_DIFFUSE_init(pvof_ctx *ctx);
/* VOF_DIFFUSE.c:1262-1359 VOF_DIFFUSE_step: WENO5 advection, explicit
 * diffusion, RK assembly, implicit biharmonic CG, clamp, history shift */
int pvof_VOF_DIFFUSE_step(pvof_ctx *ctx, pvof_stats *stats);
/* VOF_DIFFUSE.c:931-996 VOF_DIFFUSE_advect_WENO5, result in CH_RHS_CUR */
int pvof_VOF_DIFFUSE_advect_WENO5(pvof_ctx *ctx);
/* VOF_Advection.c:743-749 -> VOF_DIFFUSE.c:1453-1488 rho, mu from C */
int pvof_VOF_update_density_viscosity(pvof_ctx *ctx);
/* VOF_DIFFUSE.c:907-929 psi_LG */
int pvof_VOF_DIFFUSE_compute_psi_LG(pvof_ctx *ctx);
/* VOF_DIFFUSE.c:1364-1445 face surface-tension force into f_sigma_new */
int pvof_VOF_DIFFUSE_compute_f_sigma(pvof_ctx *ctx);
/* VOF_SurfaceTension.c:1983-2041 rhs += f_sigma_old */
int pvof_VOF_apply_f_sigma_old(pvof_ctx *ctx);
/* VOF_SurfaceTension.c:2055-2071 swap new/old force arrays */
int pvof_VOF_swap_f_sigma(pvof_ctx *ctx);
/* VOF_SurfaceTension.c:2075-2154 gravity term */
int pvof_Velocity_add_gravity_2_RHS(pvof_ctx *ctx);
/* Velocity.c:278-357 cell-centred velocity (with ghost update) */
int pvof_Velocity_cell_center(pvof_ctx *ctx);
/* Velocity.c:366-762 (component 'u'), :771-1148 ('v') */
int pvof_Velocity_set_implicit_explicit(pvof_ctx *ctx, char component);
/* Velocity.c:1494-1728 ('u'), :1739-1940 ('v') */
int pvof_Velocity_set_RHS(pvof_ctx *ctx, char component);
/* msolve_cg.c:525-722 Velocity_solve_cg; returns iterations */
int pvof_Velocity_solve_cg(pvof_ctx *ctx, char component, pvof_stats *stats);
/* Velocity.c:2427-2806 Velocity_update_boundaries (VEL_TYPE_NORMAL) */
int pvof_Velocity_update_boundaries(pvof_ctx *ctx, char component);
/* Pressure.c:100-196 (after the deltap reset of Temporal_int.c:1056) */
int pvof_Pressure_set_RHS(pvof_ctx *ctx);
/* psolve_cg.c:63-101 */
int pvof_Pressure_compute_preconditioner(pvof_ctx *ctx);
/* psolve_cg.c:130-293; returns iterations */
int pvof_Pressure_solve_cg(pvof_ctx *ctx, pvof_stats *stats);
/* Pressure.c:218-464 */
int pvof_Pressure_project_velocity(pvof_ctx *ctx);
/* Pressure.c:475-597; writes the max |div| to *div_max */
int pvof_Pressure_compute_velocity_divergence(pvof_ctx *ctx, double *div_max);

/* Eulerian/lsolver/psolve_fft.c:638-983 Pressure_solve_xz_period: the
 * constant-density Poisson equation lap(DELTAP) = P_RHS on the physical cells
 * by a Fourier transform in x and tridiagonal solves in y (Neumann walls, the
 * mean mode pinned at the first row); planar mode, x periodic, at most 2048
 * cells in x.  Not on the variable-density path of the substep. */
int pvof_Pressure_solve_fft(pvof_ctx *ctx);

/* Temporal_int.c:563-1279 Temporal_int_all_the_equations for a case without
 * solids: one complete RK substep at the stage/dt set by pvof_set_stage. */
int pvof_substep(pvof_ctx *ctx, pvof_stats *stats);
/* Temporal_int.c:399-448: nsteps time steps of three substeps each at a
 * constant dt (cell-centred velocity refreshed at stage 0 after t = 0).
 * stats (optional) receives the last substep's statistics. */
int pvof_run_steps(pvof_ctx *ctx, int nsteps, double dt, pvof_stats *stats);

/* Batched form: advances n independent contexts by nsteps each
 * (pvof_run_steps), concurrently -- one host thread per context, each on its
 * own stream, so the solvers of different cases share the GPU's SMs.
 * stats (optional) has n entries.  Returns the first failing case's code. */
int pvof_run_steps_batched(pvof_ctx *const *ctxs, int n, int nsteps, double dt, pvof_stats *stats);

/* Sum of C_L * cell measure over the physical cells (mass diagnostic,
 * VOF_DIFFUSE.c:1071-1091), computed on the device in FP64. */
int pvof_liquid_mass(pvof_ctx *ctx, double *mass);

/* --- resolved solid particles (planar cylinders, axisymmetric spheres) ----
 * The reference keeps particles in two linked lists (p_mobile, p_fixed,
 * PARTIES/src/Include/DataTypes.h:1327-1527) read from p_mobile.inp /
 * p_fixed.inp.  Here the caller passes the owned particles once; the library
 * derives markers, masses and the periodic copies itself and keeps the lists
 * in device memory: the list updates, markers, flags and the rigid-body
 * motion run on the device, so the calls below enqueue work without waiting
 * for it, except those that return particle data (pvof_particle_entries,
 * _forces, _markers, pvof_get_particles), which read the device state back,
 * and pvof_Lagrangian_advect_particles, which reads its error state. */
typedef struct pvof_particle {
    int mobile;         /* 1: mobile list, 0: fixed list */
    double X[2];        /* centre (x, y) */
    double R;           /* radius */
    double U[2];        /* translational velocity */
    double Omega_z;     /* spin about z */
    double rho_s;       /* solid density ([particle] rho_s) */
} pvof_particle;

/* Replaces the particle lists; IDs as Particle_initialize assigns them (fixed
 * first, then mobile; Lagrangian/Particle.c:213-221).  Sizes the device lists
 * (at most nine entries per particle: two periodic copies per periodic axis)
 * and drops the context's captured substep graphs. */
int pvof_set_particles(pvof_ctx *ctx, const pvof_particle *particles, int n);
/* Particle_MPI_update of both lists on one rank (periodic copies) and
 * Lagrangian_flag_points (Lagrangian/Lagrangian.c:2515-2627): markers of
 * every list entry near the domain and their on/off flags. */
int pvof_Lagrangian_flag_points(pvof_ctx *ctx);
/* number of list entries after the last update (owned particles and copies,
 * mobile list first) */
int pvof_particle_entries(pvof_ctx *ctx);
/* F and T (3 doubles per entry each) accumulated by pvof_Lagrangian_force */
int pvof_particle_forces(pvof_ctx *ctx, double *F, double *T, int max_entries);
/* markers of one entry: positions, control volumes, flags; returns the count */
int pvof_particle_markers(pvof_ctx *ctx, int entry, double *x, double *y, double *vol, int *flag, int max_markers);
/* Eulerian/VOF_DIFFUSE.c:685-813 VOF_DIFFUSE_compute_C_S: solid fraction, then
 * the clamp of C_L and the phase cache */
int pvof_VOF_DIFFUSE_compute_C_S(pvof_ctx *ctx);
/* Eulerian/VOF_IBM_wetting.c:1021-1104 VOF_DIFFUSE_compute_solid_normals_MCL:
 * solid normals into PVOF_F_NX_IBM / PVOF_F_NY_IBM */
int pvof_VOF_DIFFUSE_compute_solid_normals_MCL(pvof_ctx *ctx);
/* Eulerian/VOF_IBM_wetting.c:1946-2008 VOF_DIFFUSE_apply_contact_angle: the
 * characteristic contact-angle projection of C_L in the solid cells along the
 * contact line (no boundary update, as the reference) */
int pvof_VOF_DIFFUSE_apply_contact_angle(pvof_ctx *ctx);
/* Eulerian/VOF_IBM_wetting.c:2014-2131 VOF_DIFFUSE_extend_psi_LG_contact_angle:
 * psi_LG in the same cells along the same characteristics, then its boundary
 * values */
int pvof_VOF_DIFFUSE_extend_psi_LG_contact_angle(pvof_ctx *ctx);
/* Lagrangian/Particle.c:322-535 Particle_initialize_velocities: mobile
 * particles take the volume-averaged fluid velocity and the fluid inside them
 * is painted to that rigid motion (pvof_initialize calls it) */
int pvof_Particle_initialize_velocities(pvof_ctx *ctx);
/* Temporal_int.c:1186-1238 and Lagrangian/Lagrangian.c:283-1640 the end of a
 * substep: momentum integrals over the particles, the contact-line capillary
 * force, Lagrangian_advect_particles (fluid forces, then the substepped
 * rigid-body motion).  PVOF_EINVAL when two particles, or a particle and a
 * wall, come within the lubrication range (the collision models are not part
 * of this library).  pvof_substep calls it. */
int pvof_Lagrangian_advect_particles(pvof_ctx *ctx);
/* the owned particles in list order (mobile list, then fixed): position,
 * velocity and spin in `out` (R, rho_s and mobile as given), their IDs and the
 * total fluid force and torque of the last substep (3 doubles each); any of
 * ids, F, T may be NULL; returns the count */
int pvof_get_particles(pvof_ctx *ctx, pvof_particle *out, int *ids, double *F, double *T, int max_particles);
/* Eulerian/lsolver/msolve_direct.c:146-260 Velocity_solve_explicit (u or v) */
int pvof_Velocity_solve_explicit(pvof_ctx *ctx, char component);
/* Lagrangian/Lagrangian.c:1724-1871 Lagrangian_force: force_iter < 0 is the
 * predictor on the momentum RHS, force_iter >= 0 that many corrector passes on
 * the velocity; call pvof_Lagrangian_flag_points() first */
int pvof_Lagrangian_force(pvof_ctx *ctx, int force_iter);

/* --- learned warm start (no counterpart in the reference) --------------- */
/* The network: six 3x3 convolutions 3 -> 32 -> 32 -> 32 -> 32 -> 32 -> 1,
 * zero padding, ReLU between them, BF16 weights with FP32 accumulation; the
 * four hidden 32 -> 32 layers run on the tensor cores with BF16 activations
 * (their input gradients too).
 * Parameters are one flat FP32 array [w0, b0, ..., w5, b5], w_l laid out
 * [cout][cin][3][3]; planes are channel-major [C][H][W] floats on the device.
 * Inputs: rho, rhs / rms(rhs), phi_prev / rms(phi_prev); output: the change
 * of the pressure correction over rms(phi_prev). */
size_t pvof_cnn_param_count(void);
/* floats of the work buffer (activations) for an H x W plane */
size_t pvof_cnn_work_floats(int H, int W);
/* forward pass; y may be NULL (the output stays in the work buffer) */
int pvof_cnn_forward(const float *params, const uint16_t *params_bf16, const float *x, float *y, int H, int W,
                     float *work, void *stream);
/* backward pass after pvof_cnn_forward with the same work buffer: adds the
 * parameter gradient of dL/dy to grad */
int pvof_cnn_backward(const float *params, const uint16_t *params_bf16, const float *x, const float *dy, float *grad,
                      int H, int W, float *work, void *stream);
/* mean-square loss of y against t over n values (added to *loss on the
 * device) and its gradient dy */
int pvof_cnn_mse(const float *y, const float *t, float *dy, size_t n, double *loss, void *stream);
/* one Adam step (step counts from 1) on the FP32 parameters and their BF16 copy */
int pvof_cnn_adam(float *params, const float *grad, float *m, float *v, uint16_t *params_bf16, int step, float lr,
                  void *stream);
/* the BF16 copy of FP32 parameters */
int pvof_cnn_to_bf16(const float *params, uint16_t *params_bf16, void *stream);
/* one hidden-layer convolution on the tensor cores, as the network runs it:
 * y[co] = b[co] + sum_ci sum_tap w[co][ci][tap] x[ci][p + tap] (zero outside
 * the H x W plane) with x rounded to BF16, w in BF16 ([32][32][3][3]), FP32
 * accumulation, then the ReLU if relu; x, y: 32 planes [32][H][W]; b may be
 * NULL */
int pvof_cnn_conv32(const float *x, const uint16_t *w_bf16, const float *b, float *y, int H, int W, int relu,
                    void *stream);
/* waits for the stream; PVOF_ECUDA (and the flag cleared) if a tensor-core
 * convolution since the last call gave up waiting for its matrix
 * multiplications, else 0 */
int pvof_cnn_status(void *stream);
/* the network the context's pressure_warm_start == 2 uses (host array of
 * pvof_cnn_param_count() floats) */
int pvof_set_pressure_network(pvof_ctx *ctx, const float *params, size_t n);
/* a training sample from the last substep of `stage` (with
 * pressure_warm_start on, once two time steps have run): the network inputs
 * (x: 3 planes) and target (t: 1 plane) on the (NYM x NXM) physical cells,
 * device arrays */
int pvof_pressure_network_sample(pvof_ctx *ctx, int stage, float *x, float *t);

/* --- measurement (no counterpart in the reference) ---------------------- */
/* Number of CUDA kernels this context has launched so far. */
long long pvof_launch_count(const pvof_ctx *ctx);
/* Device time of everything issued on the context's stream between
 * pvof_timer_start and pvof_timer_stop (CUDA events on that stream);
 * pvof_timer_stop waits for the work and returns milliseconds. */
int pvof_timer_start(pvof_ctx *ctx);
int pvof_timer_stop(pvof_ctx *ctx, double *ms);
/* Write a device buffer larger than the L2 cache on the context's stream so
 * the next timed region starts with a cold L2. */
int pvof_flush_l2(pvof_ctx *ctx);
/* Per-solver launch timing, collected while enabled: PVOF_SOLVER_* selects
 * the biharmonic CG, the velocity PCG or the pressure PCG.  ms is the summed
 * device duration of its launches (CUDA events around each launch),
 * cell_iters the sum over launches of (cells in the solve range) x
 * (iterations). */
#define PVOF_SOLVER_BIHARMONIC 0
#define PVOF_SOLVER_VELOCITY 1
#define PVOF_SOLVER_PRESSURE 2
int pvof_set_solver_timing(pvof_ctx *ctx, int enabled);

/* No counterpart in the reference: the stencil tile autotuner.  The
 * cell-wise stencil kernels compute every cell alike whatever their
 * thread-block shape; with enabled = 1 the next substeps time each such
 * kernel's launches over a set of candidate tiles (32x8, 64x4, 128x2, 256x1,
 * 32x4, 64x8; two launches each, CUDA events) and keep for each kernel the
 * tile of the smallest mean time.  Results are bit for bit those of the
 * default tile.  While tuning, substeps run launch by launch; tuning ends by
 * itself once every kernel met so far is decided.  Tune a context while it
 * has the GPU to itself: a launch's event time includes its waits behind
 * other streams' work.  enabled = 0 stops it and
 * returns every kernel to the default tile.  Drops the captured substep
 * graphs. */
int pvof_set_autotune(pvof_ctx *ctx, int enabled);
/* 1 while the autotuner is still sampling, else 0. */
int pvof_autotune_active(const pvof_ctx *ctx);
/* Kernels the autotuner has met; entry q: the kernel's name, its tile, its
 * mean launch time there and at the default tile (ms).  Returns 1 when the
 * kernel is decided, 0 while undecided (the default tile), <0 on error. */
int pvof_autotune_entries(const pvof_ctx *ctx);
int pvof_autotune_entry(const pvof_ctx *ctx, int q, const char **name, int *bx, int *by, double *best_ms,
                        double *default_ms);

/* No counterpart in the reference: 1 (the default) replays the launches of
 * pvof_substep up to its first Poisson pass's divergence check from a CUDA
 * graph captured per (stage, dt, buffer parity, warm-start state); 0 issues
 * them one by one.  Results are identical.  Cases with resolved particles,
 * the learned warm start, and any substep run while solver timing is on
 * issue them one by one. */
int pvof_set_graphs(pvof_ctx *ctx, int enabled);
/* No counterpart in the reference: how many substeps so far replayed their
 * launches from a graph (-1 for a null context). */
long long pvof_graph_replays(const pvof_ctx *ctx);
/* The liquid mass the C_L clamp changed (pvof_stats.clamp_mass,
 * VOF_DIFFUSE.c:1093-1127) summed over every substep since pvof_initialize. */
int pvof_clamp_mass_total(const pvof_ctx *ctx, double *total);
/* No counterpart in the reference: 1 (the default) solves the pressure and
 * momentum systems with the cluster-resident kernels wherever their solve
 * ranges fit one thread-block cluster; 0 selects the grid-wide persistent
 * kernels for every size.  Both run the reference's iteration; results agree
 * to rounding (their inner products are summed in different orders).  Waits
 * for the context's stream and drops its captured substep graphs. */
int pvof_set_cluster_solvers(pvof_ctx *ctx, int enabled);
/* No counterpart in the reference: how the grid-wide pressure solve
 * (Pressure_solve_cg, psolve_cg.c:130-293, on ranges larger than one
 * cluster) assigns cells to threads.  -1 (the default): pairs of
 * neighbouring cells with 16-byte accesses once every resident thread has at
 * least two cells, single cells below that; 1: pairs at every size; 0:
 * single cells at every size.  The same iteration either way; results agree
 * to rounding (the inner products are summed in different orders).  Waits
 * for the context's stream and drops its captured substep graphs. */
int pvof_set_pressure_pairs(pvof_ctx *ctx, int mode);

/* No counterpart in the reference: the host-computed table of the spectral
 * pressure preconditioner's tridiagonal solves for an N x M grid (x spacing
 * squared inverse idx2, y idy2), without a GPU.  The systems
 * a_j z_{j-1} + b_j z_j + c_j z_{j+1} = r_j (a = c = -1 inside,
 * b_j = lambda_m + 2 inside, lambda_m + 1 at the walls; the mean mode's
 * first row pinned) are solved by a partition method: the M rows split into
 * P = min(32, M / 2) chunks, chunk l starting at l base + min(l, rem) with
 * base + (l < rem) rows (base = M / P, rem = M mod P; K the longest).  Per
 * wave number m = 0 .. N/2, (2K + 4) rows of 32 doubles, entry [row][l]:
 * row i (1 <= i < chunk length) the elimination pivot r_i, row K + i the
 * coupling A_i to the chunk's first unknown, row 0 the chunk's c_0, row K its
 * a_0, rows 2K .. 2K + 3 the Thomas pivot and c' of the reduced system's
 * equations 2l and 2l + 1.  Returns the number of doubles, (N/2 + 1)(2K + 4)
 * 32, and writes them to out when cap is at least that; -1 on invalid sizes
 * (N = 2^a, 3 2^a or 5 2^a and even, M >= 2). */
long long pvof_spectral_tables(int N, int M, double idx2, double idy2, double *out, long long cap);
int pvof_solver_timing(const pvof_ctx *ctx, int solver, double *ms, long long *launches, long long *iterations,
                       long long *cell_iters);
/* Name of the kernel that runs solver PVOF_SOLVER_* for this context: the
 * cluster-resident form when the solve range fits one thread-block cluster,
 * else the grid-wide persistent form. */
const char *pvof_solver_kernel(const pvof_ctx *ctx, int solver);

/* --- no-allocation variant (no counterpart in the reference) -------------
 * The pressure correction solve -- Pressure_compute_preconditioner,
 * Pressure_solve_cg and the ghost exchange of the correction -- for callers
 * that cannot allocate device memory (for example a host code that owns a
 * fixed device pool, or runs where cudaMalloc may not be called).  The
 * caller passes device planes in the reference's k = 0 plane layout
 * ((NYM+7) rows of NXM+7 doubles, element (i,j) at (j+3)*(NXM+7) + i+3):
 * rho with its ghost cells filled, the right-hand side, and phi (the initial
 * guess on entry, normally zero; the correction on return).  Every temporary
 * lives in one fixed device array of the library (about 3.7 MB, kept on each
 * GPU that loads the library until the process exits); the call allocates
 * nothing.  Limits: (NXM+7)*(NYM+7) <= 72000 and NXM, NYM <= 1024, else
 * PVOF_EINVAL.  All calls on a device share that array: calls that overlap
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the array's address with that device current; make it
 * before any stream capture.  stream is a cudaStream_t (NULL: default
 * stream); the call returns after the solve has finished, with the
 * iteration count (also the return value) and the final sqrt(r.M^-1 r).
 * As in the reference, a solve that reaches P_CG_MAXIT stops there and still
 * returns its (positive) iteration count: the solve converged only if
 * *residual < P_CG_ETOL, so a caller that needs a converged correction
 * compares the two. */
int pvof_Pressure_solve_cg_noalloc(const pvof_grid_desc *grid, const pvof_params *params, const double *rho,
                                   const double *rhs, double *phi, void *stream, int *iterations,
                                   double *residual);
const char *pvof_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
