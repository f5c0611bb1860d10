/*
 * pvof_bridge.c -- PARTIES' Cart3d_bag onto the B200 substep's C ABI.
 * See pvof_bridge.h for how a PARTIES build uses it.
 *
 * Compile-time flags read here are the reference's own (Boundary.h):
 * TWOD_CARTESIAN / AXISYM_RZ, XPERIODIC / YPERIODIC, the *_WALL_VELOCITY_*
 * wall types, SURFACE_TENSION, VOF_GRAVITY, VOF_IBM + LAG_PARTICLE_RESOLVED.
 */
#include "pvof_bridge.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "definitions.h"

#if !defined(VOF) || !defined(VOF_DIFFUSE)
#error "pvof_bridge.c bridges the diffuse-interface two-phase build (VOF, VOF_DIFFUSE)"
#endif
#if !defined(TWOD_CARTESIAN) && !defined(AXISYM_RZ)
#define PVOF_BRIDGE_3D 1   /* the 3D mode: x and z periodic, walls in y, no solids */
#if !defined(XPERIODIC) || !defined(ZPERIODIC) || defined(YPERIODIC) || defined(VOF_IBM)
#error "pvof_bridge.c bridges 3D builds with XPERIODIC, ZPERIODIC, walls in y and no solids"
#endif
#endif

static pvof_ctx *g_ctx;
static pvof_stats g_stats;

#ifdef PVOF_BRIDGE_ABORT
static int bridge_fail(int rc, const char *what)
{
    fprintf(stderr, "pvof bridge: %s: %s\n", what, pvof_last_error());
    MPI_Abort(MPI_COMM_WORLD, 1);
    return rc;
}
#else
static int bridge_fail(int rc, const char *what)
{
    (void)what;
    return rc;
}
#endif

#define TRYB(call, what)                              \
    do {                                              \
        int rc_ = (call);                             \
        if (rc_ < 0) return bridge_fail(rc_, what);   \
    } while (0)

/* first element of a field's contiguous block (PARTIES/src/Memory.c:36-89,
 * :270-323): the ghosted (L-range) or no-ghost (G-range) origin */
#define FLOW_BLOCK(a, g) (&(a)[(g)->L_Ks][(g)->L_Js][(g)->L_Is])
#define NG_BLOCK(a, g) (&(a)[(g)->G_Ks][(g)->G_Js][(g)->G_Is])

/* the reference array behind each device field (NULL where this build has
 * none); ng = 1 for the no-ghost arrays */
static double ***field_array(Cart3d_bag *b, int f, int *ng)
{
    VolumeFraction *vof = b->vof;
    *ng = (f >= PVOF_F_U_EXPLICIT && f <= PVOF_F_FSIG_NEW_Y) || (f >= PVOF_F_W_EXPLICIT && f <= PVOF_F_FSIG_NEW_Z);
    switch (f) {
    case PVOF_F_C_L: return vof->C_L;
    case PVOF_F_C_G: return vof->C_G;
    case PVOF_F_C_S: return vof->C_S;
    case PVOF_F_F: return vof->F;
    case PVOF_F_RHO: return vof->rho;
    case PVOF_F_MU: return vof->mu;
    case PVOF_F_PSI_LG: return vof->psi_LG;
    case PVOF_F_LAP_C: return vof->lap_C;
    case PVOF_F_CH_RHS_N: return vof->ch_rhs_n;
    case PVOF_F_CH_RHS_CUR: return vof->ch_aux2;
    case PVOF_F_U: return b->u->data;
    case PVOF_F_V: return b->v->data;
    case PVOF_F_W: return b->w->data;
    case PVOF_F_U_BC: return b->u->data_bc;
    case PVOF_F_V_BC: return b->v->data_bc;
    case PVOF_F_P: return b->p->p_data;
    case PVOF_F_DELTAP: return b->p->deltap;
    case PVOF_F_P_RHS: return b->p->rhs;
    case PVOF_F_U_EXPLICIT: return b->u->ng_explicit;
    case PVOF_F_U_EXPLICIT_OLD: return b->u->ng_explicit_old;
    case PVOF_F_U_IMPLICIT: return b->u->ng_implicit;
    case PVOF_F_U_VISC_EXPLICIT: return b->u->ng_visc_explicit;
    case PVOF_F_U_VISC_EXPLICIT_OLD: return b->u->ng_visc_explicit_old;
    case PVOF_F_U_RHS: return b->u->ng_rhs;
    case PVOF_F_V_EXPLICIT: return b->v->ng_explicit;
    case PVOF_F_V_EXPLICIT_OLD: return b->v->ng_explicit_old;
    case PVOF_F_V_IMPLICIT: return b->v->ng_implicit;
    case PVOF_F_V_VISC_EXPLICIT: return b->v->ng_visc_explicit;
    case PVOF_F_V_VISC_EXPLICIT_OLD: return b->v->ng_visc_explicit_old;
    case PVOF_F_V_RHS: return b->v->ng_rhs;
    case PVOF_F_FSIG_OLD_X: return vof->f_sigma_old_x;
    case PVOF_F_FSIG_OLD_Y: return vof->f_sigma_old_y;
    case PVOF_F_FSIG_NEW_X: return vof->f_sigma_new_x;
    case PVOF_F_FSIG_NEW_Y: return vof->f_sigma_new_y;
#ifdef PVOF_BRIDGE_3D
    case PVOF_F_W_EXPLICIT: return b->w->ng_explicit;
    case PVOF_F_W_EXPLICIT_OLD: return b->w->ng_explicit_old;
    case PVOF_F_W_VISC_EXPLICIT: return b->w->ng_visc_explicit;
    case PVOF_F_W_VISC_EXPLICIT_OLD: return b->w->ng_visc_explicit_old;
    case PVOF_F_W_RHS: return b->w->ng_rhs;
    case PVOF_F_FSIG_OLD_Z: return vof->f_sigma_old_z;
    case PVOF_F_FSIG_NEW_Z: return vof->f_sigma_new_z;
#endif
#ifdef VOF_IBM
    case PVOF_F_NX_IBM: return vof->nx_IBM;
    case PVOF_F_NY_IBM: return vof->ny_IBM;
#endif
    default: return NULL;
    }
}

static double *field_block(Cart3d_bag *b, int f)
{
    int ng = 0;
    double ***a = field_array(b, f, &ng);
    if (!a) return NULL;
    return ng ? NG_BLOCK(a, b->grid) : FLOW_BLOCK(a, b->grid);
}

#ifdef PVOF_BRIDGE_3D
/* the fields the 3D mode keeps: the rest are scratch or derived there */
static int kept_3d(int f, int to_device)
{
    switch (f) {
    case PVOF_F_C_G: case PVOF_F_RHO: case PVOF_F_MU:
        return !to_device;
    case PVOF_F_C_L: case PVOF_F_F: case PVOF_F_PSI_LG: case PVOF_F_CH_RHS_N: case PVOF_F_U: case PVOF_F_V:
    case PVOF_F_W: case PVOF_F_P: case PVOF_F_DELTAP:
    case PVOF_F_U_EXPLICIT_OLD: case PVOF_F_V_EXPLICIT_OLD: case PVOF_F_W_EXPLICIT_OLD:
    case PVOF_F_U_VISC_EXPLICIT_OLD: case PVOF_F_V_VISC_EXPLICIT_OLD: case PVOF_F_W_VISC_EXPLICIT_OLD:
    case PVOF_F_FSIG_OLD_X: case PVOF_F_FSIG_OLD_Y: case PVOF_F_FSIG_OLD_Z:
    case PVOF_F_FSIG_NEW_X: case PVOF_F_FSIG_NEW_Y: case PVOF_F_FSIG_NEW_Z:
        return 1;
    default:
        return 0;
    }
}
#endif

static int copy_field(Cart3d_bag *b, int f, int to_device)
{
#ifdef PVOF_BRIDGE_3D
    if (!kept_3d(f, to_device)) return PVOF_OK;
#endif
    double *blk = field_block(b, f);
    if (!blk) return PVOF_OK;
    size_t n = pvof_field_block_count(g_ctx, f);
    return to_device ? pvof_upload_field(g_ctx, f, blk, n) : pvof_download_field(g_ctx, f, blk, n);
}

/* the case description: [geometry], [grid], [twod] of parties.inp and the
 * boundary flags of Boundary.h */
static void grid_desc(Cart3d_bag *b, pvof_grid_desc *gd)
{
    Parameters *p = b->params;
    memset(gd, 0, sizeof(*gd));
    gd->NXM = p->NXM;
    gd->NYM = p->NYM;
    gd->NZM = p->NZM;
    gd->ghost_nodes = p->ghost_nodes;
#if defined(AXISYM_RZ)
    gd->geometry = PVOF_GEOM_AXISYM;
#elif defined(TWOD_CARTESIAN)
    gd->geometry = PVOF_GEOM_PLANAR;
#else
    gd->geometry = PVOF_GEOM_3D;
#endif
#ifdef XPERIODIC
    gd->periodic[0] = 1;
#endif
#ifdef YPERIODIC
    gd->periodic[1] = 1;
#endif
    gd->periodic[2] = 1;   /* ZPERIODIC, or the collapsed storage direction of the 2D modes */
    for (int f = 0; f < 6; f++) gd->wall[f] = PVOF_WALL_NOSLIP;
#ifdef LEFT_WALL_VELOCITY_FREESLIP
    gd->wall[PVOF_LEFT] = PVOF_WALL_FREESLIP;
#endif
#ifdef RIGHT_WALL_VELOCITY_FREESLIP
    gd->wall[PVOF_RIGHT] = PVOF_WALL_FREESLIP;
#endif
#ifdef BOTTOM_WALL_VELOCITY_FREESLIP
    gd->wall[PVOF_BOTTOM] = PVOF_WALL_FREESLIP;
#endif
#ifdef TOP_WALL_VELOCITY_FREESLIP
    gd->wall[PVOF_TOP] = PVOF_WALL_FREESLIP;
#endif
    gd->xmin = p->xmin;
    gd->xmax = p->xmax;
    gd->ymin = p->ymin;
    gd->ymax = p->ymax;
    gd->zmin = p->zmin;
    gd->zmax = p->zmax;
    gd->slab_thickness = p->twod_slab_thickness;
    gd->theta_span = p->axisym_theta_span;
}

/* [flow], [vof], [particle], [conc] and [lsolve] of parties.inp */
static void solver_params(Cart3d_bag *b, pvof_params *pp)
{
    Parameters *p = b->params;
    memset(pp, 0, sizeof(*pp));
    pp->Re = p->Re;
    pp->We = p->We;
    pp->rho1 = p->rho1;
    pp->rho2 = p->rho2;
    pp->mu1 = p->mu1;
    pp->mu2 = p->mu2;
    pp->Cn = p->Cn;
    pp->Pe_CH = p->Pe_CH;
    for (int i = 0; i < 3; i++) pp->grav[i] = p->grav ? p->grav[i] : 0.0;
    pp->richardson = p->richardson ? p->richardson[0] : 1.0;
    pp->dp_dx = p->dp_dx;
    pp->weno_order = p->weno_order;
    pp->ch_iter_max = p->ch_iter_max;
    pp->ch_tol = p->ch_tol;
    pp->CG_MAXIT = p->CG_MAXIT;
    pp->CG_ETOL = p->CG_ETOL;
    pp->P_CG_MAXIT = p->P_CG_MAXIT;
    pp->P_CG_ETOL = p->P_CG_ETOL;
#ifdef SURFACE_TENSION
    pp->surface_tension = 1;
#endif
#ifdef VOF_GRAVITY
    pp->gravity = 1;
#endif
    pp->contact_angle_deg = p->contact_angle_deg;
    pp->N_forcing_loops = p->N_forcing_loops;
}

#if defined(VOF_IBM) && defined(LAG_PARTICLE_RESOLVED)
/* the owned particles of both lists, fixed first (the order in which
 * Particle_initialize numbers them, PARTIES/src/Lagrangian/Particle.c:213-221) */
static int set_particles(Cart3d_bag *b)
{
    Particle_list *lists[2] = {b->lag->p_fixed_list, b->lag->p_mobile_list};
    int n = 0;
    for (int l = 0; l < 2; l++)
        for (Particle *q = lists[l]->start; q; q = q->next) n++;
    pvof_particle *pa = (pvof_particle *)calloc(n > 0 ? (size_t)n : 1, sizeof(pvof_particle));
    if (!pa) return PVOF_ENOMEM;
    int k = 0;
    for (int l = 0; l < 2; l++)
        for (Particle *q = lists[l]->start; q; q = q->next, k++) {
            pa[k].mobile = (l == 1);
            pa[k].X[0] = q->X[0];
            pa[k].X[1] = q->X[1];
            pa[k].R = q->R;
            pa[k].U[0] = q->U[0];
            pa[k].U[1] = q->U[1];
            pa[k].Omega_z = q->Omega[2];
            pa[k].rho_s = q->rho_s;
        }
    int rc = pvof_set_particles(g_ctx, pa, n);
    free(pa);
    return rc;
}

/* the particles' state back into the reference's lists, matched by ID */
static int get_particles(Cart3d_bag *b)
{
    int n = 0;
    Particle_list *lists[2] = {b->lag->p_mobile_list, b->lag->p_fixed_list};
    for (int l = 0; l < 2; l++)
        for (Particle *q = lists[l]->start; q; q = q->next) n++;
    if (n == 0) return PVOF_OK;
    pvof_particle *pa = (pvof_particle *)calloc((size_t)n, sizeof(pvof_particle));
    int *ids = (int *)calloc((size_t)n, sizeof(int));
    double *F = (double *)calloc(3 * (size_t)n, sizeof(double));
    double *T = (double *)calloc(3 * (size_t)n, sizeof(double));
    int got = (pa && ids && F && T) ? pvof_get_particles(g_ctx, pa, ids, F, T, n) : PVOF_ENOMEM;
    for (int k = 0; k < got; k++)
        for (int l = 0; l < 2; l++)
            for (Particle *q = lists[l]->start; q; q = q->next) {
                if (q->ID != ids[k]) continue;
                q->X[0] = pa[k].X[0];
                q->X[1] = pa[k].X[1];
                q->U[0] = pa[k].U[0];
                q->U[1] = pa[k].U[1];
                q->Omega[2] = pa[k].Omega_z;
                for (int i = 0; i < 3; i++) q->F[i] = F[3 * k + i];
                for (int i = 0; i < 3; i++) q->T[i] = T[3 * k + i];
            }
    free(pa);
    free(ids);
    free(F);
    free(T);
    return got < 0 ? got : PVOF_OK;
}
#endif

int pvof_bridge_start(Cart3d_bag *b, int device)
{
    pvof_grid_desc gd;
    pvof_params pp;
    grid_desc(b, &gd);
    solver_params(b, &pp);
    if (g_ctx) pvof_bridge_stop();
    TRYB(pvof_create(&gd, &pp, device, &g_ctx), "pvof_create");
    /* the primary fields; C_L starts as F, as the reference's initialisers
     * leave it (PARTIES/src/IO/VoF_Init.c) */
    TRYB(copy_field(b, PVOF_F_F, 1), "upload F");
    {
        size_t n = pvof_field_block_count(g_ctx, PVOF_F_C_L);
        TRYB(pvof_upload_field(g_ctx, PVOF_F_C_L, FLOW_BLOCK(b->vof->F, b->grid), n), "upload C_L");
    }
    TRYB(copy_field(b, PVOF_F_U, 1), "upload u");
    TRYB(copy_field(b, PVOF_F_V, 1), "upload v");
#ifdef PVOF_BRIDGE_3D
    TRYB(copy_field(b, PVOF_F_W, 1), "upload w");
#endif
    TRYB(copy_field(b, PVOF_F_P, 1), "upload p");
#if defined(VOF_IBM) && defined(LAG_PARTICLE_RESOLVED)
    TRYB(set_particles(b), "pvof_set_particles");
#endif
    TRYB(pvof_set_stage(g_ctx, 0, b->params->dt > 0.0 ? b->params->dt : 1.0), "pvof_set_stage");
    TRYB(pvof_initialize(g_ctx), "pvof_initialize");
    return PVOF_OK;
}

int pvof_bridge_substep(Cart3d_bag *b)
{
    Parameters *p = b->params;
    TRYB(pvof_set_stage(g_ctx, p->which_stage, p->dt), "pvof_set_stage");
    /* Temporal_int_rk3 refreshes the cell-centred velocity before the first
     * stage of every step after the first (Temporal_int.c:420-424) */
#ifndef PVOF_BRIDGE_3D
    /* (the 3D mode evaluates the cell-centred velocity where it reads it) */
    if (p->which_stage == 0 && p->time != 0.0) TRYB(pvof_Velocity_cell_center(g_ctx), "Velocity_cell_center");
#endif
    TRYB(pvof_substep(g_ctx, &g_stats), "pvof_substep");
    return PVOF_OK;
}

int pvof_bridge_download(Cart3d_bag *b)
{
    for (int f = 0; f < PVOF_F_COUNT; f++) TRYB(copy_field(b, f, 0), "download");
#if defined(VOF_IBM) && defined(LAG_PARTICLE_RESOLVED)
    TRYB(get_particles(b), "pvof_get_particles");
#endif
    return PVOF_OK;
}

int pvof_bridge_upload(Cart3d_bag *b)
{
    for (int f = 0; f < PVOF_F_COUNT; f++) TRYB(copy_field(b, f, 1), "upload");
    return PVOF_OK;
}

const pvof_stats *pvof_bridge_stats(void) { return &g_stats; }
pvof_ctx *pvof_bridge_context(void) { return g_ctx; }

void pvof_bridge_stop(void)
{
    if (g_ctx) pvof_destroy(g_ctx);
    g_ctx = NULL;
}

#ifdef PVOF_BRIDGE_ROUTINES
/*
 * The reference's routine names and signatures over the device state.  Each
 * copies the host state to the device, sets the stage and dt from
 * Parameters, runs the pvof_ routine and copies the state back, so the
 * reference's orchestration and its host-side operations between the calls
 * see the arrays they expect.
 */
static void routine_enter(Cart3d_bag *b)
{
    if (pvof_bridge_upload(b) < 0 || pvof_set_stage(g_ctx, b->params->which_stage, b->params->dt) < 0) {
        fprintf(stderr, "pvof bridge: %s\n", pvof_last_error());
        MPI_Abort(MPI_COMM_WORLD, 1);
    }
}

static void routine_leave(Cart3d_bag *b, int rc, const char *name)
{
    if (rc < 0 || pvof_bridge_download(b) < 0) {
        fprintf(stderr, "pvof bridge: %s: %s\n", name, pvof_last_error());
        MPI_Abort(MPI_COMM_WORLD, 1);
    }
}

#define ROUTINE(name, call)            \
    void name(Cart3d_bag *b)           \
    {                                  \
        routine_enter(b);              \
        routine_leave(b, call, #name); \
    }

/* Include/VOF_DIFFUSE.h:7-30 */
ROUTINE(VOF_DIFFUSE_step, pvof_VOF_DIFFUSE_step(g_ctx, &g_stats))
ROUTINE(VOF_DIFFUSE_compute_psi_LG, pvof_VOF_DIFFUSE_compute_psi_LG(g_ctx))
ROUTINE(VOF_DIFFUSE_compute_f_sigma, pvof_VOF_DIFFUSE_compute_f_sigma(g_ctx))
/* Include/VolumeFraction.h:52-84, Eulerian/VOF_SurfaceTension.c:1983-2154 */
ROUTINE(VOF_update_density_viscosity, pvof_VOF_update_density_viscosity(g_ctx))
ROUTINE(VOF_apply_f_sigma_old, pvof_VOF_apply_f_sigma_old(g_ctx))
ROUTINE(VOF_swap_f_sigma, pvof_VOF_swap_f_sigma(g_ctx))
ROUTINE(Velocity_add_gravity_2_RHS, pvof_Velocity_add_gravity_2_RHS(g_ctx))
/* Include/Velocity.h */
ROUTINE(Velocity_cell_center, pvof_Velocity_cell_center(g_ctx))
ROUTINE(Velocity_u_set_implicit_explicit, pvof_Velocity_set_implicit_explicit(g_ctx, 'u'))
ROUTINE(Velocity_v_set_implicit_explicit, pvof_Velocity_set_implicit_explicit(g_ctx, 'v'))
ROUTINE(Velocity_u_set_RHS, pvof_Velocity_set_RHS(g_ctx, 'u'))
ROUTINE(Velocity_v_set_RHS, pvof_Velocity_set_RHS(g_ctx, 'v'))
/* Include/Pressure.h:6-65 */
ROUTINE(Pressure_set_RHS, pvof_Pressure_set_RHS(g_ctx))
ROUTINE(Pressure_compute_preconditioner, pvof_Pressure_compute_preconditioner(g_ctx))
ROUTINE(Pressure_project_velocity, pvof_Pressure_project_velocity(g_ctx))

/* the collapsed third component carries nothing in the 2D modes
 * (TwodOps_collapsed_component_is_inactive, TwodOps.c:3-10) */
void Velocity_w_set_implicit_explicit(Cart3d_bag *b) { (void)b; }
void Velocity_w_set_RHS(Cart3d_bag *b) { (void)b; }

int Pressure_solve_cg(Cart3d_bag *b)
{
    routine_enter(b);
    int rc = pvof_Pressure_solve_cg(g_ctx, &g_stats);
    routine_leave(b, rc, "Pressure_solve_cg");
    return rc;
}

double Pressure_compute_velocity_divergence(Cart3d_bag *b)
{
    double div = 0.0;
    routine_enter(b);
    routine_leave(b, pvof_Pressure_compute_velocity_divergence(g_ctx, &div), "Pressure_compute_velocity_divergence");
    return div;
}

/* msolve_cg.c:525-722 (the Velocity_solve macro of definitions.h:266-267) */
int Velocity_solve_cg(Velocity *vel, Cart3d_bag *b)
{
    if (vel->component == 'w') return 0;
    routine_enter(b);
    int rc = pvof_Velocity_solve_cg(g_ctx, vel->component, &g_stats);
    routine_leave(b, rc, "Velocity_solve_cg");
    return rc;
}

/* Velocity.c:2427-2806 for VEL_TYPE_NORMAL on the velocity arrays themselves;
 * any other array or type stays with the reference's host routine, which a
 * build keeps under another name and passes here */
void Velocity_update_boundaries(double ***a, char which, int type, Cart3d_bag *b)
{
    if (which == 'w') return;
    if (type != VEL_TYPE_NORMAL || (a != b->u->data && a != b->v->data)) {
        fprintf(stderr, "pvof bridge: Velocity_update_boundaries only bridges the velocity arrays\n");
        MPI_Abort(MPI_COMM_WORLD, 1);
    }
    routine_enter(b);
    routine_leave(b, pvof_Velocity_update_boundaries(g_ctx, which), "Velocity_update_boundaries");
}
#endif /* PVOF_BRIDGE_ROUTINES */
