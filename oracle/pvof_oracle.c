/*
 * CPU restatement (oracle) of PARTIES' diffuse-interface RK3 substep.
 *
 * TEST INFRASTRUCTURE ONLY -- see pvof_oracle.h.  Nothing in the product
 * path calls this file.
 *
 * Storage: one ghosted k plane per field, index (i,j) with i in [-G, NX+G),
 * j in [-G, NY+G) exactly as the reference's flow variables, so every loop
 * below runs over the reference's own index ranges.  The 2D modes keep
 * NZ = 2 planes in the reference (NZM = 1, Grid.c:62-64), both identical; the
 * loops that sum over the G range of k (inner products, mass sums) therefore
 * visit the plane twice, in the same accumulation order as the reference.
 * Every arithmetic expression keeps the reference's operand order so that,
 * compiled without FMA contraction, stencil results are bitwise equal to the
 * reference's.
 *
 * File:line citations are to PARTIES/src in the reference tree.
 */
#include "pvof_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* RK3 coefficients, definitions.h:197-204 */
static const double BET[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
static const double BET2[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};
static const double GAMB[3] = {2.0, 25.0 / 4.0, 9.0 / 2.0};
static const double ZETB[3] = {0.0, -17.0 / 4.0, -2.5};

#define NG 3
#define TWOD_RADIAL_EPS 1.0e-14
#define SOLID_MASS_CUTOFF 0.05 /* VOF_DIFFUSE.c:21 */

/* ghost-exchange component classes (Communication.c:168-185, :335-347) */
enum { X_SCALAR = 0, X_UFACE = 1 };

/* scratch arrays beyond the public fields */
enum {
    S_PSI = 0, S_BULK_S, S_CH_AUX1, S_CH_RHS_NM1, S_CH_RES, S_CH_DIR,
    S_FLUX_X, S_FLUX_Y, S_P_RES, S_P_D, S_P_AD, S_P_MINV, S_P_Z,
    S_U_R, S_U_D, S_U_AD, S_V_R, S_V_D, S_V_AD, S_COUNT
};

struct orc {
    pvof_grid_desc g;
    pvof_params p;
    int NX, NY, NZ;
    int SX, SY;          /* plane extents with ghosts */
    int nk;              /* G range planes of the reference (NZ) */
    int twod, planar, axisym;
    double *f[PVOF_F_COUNT];
    double *s[S_COUNT];
    /* metrics, offset so that index -NG is element 0 */
    double *xu, *xc, *dx_u, *dx_c, *idx_u, *idx_c, *i2dx_c;
    double *yv, *yc, *dy_v, *dy_c, *idy_v, *idy_c, *i2dy_c;
    double dz_w0;        /* dz_w at k = 0 */
    double *r_u, *r_c, *inv_r_u, *inv_r_c, *ring_wt_c;
    double slab;
    int stage;
    double dt;
    double time;
};

#define AT(o, a, i, j) ((a)[((size_t)((j) + NG)) * (size_t)(o)->SX + (size_t)((i) + NG)])
#define F(o, id) ((o)->f[(id)])
#define S(o, id) ((o)->s[(id)])

static double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

/* ------------------------------------------------------------------------ */
/* metrics: Grid.c:797-862 (uniform coordinates), :372-420 (widths),        */
/* :871-918 (axisymmetric radii)                                            */
/* ------------------------------------------------------------------------ */
static double *metric(int n) { return (double *)calloc((size_t)n, sizeof(double)) + NG; }
static void metric_free(double *m) { if (m) free(m - NG); }

static void build_metrics(orc_t *o)
{
    int NX = o->NX, NY = o->NY;
    int nxg = NX + 2 * NG, nyg = NY + 2 * NG;
    double Lx = o->g.xmax - o->g.xmin;
    double Ly = o->g.ymax - o->g.ymin;
    double dx = Lx / (double)(NX - 1);
    double dy = Ly / (double)(NY - 1);
    o->xu = metric(nxg); o->xc = metric(nxg); o->dx_u = metric(nxg); o->dx_c = metric(nxg);
    o->idx_u = metric(nxg); o->idx_c = metric(nxg); o->i2dx_c = metric(nxg);
    o->yv = metric(nyg); o->yc = metric(nyg); o->dy_v = metric(nyg); o->dy_c = metric(nyg);
    o->idy_v = metric(nyg); o->idy_c = metric(nyg); o->i2dy_c = metric(nyg);
    for (int i = -NG; i < NX + NG; i++) {
        o->xu[i] = o->g.xmin + i * dx;
        o->xc[i] = o->g.xmin + (0.5 + i) * dx;
    }
    for (int j = -NG; j < NY + NG; j++) {
        o->yv[j] = o->g.ymin + j * dy;
        o->yc[j] = o->g.ymin + (0.5 + j) * dy;
    }
    for (int i = -NG; i < NX + NG - 1; i++) {
        o->dx_u[i] = o->xu[i + 1] - o->xu[i];
        o->dx_c[i] = o->xc[i + 1] - o->xc[i];
        o->idx_u[i] = 1.0 / o->dx_u[i];
        o->idx_c[i] = 1.0 / o->dx_c[i];
    }
    for (int j = -NG; j < NY + NG - 1; j++) {
        o->dy_v[j] = o->yv[j + 1] - o->yv[j];
        o->dy_c[j] = o->yc[j + 1] - o->yc[j];
        o->idy_v[j] = 1.0 / o->dy_v[j];
        o->idy_c[j] = 1.0 / o->dy_c[j];
    }
    for (int i = -NG + 1; i < NX + NG - 1; i++)
        o->i2dx_c[i] = 1.0 / (o->xc[i + 1] - o->xc[i - 1]);
    for (int j = -NG + 1; j < NY + NG - 1; j++)
        o->i2dy_c[j] = 1.0 / (o->yc[j + 1] - o->yc[j - 1]);
    {
        double Lz = o->g.zmax - o->g.zmin;
        double dz = Lz / (double)(o->NZ - 1);
        double zw0 = o->g.zmin + 0 * dz, zw1 = o->g.zmin + 1 * dz;
        o->dz_w0 = zw1 - zw0;
    }
    o->r_u = metric(nxg); o->r_c = metric(nxg); o->inv_r_u = metric(nxg);
    o->inv_r_c = metric(nxg); o->ring_wt_c = metric(nxg);
    if (o->axisym) {
        for (int i = -NG; i <= NX + NG - 1; i++) {
            if (i >= NX + NG) break;
            double ru = fabs(o->xu[i]);
            double rc = fabs(o->xc[i]);
            o->r_u[i] = ru;
            o->r_c[i] = rc;
            o->inv_r_u[i] = (ru > TWOD_RADIAL_EPS) ? 1.0 / ru : 0.0;
            o->inv_r_c[i] = (rc > TWOD_RADIAL_EPS) ? 1.0 / rc : 0.0;
            o->ring_wt_c[i] = o->g.theta_span * rc;
        }
    }
}

/* TwodOps_cell_measure_c (TwodOps.c:311-333) */
static double cell_measure(const orc_t *o, int i, int j)
{
    if (o->planar)
        return o->dx_u[i] * o->dy_v[j] * o->slab;
    return o->dx_u[i] * o->dy_v[j] * o->ring_wt_c[i];
}

/* ------------------------------------------------------------------------ */
/* ghost updates                                                            */
/* ------------------------------------------------------------------------ */

/* Periodic part of Communication_update_ghost_nodes_{x,y} for one rank that
 * is its own neighbour (Communication.c:146-291 and the y analogue). */
static void comm_x(orc_t *o, double *a, int uface)
{
    if (!o->g.periodic[0]) return;
    int NX = o->NX;
    int Is = 0, Ie = NX, ns = NG, nr = NG;
    if (uface) { Is = 1; nr = NG + 1; ns = NG + 1; }
    else Ie = NX - 1;
    double buf[NG + 1];
    for (int j = -NG; j < o->NY + NG; j++) {
        /* send upper, receive lower */
        for (int i = 0; i < ns; i++) buf[i] = AT(o, a, Ie - i - 1, j);
        for (int i = 0; i < nr; i++) AT(o, a, Is - i - 1, j) = buf[i];
        /* send lower, receive upper */
        for (int i = 0; i < NG; i++) buf[i] = AT(o, a, Is + i, j);
        for (int i = 0; i < NG; i++) AT(o, a, Ie + i, j) = buf[i];
    }
}

static void comm_y(orc_t *o, double *a, int vface)
{
    if (!o->g.periodic[1]) return;
    int NY = o->NY;
    int Js = 0, Je = NY, ns = NG, nr = NG;
    if (vface) { Js = 1; nr = NG + 1; ns = NG + 1; }
    else Je = NY - 1;
    double buf[NG + 1];
    for (int i = -NG; i < o->NX + NG; i++) {
        for (int j = 0; j < ns; j++) buf[j] = AT(o, a, i, Je - j - 1);
        for (int j = 0; j < nr; j++) AT(o, a, i, Js - j - 1) = buf[j];
        for (int j = 0; j < NG; j++) buf[j] = AT(o, a, i, Js + j);
        for (int j = 0; j < NG; j++) AT(o, a, i, Je + j) = buf[j];
    }
}

/* component classes: 'c' scalar, 'u' x-face, 'v' y-face */
static void comm(orc_t *o, double *a, char cls)
{
    comm_x(o, a, cls == 'u');
    comm_y(o, a, cls == 'v');
}

/* VOF_DIFFUSE_set_boundary_values (VOF_DIFFUSE.c:571-683) */
static void bc_scalar(orc_t *o, double *f)
{
    int NX = o->NX, NY = o->NY;
    if (!o->g.periodic[0]) {
        for (int j = -NG; j < NY + NG; j++)
            for (int g = 1; g <= NG; g++) {
                if (o->axisym) AT(o, f, -g, j) = AT(o, f, 0, j);
                else if (o->g.wall[PVOF_LEFT] == PVOF_WALL_FREESLIP) AT(o, f, -g, j) = AT(o, f, g - 1, j);
                else AT(o, f, -g, j) = AT(o, f, 0, j);
            }
        int i1 = NX - 1;
        for (int j = -NG; j < NY + NG; j++)
            for (int g = 0; g < NG; g++) {
                if (o->g.wall[PVOF_RIGHT] == PVOF_WALL_FREESLIP) AT(o, f, i1 + g, j) = AT(o, f, i1 - 1 - g, j);
                else AT(o, f, i1 + g, j) = AT(o, f, i1 - 1, j);
            }
    }
    if (!o->g.periodic[1]) {
        for (int i = -NG; i < NX + NG; i++)
            for (int g = 1; g <= NG; g++) {
                if (o->g.wall[PVOF_BOTTOM] == PVOF_WALL_FREESLIP) AT(o, f, i, -g) = AT(o, f, i, g - 1);
                else AT(o, f, i, -g) = AT(o, f, i, 0);
            }
        int j1 = NY - 1;
        for (int i = -NG; i < NX + NG; i++)
            for (int g = 0; g < NG; g++) {
                if (o->g.wall[PVOF_TOP] == PVOF_WALL_FREESLIP) AT(o, f, i, j1 + g) = AT(o, f, i, j1 - 1 - g);
                else AT(o, f, i, j1 + g) = AT(o, f, i, j1 - 1);
            }
    }
    comm(o, f, 'c');
}

/* Pressure_apply_BCs (psolve_cg.c:358-529) */
static void bc_pressure(orc_t *o, double *phi)
{
    int NX = o->NX, NY = o->NY;
    if (!o->g.periodic[0]) {
        for (int j = -NG; j < NY + NG; j++) {
            AT(o, phi, -1, j) = AT(o, phi, 0, j);
            AT(o, phi, NX - 1, j) = AT(o, phi, NX - 2, j);
        }
    }
    if (!o->g.periodic[1]) {
        for (int i = -NG; i < NX + NG; i++) {
            AT(o, phi, i, -1) = AT(o, phi, i, 0);
            AT(o, phi, i, NY - 1) = AT(o, phi, i, NY - 2);
        }
    }
}

/* Velocity_update_boundaries (Velocity.c:2427-2806), planar/axisymmetric
 * walls, no lid velocity; cg != 0 is VEL_TYPE_CG. */
static void bc_velocity(orc_t *o, double *a, char comp, int cg)
{
    int NX = o->NX, NY = o->NY;
    if (!o->g.periodic[0]) {
        if (comp == 'u') {
            if (!cg || o->axisym)
                for (int j = -NG; j < NY + NG; j++) AT(o, a, 0, j) = 0.0;
        } else {
            for (int j = 0; j < NY; j++) {
                if (o->axisym) AT(o, a, -1, j) = AT(o, a, 0, j);
                else if (o->g.wall[PVOF_LEFT] == PVOF_WALL_NOSLIP) AT(o, a, -1, j) = -AT(o, a, 0, j);
                else AT(o, a, -1, j) = AT(o, a, 0, j);
            }
        }
        if (comp == 'u') {
            if (!cg)
                for (int j = -NG; j < NY + NG; j++) AT(o, a, NX - 1, j) = 0.0;
        } else {
            for (int j = 0; j < NY; j++) {
                if (o->g.wall[PVOF_RIGHT] == PVOF_WALL_NOSLIP) AT(o, a, NX - 1, j) = -AT(o, a, NX - 2, j);
                else AT(o, a, NX - 1, j) = AT(o, a, NX - 2, j);
            }
        }
    }
    if (!o->g.periodic[1]) {
        if (comp == 'v') {
            if (!cg)
                for (int i = -NG; i < NX + NG; i++) AT(o, a, i, 0) = 0.0;
        } else {
            for (int i = 0; i < NX; i++) {
                if (o->g.wall[PVOF_BOTTOM] == PVOF_WALL_NOSLIP) AT(o, a, i, -1) = -AT(o, a, i, 0);
                else AT(o, a, i, -1) = AT(o, a, i, 0);
            }
        }
        if (comp == 'v') {
            if (!cg)
                for (int i = -NG; i < NX + NG; i++) AT(o, a, i, NY - 1) = 0.0;
        } else {
            for (int i = 0; i < NX; i++) {
                if (o->g.wall[PVOF_TOP] == PVOF_WALL_NOSLIP) AT(o, a, i, NY - 1) = -AT(o, a, i, NY - 2);
                else AT(o, a, i, NY - 1) = AT(o, a, i, NY - 2);
            }
        }
    }
    comm(o, a, comp == 'u' ? 'u' : (comp == 'v' ? 'v' : 'c'));
}

static void copy_withghost(orc_t *o, const double *src, double *dst)
{
    memcpy(dst, src, sizeof(double) * (size_t)o->SX * (size_t)o->SY);
}

static void zero_withghost(orc_t *o, double *a)
{
    memset(a, 0, sizeof(double) * (size_t)o->SX * (size_t)o->SY);
}

/* ------------------------------------------------------------------------ */
/* TwodOps helpers (TwodOps.c)                                              */
/* ------------------------------------------------------------------------ */

/* TwodOps_scalar_laplacian (TwodOps.c:159-199) */
static double scalar_laplacian(const orc_t *o, const double *phi, int i, int j)
{
    double dfdxE = (AT(o, phi, i + 1, j) - AT(o, phi, i, j)) * o->idx_c[i];
    double dfdxW = (AT(o, phi, i, j) - AT(o, phi, i - 1, j)) * ((i != 0) ? o->idx_c[i - 1] : o->idx_c[i]);
    double dfdyN = (AT(o, phi, i, j + 1) - AT(o, phi, i, j)) * o->idy_c[j];
    double dfdyS = (AT(o, phi, i, j) - AT(o, phi, i, j - 1)) * ((j != 0) ? o->idy_c[j - 1] : o->idy_c[j]);
    if (o->planar)
        return (dfdxE - dfdxW) * o->idx_u[i] + (dfdyN - dfdyS) * o->idy_v[j];
    return (o->r_u[i + 1] * dfdxE - o->r_u[i] * dfdxW) * o->idx_u[i] * o->inv_r_c[i] +
           (dfdyN - dfdyS) * o->idy_v[j];
}

/* TwodOps_scalar_flux_divergence (TwodOps.c:201-229) */
static double scalar_flux_divergence(const orc_t *o, const double *fx, const double *fy, int i, int j)
{
    double div_x = (AT(o, fx, i + 1, j) - AT(o, fx, i, j)) / o->dx_c[i];
    double div_y = (AT(o, fy, i, j + 1) - AT(o, fy, i, j)) / o->dy_c[j];
    if (o->planar)
        return div_x + div_y;
    return (o->r_u[i + 1] * AT(o, fx, i + 1, j) - o->r_u[i] * AT(o, fx, i, j)) * o->inv_r_c[i] / o->dx_c[i] + div_y;
}

/* TwodOps_cell_center_divergence (TwodOps.c:12-43) */
static double cell_center_divergence(const orc_t *o, const double *u, const double *v, int i, int j,
                                     double idx_u, double idy_v)
{
    double dudx = (AT(o, u, i + 1, j) - AT(o, u, i, j)) * idx_u;
    double dvdy = (AT(o, v, i, j + 1) - AT(o, v, i, j)) * idy_v;
    if (o->planar)
        return dudx + dvdy;
    return (o->r_u[i + 1] * AT(o, u, i + 1, j) - o->r_u[i] * AT(o, u, i, j)) * idx_u * o->inv_r_c[i] + dvdy;
}

/* TwodOps_build_scalar_face_coeffs (TwodOps.c:45-88), z couplings dropped */
static void scalar_face_coeffs(const orc_t *o, int i, double bxm, double bxp, double bym, double byp,
                               double *cxm, double *cxp, double *cym, double *cyp)
{
    const double idx2 = o->idx_c[1] * o->idx_c[1];
    const double idy2 = o->idy_c[1] * o->idy_c[1];
    *cxm = bxm * idx2;
    *cxp = bxp * idx2;
    *cym = bym * idy2;
    *cyp = byp * idy2;
    if (o->planar) return;
    *cxm = o->r_u[i] * bxm * o->inv_r_c[i] * idx2;
    *cxp = o->r_u[i + 1] * bxp * o->inv_r_c[i] * idx2;
}

/* TwodOps_pressure_row_weight (TwodOps.c:144-157) */
static double row_weight(const orc_t *o, int i) { return o->axisym ? o->r_c[i] : 1.0; }

/* TwodOps_u_cv_x_flux_divergence / v_cv / diag / radial (TwodOps.c:231-309) */
static double u_cv_x_div(const orc_t *o, int i, double fe, double fw)
{
    if (!o->axisym) return (fe - fw) * o->idx_c[i - 1];
    return (o->r_c[i] * fe - o->r_c[i - 1] * fw) * o->idx_c[i - 1] * o->inv_r_u[i];
}
static double v_cv_x_div(const orc_t *o, int i, double fe, double fw)
{
    if (!o->axisym) return (fe - fw) * o->idx_u[i];
    return (o->r_u[i + 1] * fe - o->r_u[i] * fw) * o->idx_u[i] * o->inv_r_c[i];
}
static double u_cv_x_diag(const orc_t *o, int i, double ce, double cw)
{
    if (!o->axisym) return (ce + cw) * o->idx_c[i - 1];
    return (o->r_c[i] * ce + o->r_c[i - 1] * cw) * o->idx_c[i - 1] * o->inv_r_u[i];
}
static double v_cv_x_diag(const orc_t *o, int i, double ce, double cw)
{
    if (!o->axisym) return (ce + cw) * o->idx_u[i];
    return (o->r_u[i + 1] * ce + o->r_u[i] * cw) * o->idx_u[i] * o->inv_r_c[i];
}
static double axisym_ur_term(const orc_t *o, int i, double coeff, double u)
{
    if (!o->axisym) return 0.0;
    return -2.0 * coeff * u * o->inv_r_u[i] * o->inv_r_u[i];
}
static double axisym_ur_coeff(const orc_t *o, int i, double coeff)
{
    if (!o->axisym) return 0.0;
    return 2.0 * coeff * o->inv_r_u[i] * o->inv_r_u[i];
}

/* ------------------------------------------------------------------------ */
/* Cahn-Hilliard substep                                                    */
/* ------------------------------------------------------------------------ */

/* sum over the G range of k (nk identical planes) of measure * a * b,
 * diffuse_inner_product (VOF_DIFFUSE.c:128-146) */
static double ch_inner(const orc_t *o, const double *a, const double *b)
{
    double s = 0.0;
    for (int k = 0; k < o->nk; k++)
        for (int j = 0; j < o->NY; j++)
            for (int i = 0; i < o->NX; i++)
                s += cell_measure(o, i, j) * AT(o, a, i, j) * AT(o, b, i, j);
    return s;
}

/* VOF_DIFFUSE_compute_laplacian (VOF_DIFFUSE.c:834-861) */
static void compute_laplacian(orc_t *o, double *in, double *lap)
{
    bc_scalar(o, in);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, lap, i, j) = scalar_laplacian(o, in, i, j);
    bc_scalar(o, lap);
}

/* VOF_DIFFUSE_update_phase_cache (VOF_DIFFUSE.c:108-126) */
static void update_phase_cache(orc_t *o)
{
    double *CL = F(o, PVOF_F_C_L), *CS = F(o, PVOF_F_C_S), *CG = F(o, PVOF_F_C_G);
    size_t n = (size_t)o->SX * (size_t)o->SY;
    for (size_t q = 0; q < n; q++)
        CG[q] = clamp01(1.0 - CL[q] - CS[q]);
    copy_withghost(o, CL, F(o, PVOF_F_F));
}

/* diffuse_bound_liquid_fraction (VOF_DIFFUSE.c:1093-1127).  The reference
 * clamps each of its nk identical planes; the second visit here reads the
 * pre-clamp values kept in scratch so the returned mass change accumulates
 * exactly as in the reference. */
static double bound_liquid_fraction(orc_t *o)
{
    double *CL = F(o, PVOF_F_C_L), *CS = F(o, PVOF_F_C_S), *CG = F(o, PVOF_F_C_G);
    double *old = S(o, S_P_Z);
    copy_withghost(o, CL, old);
    double delta = 0.0;
    for (int k = 0; k < o->nk; k++)
        for (int j = 0; j < o->NY; j++)
            for (int i = 0; i < o->NX; i++) {
                double old_cl = AT(o, old, i, j);
                double cs = AT(o, CS, i, j);
                double max_cl = 1.0 - cs;
                if (max_cl < 0.0) max_cl = 0.0;
                if (max_cl > 1.0) max_cl = 1.0;
                double new_cl = old_cl;
                if (new_cl < 0.0) new_cl = 0.0;
                if (new_cl > max_cl) new_cl = max_cl;
                AT(o, CL, i, j) = new_cl;
                AT(o, CG, i, j) = clamp01(1.0 - new_cl - cs);
                if (cs < SOLID_MASS_CUTOFF) {
                    double m = cell_measure(o, i, j);
                    if (o->twod && o->nk > 1) m /= (double)o->nk;
                    delta += (new_cl - old_cl) * m;
                }
            }
    return delta;
}

/* VOF_DIFFUSE_init (VOF_DIFFUSE.c:524-568), no solids */
static void vof_diffuse_init(orc_t *o)
{
    double *CL = F(o, PVOF_F_C_L), *Fv = F(o, PVOF_F_F);
    size_t n = (size_t)o->SX * (size_t)o->SY;
    for (size_t q = 0; q < n; q++) CL[q] = clamp01(Fv[q]);
    bc_scalar(o, CL);
    update_phase_cache(o);
    bound_liquid_fraction(o);
    bc_scalar(o, CL);
    update_phase_cache(o);
    bc_scalar(o, CL);
    update_phase_cache(o);
    bc_scalar(o, F(o, PVOF_F_C_G));
}

/* diffuse_weno5_left (VOF_DIFFUSE.c:431-451); squares through pow(., 2.0)
 * as the reference does, so the oracle rounds exactly like it on this CPU */
static double weno5_left(double v0, double v1, double v2, double v3, double v4)
{
    const double eps = 1e-6;
    double q0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
    double q1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
    double q2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
    double b0 = 13.0 / 12.0 * pow(v0 - 2.0 * v1 + v2, 2.0) + 0.25 * pow(v0 - 4.0 * v1 + 3.0 * v2, 2.0);
    double b1 = 13.0 / 12.0 * pow(v1 - 2.0 * v2 + v3, 2.0) + 0.25 * pow(v1 - v3, 2.0);
    double b2 = 13.0 / 12.0 * pow(v2 - 2.0 * v3 + v4, 2.0) + 0.25 * pow(3.0 * v2 - 4.0 * v3 + v4, 2.0);
    double a0 = 0.1 / ((eps + b0) * (eps + b0));
    double a1 = 0.6 / ((eps + b1) * (eps + b1));
    double a2 = 0.3 / ((eps + b2) * (eps + b2));
    double asum = a0 + a1 + a2;
    return (a0 * q0 + a1 * q1 + a2 * q2) / asum;
}

/* VOF_DIFFUSE_advect_WENO5 (VOF_DIFFUSE.c:931-996) */
static void advect_weno5(orc_t *o, double *rhs_out)
{
    double *CL = F(o, PVOF_F_C_L), *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V);
    double *fx = S(o, S_FLUX_X), *fy = S(o, S_FLUX_Y);
    int w5 = (o->p.weno_order == 5);
    bc_scalar(o, CL);
    zero_withghost(o, fx);
    zero_withghost(o, fy);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            double vel = AT(o, u, i, j), st;
            if (w5) st = (vel >= 0.0) ? weno5_left(AT(o, CL, i - 3, j), AT(o, CL, i - 2, j), AT(o, CL, i - 1, j), AT(o, CL, i, j), AT(o, CL, i + 1, j))
                                      : weno5_left(AT(o, CL, i + 2, j), AT(o, CL, i + 1, j), AT(o, CL, i, j), AT(o, CL, i - 1, j), AT(o, CL, i - 2, j));
            else st = (vel >= 0.0) ? AT(o, CL, i - 1, j) : AT(o, CL, i, j);
            AT(o, fx, i, j) = vel * st;
            vel = AT(o, v, i, j);
            if (w5) st = (vel >= 0.0) ? weno5_left(AT(o, CL, i, j - 3), AT(o, CL, i, j - 2), AT(o, CL, i, j - 1), AT(o, CL, i, j), AT(o, CL, i, j + 1))
                                      : weno5_left(AT(o, CL, i, j + 2), AT(o, CL, i, j + 1), AT(o, CL, i, j), AT(o, CL, i, j - 1), AT(o, CL, i, j - 2));
            else st = (vel >= 0.0) ? AT(o, CL, i, j - 1) : AT(o, CL, i, j);
            AT(o, fy, i, j) = vel * st;
        }
    comm(o, fx, 'u');
    comm(o, fy, 'v');
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, rhs_out, i, j) = -scalar_flux_divergence(o, fx, fy, i, j);
    bc_scalar(o, rhs_out);
}

/* VOF_DIFFUSE_compute_bulk_S + explicit_diffusion (VOF_DIFFUSE.c:865-885, :998-1016) */
static void explicit_diffusion(orc_t *o, double *rhs_out)
{
    double *CL = F(o, PVOF_F_C_L), *CS = F(o, PVOF_F_C_S), *bS = S(o, S_BULK_S), *aux = S(o, S_CH_AUX1);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            double c = AT(o, CL, i, j), cs = AT(o, CS, i, j);
            AT(o, bS, i, j) = 0.5 * c - 1.5 * c * c + c * c * c - c * cs * (1.0 - c - cs);
        }
    bc_scalar(o, bS);
    compute_laplacian(o, bS, aux);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, rhs_out, i, j) = AT(o, aux, i, j) / o->p.Pe_CH;
    bc_scalar(o, rhs_out);
}

/* diffuse_apply_biharmonic_operator (VOF_DIFFUSE.c:318-337) */
static void apply_biharmonic(orc_t *o, double *x, double *Ax, double a_dt, double bih)
{
    double *lap = S(o, S_CH_AUX1), *b2 = F(o, PVOF_F_PSI_LG);
    compute_laplacian(o, x, lap);
    compute_laplacian(o, lap, b2);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, Ax, i, j) = a_dt * AT(o, x, i, j) + bih * AT(o, b2, i, j);
}

/* diffuse_solve_biharmonic_pcg (VOF_DIFFUSE.c:339-429) */
static int solve_biharmonic(orc_t *o, double *x, double *b, double a_dt, double bih, double *rel_out)
{
    double *r = S(o, S_CH_RES), *p = S(o, S_CH_DIR), *z = S(o, S_BULK_S), *Ap = F(o, PVOF_F_LAP_C);
    int maxit = (o->p.ch_iter_max > 0) ? o->p.ch_iter_max : o->p.CG_MAXIT;
    double tol = (o->p.ch_tol > 0.0) ? o->p.ch_tol : o->p.CG_ETOL;
    apply_biharmonic(o, x, Ap, a_dt, bih);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            AT(o, r, i, j) = AT(o, b, i, j) - AT(o, Ap, i, j);
            AT(o, z, i, j) = AT(o, r, i, j);
            AT(o, p, i, j) = AT(o, z, i, j);
        }
    double rhs_norm = sqrt(ch_inner(o, b, b));
    if (rhs_norm < 1e-30) rhs_norm = 1.0;
    double rz = ch_inner(o, r, z);
    double rel = sqrt(ch_inner(o, r, r)) / rhs_norm;
    int iter = 0;
    if (rel < tol) {
        *rel_out = rel;
        bc_scalar(o, x);
        return iter;
    }
    while (iter < maxit) {
        apply_biharmonic(o, p, Ap, a_dt, bih);
        double pAp = ch_inner(o, p, Ap);
        if (fabs(pAp) < 1e-30) break;
        double alpha = rz / pAp;
        for (int j = 0; j < o->NY; j++)
            for (int i = 0; i < o->NX; i++) {
                AT(o, x, i, j) += alpha * AT(o, p, i, j);
                AT(o, r, i, j) -= alpha * AT(o, Ap, i, j);
                AT(o, z, i, j) = AT(o, r, i, j);
            }
        ++iter;
        rel = sqrt(ch_inner(o, r, r)) / rhs_norm;
        if (rel < tol) break;
        double rz_new = ch_inner(o, r, z);
        double beta = rz_new / (rz + 1e-30);
        for (int j = 0; j < o->NY; j++)
            for (int i = 0; i < o->NX; i++)
                AT(o, p, i, j) = AT(o, z, i, j) + beta * AT(o, p, i, j);
        rz = rz_new;
    }
    *rel_out = rel;
    bc_scalar(o, x);
    return iter;
}

/* VOF_DIFFUSE_solve_implicit_biharmonic (VOF_DIFFUSE.c:1018-1069) */
static int solve_implicit_biharmonic(orc_t *o, double *rhs, double *rel_out)
{
    double a_dt = 1.0 / (o->dt * BET[o->stage]);
    double bih = o->p.Cn * o->p.Cn / o->p.Pe_CH;
    double *psi = S(o, S_PSI), *aux = S(o, S_CH_AUX1), *psiLG = F(o, PVOF_F_PSI_LG);
    copy_withghost(o, F(o, PVOF_F_C_L), psi);
    compute_laplacian(o, psi, aux);
    compute_laplacian(o, aux, psiLG);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, rhs, i, j) -= bih * AT(o, psiLG, i, j);
    return solve_biharmonic(o, F(o, PVOF_F_C_L), rhs, a_dt, bih, rel_out);
}

/* VOF_DIFFUSE_step (VOF_DIFFUSE.c:1262-1359), no solids */
static void vof_diffuse_step(orc_t *o, pvof_stats *st)
{
    int s = o->stage;
    double a_dt = 1.0 / (o->dt * BET[s]);
    double *cur = F(o, PVOF_F_CH_RHS_CUR), *tmp = S(o, S_CH_AUX1), *vec = S(o, S_CH_RHS_NM1);
    double *CL = F(o, PVOF_F_C_L), *rn = F(o, PVOF_F_CH_RHS_N);
    advect_weno5(o, cur);
    explicit_diffusion(o, tmp);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++)
            AT(o, cur, i, j) += AT(o, tmp, i, j);
    bc_scalar(o, cur);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            if (s == 0) AT(o, vec, i, j) = a_dt * AT(o, CL, i, j) + GAMB[0] * AT(o, cur, i, j);
            else AT(o, vec, i, j) = a_dt * AT(o, CL, i, j) + GAMB[s] * AT(o, cur, i, j) + ZETB[s] * AT(o, rn, i, j);
        }
    bc_scalar(o, vec);
    double rel = 0.0;
    int it = solve_implicit_biharmonic(o, vec, &rel);
    double dm = bound_liquid_fraction(o);
    bc_scalar(o, CL);
    update_phase_cache(o);
    /* history shift: ch_rhs_nm1 <- ch_rhs_n, ch_rhs_n <- rhs_cur */
    copy_withghost(o, rn, vec);
    copy_withghost(o, cur, rn);
    if (st) { st->ch_iters = it; st->ch_rel_res = rel; st->clamp_mass = dm; }
}

/* VOF_DIFFUSE_update_density_viscosity (VOF_DIFFUSE.c:1453-1488) */
static void update_density_viscosity(orc_t *o)
{
    const double rho_g = o->p.rho2 / o->p.rho1, mu_g = o->p.mu2 / o->p.mu1;
    const double rho_s = 1.0, mu_s = 1.0;
    double *CL = F(o, PVOF_F_C_L), *CS = F(o, PVOF_F_C_S), *CG = F(o, PVOF_F_C_G);
    double *rho = F(o, PVOF_F_RHO), *mu = F(o, PVOF_F_MU);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            AT(o, rho, i, j) = AT(o, CL, i, j) + rho_s * AT(o, CS, i, j) + rho_g * AT(o, CG, i, j);
            AT(o, mu, i, j) = AT(o, CL, i, j) + mu_s * AT(o, CS, i, j) + mu_g * AT(o, CG, i, j);
        }
    bc_scalar(o, rho);
    bc_scalar(o, mu);
}

/* VOF_DIFFUSE_compute_psi_LG (VOF_DIFFUSE.c:907-929) */
static void compute_psi_LG(orc_t *o)
{
    double *CL = F(o, PVOF_F_C_L), *lap = F(o, PVOF_F_LAP_C), *psi = F(o, PVOF_F_PSI_LG);
    double cn2 = o->p.Cn * o->p.Cn;
    compute_laplacian(o, CL, lap);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) {
            double c = AT(o, CL, i, j);
            AT(o, psi, i, j) = c * c * c - 1.5 * c * c + 0.5 * c - cn2 * AT(o, lap, i, j);
        }
    bc_scalar(o, psi);
}

/* loop bounds of the face-centred momentum arrays (e.g. Velocity.c:395-410) */
static void u_range(const orc_t *o, int *i0, int *i1, int *j0, int *j1)
{
    *i0 = 1; *i1 = o->NX - 1; *j0 = 0; *j1 = o->NY - 1;
    if (o->g.periodic[0]) *i1 = o->NX;
}
static void v_range(const orc_t *o, int *i0, int *i1, int *j0, int *j1)
{
    *i0 = 0; *i1 = o->NX - 1; *j0 = 1; *j1 = o->NY - 1;
    if (o->g.periodic[1]) *j1 = o->NY;
}

/* VOF_DIFFUSE_compute_f_sigma (VOF_DIFFUSE.c:1364-1445) */
static void compute_f_sigma(orc_t *o)
{
    double *CL = F(o, PVOF_F_C_L), *CG = F(o, PVOF_F_C_G), *CS = F(o, PVOF_F_C_S), *psi = F(o, PVOF_F_PSI_LG);
    double *fx = F(o, PVOF_F_FSIG_NEW_X), *fy = F(o, PVOF_F_FSIG_NEW_Y);
    const double scale = 2.0 * 6.0 * sqrt(2.0) / (o->p.Cn * o->p.We + 1e-30);
    for (int j = 0; j < o->NY; j++)
        for (int i = 0; i < o->NX; i++) { AT(o, fx, i, j) = 0.0; AT(o, fy, i, j) = 0.0; }
    int i0, i1, j0, j1;
    u_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double cl = 0.5 * (AT(o, CL, i, j) + AT(o, CL, i - 1, j));
            double cg = 0.5 * (AT(o, CG, i, j) + AT(o, CG, i - 1, j));
            double cs = 0.5 * (AT(o, CS, i, j) + AT(o, CS, i - 1, j));
            if (cl < 0.005 || cl > 0.995 || cg < 0.005 || cg > 0.995 || cs > 0.05) continue;
            double pf = 0.5 * (AT(o, psi, i, j) + AT(o, psi, i - 1, j));
            double gc = (AT(o, CL, i, j) - AT(o, CL, i - 1, j)) * o->idx_c[i - 1];
            AT(o, fx, i, j) = scale * pf * gc;
        }
    v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double cl = 0.5 * (AT(o, CL, i, j) + AT(o, CL, i, j - 1));
            double cg = 0.5 * (AT(o, CG, i, j) + AT(o, CG, i, j - 1));
            double cs = 0.5 * (AT(o, CS, i, j) + AT(o, CS, i, j - 1));
            if (cl < 0.005 || cl > 0.995 || cg < 0.005 || cg > 0.995 || cs > 0.05) continue;
            double pf = 0.5 * (AT(o, psi, i, j) + AT(o, psi, i, j - 1));
            double gc = (AT(o, CL, i, j) - AT(o, CL, i, j - 1)) * o->idy_c[j - 1];
            AT(o, fy, i, j) = scale * pf * gc;
        }
}

/* VOF_apply_f_sigma_old (VOF_SurfaceTension.c:1983-2041) */
static void apply_f_sigma_old(orc_t *o)
{
    int i0, i1, j0, j1;
    double *ru = F(o, PVOF_F_U_RHS), *rv = F(o, PVOF_F_V_RHS);
    double *fx = F(o, PVOF_F_FSIG_OLD_X), *fy = F(o, PVOF_F_FSIG_OLD_Y);
    u_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) AT(o, ru, i, j) += AT(o, fx, i, j);
    v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) AT(o, rv, i, j) += AT(o, fy, i, j);
}

/* VOF_swap_f_sigma (VOF_SurfaceTension.c:2055-2071) */
static void swap_f_sigma(orc_t *o)
{
    double *t = o->f[PVOF_F_FSIG_OLD_X];
    o->f[PVOF_F_FSIG_OLD_X] = o->f[PVOF_F_FSIG_NEW_X];
    o->f[PVOF_F_FSIG_NEW_X] = t;
    t = o->f[PVOF_F_FSIG_OLD_Y];
    o->f[PVOF_F_FSIG_OLD_Y] = o->f[PVOF_F_FSIG_NEW_Y];
    o->f[PVOF_F_FSIG_NEW_Y] = t;
}

/* Velocity_add_gravity_2_RHS (VOF_SurfaceTension.c:2075-2154) */
static void add_gravity(orc_t *o)
{
    const double *gr = o->p.grav;
    double Ri = o->p.richardson;
    double gm = sqrt(gr[0] * gr[0] + gr[1] * gr[1]);
    double gx = 0, gy = 0;
    if (gm > 0.0) { gx = gr[0] / gm; gy = gr[1] / gm; }
    double *rho = F(o, PVOF_F_RHO), *ru = F(o, PVOF_F_U_RHS), *rv = F(o, PVOF_F_V_RHS);
    int i0, i1, j0, j1;
    u_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i - 1, j));
            AT(o, ru, i, j) += 2.0 * rf * Ri * gx;
        }
    v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i, j - 1));
            AT(o, rv, i, j) += 2.0 * rf * Ri * gy;
        }
}

/* Velocity_cell_center (Velocity.c:278-357) */
static void cell_center(orc_t *o)
{
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V), *ub = F(o, PVOF_F_U_BC), *vb = F(o, PVOF_F_V_BC);
    comm(o, u, 'u');
    comm(o, v, 'v');
    for (int j = -NG; j < o->NY + NG - 1; j++)
        for (int i = -NG; i < o->NX + NG - 1; i++) {
            AT(o, ub, i, j) = 0.5 * (AT(o, u, i, j) + AT(o, u, i + 1, j));
            AT(o, vb, i, j) = 0.5 * (AT(o, v, i, j) + AT(o, v, i, j + 1));
        }
}

/* harmonic of averaged viscosities (Velocity.c:446-470, msolve_cg.c:78-79) */
static double harm(double a, double b) { return 2.0 * a * b / (a + b + 1e-12); }
static double avg2(double a, double b) { return 0.5 * (a + b); }

/* Velocity_u_set_implicit_explicit (Velocity.c:366-762), diffuse VOF */
static void u_implicit_explicit(orc_t *o)
{
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V), *ub = F(o, PVOF_F_U_BC), *mu = F(o, PVOF_F_MU);
    double *ex = F(o, PVOF_F_U_EXPLICIT), *im = F(o, PVOF_F_U_IMPLICIT), *vx = F(o, PVOF_F_U_VISC_EXPLICIT);
    double iRe = 1.0 / o->p.Re;
    int i0, i1, j0, j1;
    u_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double muE = AT(o, mu, i, j), muW = AT(o, mu, i - 1, j);
            double mu_yp = 2.0 * (0.5 * (AT(o, mu, i - 1, j + 1) + AT(o, mu, i, j + 1))) * (0.5 * (AT(o, mu, i - 1, j) + AT(o, mu, i, j))) /
                           ((0.5 * (AT(o, mu, i - 1, j + 1) + AT(o, mu, i, j + 1))) + (0.5 * (AT(o, mu, i - 1, j) + AT(o, mu, i, j))) + 1e-12);
            double mu_ym = 2.0 * (0.5 * (AT(o, mu, i - 1, j) + AT(o, mu, i, j))) * (0.5 * (AT(o, mu, i - 1, j - 1) + AT(o, mu, i, j - 1))) /
                           ((0.5 * (AT(o, mu, i - 1, j) + AT(o, mu, i, j))) + (0.5 * (AT(o, mu, i - 1, j - 1) + AT(o, mu, i, j - 1))) + 1e-12);
            double dudxE = (AT(o, u, i + 1, j) - AT(o, u, i, j)) * o->idx_u[i];
            double dudxW = (AT(o, u, i, j) - AT(o, u, i - 1, j)) * o->idx_u[i - 1];
            double dudyN = (AT(o, u, i, j + 1) - AT(o, u, i, j)) * o->idy_c[j];
            double dudyS = (AT(o, u, i, j) - AT(o, u, i, j - 1)) * o->idy_c[j - 1];
            double d2udy2 = iRe * (mu_yp * dudyN - mu_ym * dudyS) * o->idy_v[j];
            double dvdxN = (AT(o, v, i, j + 1) - AT(o, v, i - 1, j + 1)) * o->idx_c[i - 1];
            double dvdxS = (AT(o, v, i, j) - AT(o, v, i - 1, j)) * o->idx_c[i - 1];
            double d2udx2 = iRe * u_cv_x_div(o, i, muE * dudxE, muW * dudxW);
            double ddydvdx = iRe * (mu_yp * dvdxN - mu_ym * dvdxS) * o->idy_v[j];
            double axc = axisym_ur_term(o, i, iRe * 0.5 * (muE + muW), AT(o, u, i, j));
            double vCN = 0.5 * (AT(o, v, i, j + 1) + AT(o, v, i - 1, j + 1));
            double vCS = 0.5 * (AT(o, v, i, j) + AT(o, v, i - 1, j));
            double uuE = AT(o, ub, i, j) * AT(o, ub, i, j);
            double uuW = AT(o, ub, i - 1, j) * AT(o, ub, i - 1, j);
            double uvN = 0.5 * (AT(o, u, i, j) + AT(o, u, i, j + 1)) * vCN;
            double uvS = 0.5 * (AT(o, u, i, j) + AT(o, u, i, j - 1)) * vCS;
            double duudx = u_cv_x_div(o, i, uuE, uuW);
            double duvdy = (uvN - uvS) * o->idy_v[j];
            AT(o, ex, i, j) = -(duudx + duvdy);
            AT(o, vx, i, j) = d2udx2 + ddydvdx;
            AT(o, im, i, j) = d2udx2 + d2udy2 + axc;
        }
}

/* Velocity_v_set_implicit_explicit (Velocity.c:771-1148), diffuse VOF */
static void v_implicit_explicit(orc_t *o)
{
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V), *vb = F(o, PVOF_F_V_BC), *mu = F(o, PVOF_F_MU);
    double *ex = F(o, PVOF_F_V_EXPLICIT), *im = F(o, PVOF_F_V_IMPLICIT), *vx = F(o, PVOF_F_V_VISC_EXPLICIT);
    double iRe = 1.0 / o->p.Re;
    int i0, i1, j0, j1;
    v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double mu_xp = 2.0 * (0.5 * (AT(o, mu, i + 1, j - 1) + AT(o, mu, i + 1, j))) * (0.5 * (AT(o, mu, i, j - 1) + AT(o, mu, i, j))) /
                           ((0.5 * (AT(o, mu, i + 1, j - 1) + AT(o, mu, i + 1, j))) + (0.5 * (AT(o, mu, i, j - 1) + AT(o, mu, i, j))) + 1e-12);
            double mu_xm = 2.0 * (0.5 * (AT(o, mu, i, j - 1) + AT(o, mu, i, j))) * (0.5 * (AT(o, mu, i - 1, j - 1) + AT(o, mu, i - 1, j))) /
                           ((0.5 * (AT(o, mu, i, j - 1) + AT(o, mu, i, j))) + (0.5 * (AT(o, mu, i - 1, j - 1) + AT(o, mu, i - 1, j))) + 1e-12);
            double mu_yp = AT(o, mu, i, j), mu_ym = AT(o, mu, i, j - 1);
            double dvdxE = (AT(o, v, i + 1, j) - AT(o, v, i, j)) * o->idx_c[i];
            double dvdxW = (AT(o, v, i, j) - AT(o, v, i - 1, j)) * o->idx_c[i - 1];
            double dvdyN = (AT(o, v, i, j + 1) - AT(o, v, i, j)) * o->idy_v[j];
            double dvdyS = (AT(o, v, i, j) - AT(o, v, i, j - 1)) * o->idy_v[j - 1];
            double d2vdx2 = iRe * v_cv_x_div(o, i, mu_xp * dvdxE, mu_xm * dvdxW);
            double d2vdy2 = iRe * (mu_yp * dvdyN - mu_ym * dvdyS) * o->idy_c[j - 1];
            double dudyE = (AT(o, u, i + 1, j) - AT(o, u, i + 1, j - 1)) * o->idy_c[j - 1];
            double dudyW = (AT(o, u, i, j) - AT(o, u, i, j - 1)) * o->idy_c[j - 1];
            double ddxdudy = iRe * v_cv_x_div(o, i, mu_xp * dudyE, mu_xm * dudyW);
            double ddydvdy = d2vdy2;
            double uCE = 0.5 * (AT(o, u, i + 1, j) + AT(o, u, i + 1, j - 1));
            double uCW = 0.5 * (AT(o, u, i, j) + AT(o, u, i, j - 1));
            double vuE = 0.5 * (AT(o, v, i, j) + AT(o, v, i + 1, j)) * uCE;
            double vuW = 0.5 * (AT(o, v, i, j) + AT(o, v, i - 1, j)) * uCW;
            double vvN = AT(o, vb, i, j) * AT(o, vb, i, j);
            double vvS = AT(o, vb, i, j - 1) * AT(o, vb, i, j - 1);
            double dvudx = v_cv_x_div(o, i, vuE, vuW);
            double dvvdy = (vvN - vvS) * o->idy_c[j - 1];
            AT(o, ex, i, j) = -(dvudx + dvvdy);
            AT(o, vx, i, j) = ddxdudy + ddydvdy;
            AT(o, im, i, j) = d2vdx2 + d2vdy2;
        }
}

/* Velocity_{u,v}_set_RHS (Velocity.c:1494-1728, :1739-1940), diffuse VOF,
 * no solids */
static void set_rhs(orc_t *o, char comp)
{
    int s = o->stage;
    double a_dt = 1.0 / (o->dt * BET[s]);
    double *pd = F(o, PVOF_F_P), *rho = F(o, PVOF_F_RHO);
    int isu = (comp == 'u');
    double *data = F(o, isu ? PVOF_F_U : PVOF_F_V);
    double *rhs = F(o, isu ? PVOF_F_U_RHS : PVOF_F_V_RHS);
    double *ex = F(o, isu ? PVOF_F_U_EXPLICIT : PVOF_F_V_EXPLICIT);
    double *exo = F(o, isu ? PVOF_F_U_EXPLICIT_OLD : PVOF_F_V_EXPLICIT_OLD);
    double *vx = F(o, isu ? PVOF_F_U_VISC_EXPLICIT : PVOF_F_V_VISC_EXPLICIT);
    double *vxo = F(o, isu ? PVOF_F_U_VISC_EXPLICIT_OLD : PVOF_F_V_VISC_EXPLICIT_OLD);
    double *im = F(o, isu ? PVOF_F_U_IMPLICIT : PVOF_F_V_IMPLICIT);
    double dp_dx_source = -o->p.dp_dx;
    int i0, i1, j0, j1;
    if (isu) u_range(o, &i0, &i1, &j0, &j1); else v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double dp, rf;
            if (isu) {
                dp = (AT(o, pd, i, j) - AT(o, pd, i - 1, j)) * o->idx_c[i - 1];
                rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i - 1, j));
            } else {
                dp = (AT(o, pd, i, j) - AT(o, pd, i, j - 1)) * o->idy_c[j - 1];
                rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i, j - 1));
            }
            double conv = GAMB[s] * AT(o, ex, i, j) + ZETB[s] * AT(o, exo, i, j);
            conv *= rf;
            double r = rf * a_dt * AT(o, data, i, j) + conv + AT(o, im, i, j) +
                       (GAMB[s] * AT(o, vx, i, j) + ZETB[s] * AT(o, vxo, i, j)) - 2.0 * dp;
            if (isu && o->g.periodic[0]) r += 2.0 * dp_dx_source;
            AT(o, rhs, i, j) = r;
            AT(o, exo, i, j) = AT(o, ex, i, j);
            AT(o, vxo, i, j) = AT(o, vx, i, j);
        }
}

/* vel_jacobi_diag (msolve_cg.c:98-249) and matVec (:255-493), diffuse VOF */
static double vel_diag(const orc_t *o, char comp, int i, int j, double alpha_k)
{
    const double *rho = F(o, PVOF_F_RHO), *mu = F(o, PVOF_F_MU);
    double iRe = 1.0 / o->p.Re;
    double dt = o->dt;
    if (comp == 'u') {
        double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i - 1, j));
        double d_time = rf / (alpha_k * dt);
        double mu_xp = AT(o, mu, i, j), mu_xm = AT(o, mu, i - 1, j);
        double mu_yp = harm(avg2(AT(o, mu, i - 1, j + 1), AT(o, mu, i, j + 1)), avg2(AT(o, mu, i - 1, j), AT(o, mu, i, j)));
        double mu_ym = harm(avg2(AT(o, mu, i - 1, j), AT(o, mu, i, j)), avg2(AT(o, mu, i - 1, j - 1), AT(o, mu, i, j - 1)));
        double dx = iRe * u_cv_x_diag(o, i, mu_xp * o->idx_u[i], mu_xm * o->idx_u[i - 1]);
        double dy = iRe * (mu_yp * o->idy_c[j] + mu_ym * o->idy_c[j - 1]) * o->idy_v[j];
        double da = axisym_ur_coeff(o, i, iRe * 0.5 * (mu_xp + mu_xm));
        return d_time + dx + dy + 0.0 + da;
    } else {
        double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i, j - 1));
        double d_time = rf / (alpha_k * dt);
        double mu_yp = AT(o, mu, i, j), mu_ym = AT(o, mu, i, j - 1);
        double mu_xp = harm(avg2(AT(o, mu, i + 1, j - 1), AT(o, mu, i + 1, j)), avg2(AT(o, mu, i, j - 1), AT(o, mu, i, j)));
        double mu_xm = harm(avg2(AT(o, mu, i, j - 1), AT(o, mu, i, j)), avg2(AT(o, mu, i - 1, j - 1), AT(o, mu, i - 1, j)));
        double dx = iRe * v_cv_x_diag(o, i, mu_xp * o->idx_c[i], mu_xm * o->idx_c[i - 1]);
        double dy = iRe * (mu_yp * o->idy_v[j] + mu_ym * o->idy_v[j - 1]) * o->idy_c[j - 1];
        return d_time + dx + dy + 0.0 + 0.0;
    }
}

static double vel_op(const orc_t *o, char comp, const double *x, int i, int j, double alpha_k)
{
    const double *rho = F(o, PVOF_F_RHO), *mu = F(o, PVOF_F_MU);
    double iRe = 1.0 / o->p.Re;
    double dt = o->dt;
    double op = 0.0;
    if (comp == 'u') {
        double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i - 1, j));
        double ft = rf / (alpha_k * dt);
        double Ax = ft * AT(o, x, i, j);
        double mu_xp = AT(o, mu, i, j), mu_xm = AT(o, mu, i - 1, j);
        double mu_yp = harm(avg2(AT(o, mu, i - 1, j + 1), AT(o, mu, i, j + 1)), avg2(AT(o, mu, i - 1, j), AT(o, mu, i, j)));
        double mu_ym = harm(avg2(AT(o, mu, i - 1, j), AT(o, mu, i, j)), avg2(AT(o, mu, i - 1, j - 1), AT(o, mu, i, j - 1)));
        double fxp = mu_xp * (AT(o, x, i + 1, j) - AT(o, x, i, j)) * o->idx_u[i];
        double fxm = mu_xm * (AT(o, x, i, j) - AT(o, x, i - 1, j)) * o->idx_u[i - 1];
        double fyp = mu_yp * (AT(o, x, i, j + 1) - AT(o, x, i, j)) * o->idy_c[j];
        double fym = mu_ym * (AT(o, x, i, j) - AT(o, x, i, j - 1)) * o->idy_c[j - 1];
        op += iRe * u_cv_x_div(o, i, fxp, fxm);
        op += iRe * (fyp - fym) * o->idy_v[j];
        op += axisym_ur_term(o, i, iRe * 0.5 * (mu_xp + mu_xm), AT(o, x, i, j));
        return Ax - op;
    } else {
        double rf = 0.5 * (AT(o, rho, i, j) + AT(o, rho, i, j - 1));
        double ft = rf / (alpha_k * dt);
        double Ax = ft * AT(o, x, i, j);
        double mu_yp = AT(o, mu, i, j), mu_ym = AT(o, mu, i, j - 1);
        double mu_xp = harm(avg2(AT(o, mu, i + 1, j - 1), AT(o, mu, i + 1, j)), avg2(AT(o, mu, i, j - 1), AT(o, mu, i, j)));
        double mu_xm = harm(avg2(AT(o, mu, i, j - 1), AT(o, mu, i, j)), avg2(AT(o, mu, i - 1, j - 1), AT(o, mu, i - 1, j)));
        double fxp = mu_xp * (AT(o, x, i + 1, j) - AT(o, x, i, j)) * o->idx_c[i];
        double fxm = mu_xm * (AT(o, x, i, j) - AT(o, x, i - 1, j)) * o->idx_c[i - 1];
        double fyp = mu_yp * (AT(o, x, i, j + 1) - AT(o, x, i, j)) * o->idy_v[j];
        double fym = mu_ym * (AT(o, x, i, j) - AT(o, x, i, j - 1)) * o->idy_v[j - 1];
        op += iRe * v_cv_x_div(o, i, fxp, fxm);
        op += iRe * (fyp - fym) * o->idy_c[j - 1];
        return Ax - op;
    }
}

/* Velocity_solve_cg (msolve_cg.c:525-722) */
static int velocity_solve_cg(orc_t *o, char comp, double *rms_out)
{
    int isu = (comp == 'u');
    double *data = F(o, isu ? PVOF_F_U : PVOF_F_V);
    double *rhs = F(o, isu ? PVOF_F_U_RHS : PVOF_F_V_RHS);
    double *r = S(o, isu ? S_U_R : S_V_R), *d = S(o, isu ? S_U_D : S_V_D), *Ad = S(o, isu ? S_U_AD : S_V_AD);
    const double EPS = 1e-14;
    double alpha_k = BET[o->stage];
    int NX = o->NX, NY = o->NY, NZ = o->NZ;
    int i0, i1, j0, j1;
    if (isu) u_range(o, &i0, &i1, &j0, &j1); else v_range(o, &i0, &i1, &j0, &j1);
    double in_tot;
    if (isu) in_tot = o->g.periodic[0] ? 1.0 / (double)((NX - 1) * (NY - 1) * (NZ - 1)) : 1.0 / (double)((NX - 2) * (NY - 1) * (NZ - 1));
    else in_tot = o->g.periodic[1] ? 1.0 / (double)((NX - 1) * (NY - 1) * (NZ - 1)) : 1.0 / (double)((NX - 1) * (NY - 2) * (NZ - 1));
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            AT(o, Ad, i, j) = vel_op(o, comp, data, i, j, alpha_k);
            AT(o, r, i, j) = AT(o, rhs, i, j) - AT(o, Ad, i, j);
            AT(o, d, i, j) = AT(o, r, i, j) / (vel_diag(o, comp, i, j, alpha_k) + EPS);
        }
    double rz = 0.0;
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) rz += AT(o, r, i, j) * AT(o, d, i, j);
    double RMS = 0.0;
    int iters = 0;
    while (iters < o->p.CG_MAXIT) {
        iters++;
        bc_velocity(o, d, comp, 1);
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) AT(o, Ad, i, j) = vel_op(o, comp, d, i, j, alpha_k);
        double dAd = 0.0;
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) dAd += AT(o, d, i, j) * AT(o, Ad, i, j);
        double alpha = rz / (dAd + EPS);
        double lv0 = 0.0, lv1 = 0.0;
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) {
                AT(o, data, i, j) += alpha * AT(o, d, i, j);
                AT(o, r, i, j) -= alpha * AT(o, Ad, i, j);
                double ri = AT(o, r, i, j);
                double dg = vel_diag(o, comp, i, j, alpha_k);
                lv0 += ri * ri / (dg + EPS);
                lv1 += ri * ri;
            }
        double rz_new = lv0, rr = lv1;
        RMS = sqrt(in_tot * rr);
        if (RMS < o->p.CG_ETOL) break;
        double beta = rz_new / (rz + EPS);
        rz = rz_new;
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++)
                AT(o, d, i, j) = AT(o, r, i, j) / (vel_diag(o, comp, i, j, alpha_k) + EPS) + beta * AT(o, d, i, j);
    }
    *rms_out = RMS;
    return iters;
}

/* Pressure_set_RHS (Pressure.c:100-196), GRID_UNIFORM */
static void pressure_set_rhs(orc_t *o)
{
    double a_dt = 1.0 / (o->dt * 2.0 * BET[o->stage]);
    double ihdt = o->idx_u[1] * a_dt;
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V), *rhs = F(o, PVOF_F_P_RHS);
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++)
            AT(o, rhs, i, j) = cell_center_divergence(o, u, v, i, j, ihdt, ihdt);
}

/* Pressure_compute_preconditioner (psolve_cg.c:63-101) */
static void pressure_preconditioner(orc_t *o)
{
    double *rho = F(o, PVOF_F_RHO), *M = S(o, S_P_MINV);
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) {
            double r0 = AT(o, rho, i, j);
            double bxp = 2.0 / (r0 + AT(o, rho, i + 1, j));
            double bxm = 2.0 / (r0 + AT(o, rho, i - 1, j));
            double byp = 2.0 / (r0 + AT(o, rho, i, j + 1));
            double bym = 2.0 / (r0 + AT(o, rho, i, j - 1));
            double cxm, cxp, cym, cyp;
            scalar_face_coeffs(o, i, bxm, bxp, bym, byp, &cxm, &cxp, &cym, &cyp);
            double aii = cxm + cxp + cym + cyp + 0.0 + 0.0;
            AT(o, M, i, j) = 1.0 / (row_weight(o, i) * aii + 1e-12);
        }
}

/* Pressure_operator_variableCoeff (psolve_cg.c:302-344) */
static void pressure_operator(orc_t *o, double *Aphi, double *phi)
{
    double *rho = F(o, PVOF_F_RHO);
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) {
            double r0 = AT(o, rho, i, j);
            double bxp = 2.0 / (r0 + AT(o, rho, i + 1, j));
            double bxm = 2.0 / (r0 + AT(o, rho, i - 1, j));
            double byp = 2.0 / (r0 + AT(o, rho, i, j + 1));
            double bym = 2.0 / (r0 + AT(o, rho, i, j - 1));
            double cxm, cxp, cym, cyp;
            scalar_face_coeffs(o, i, bxm, bxp, bym, byp, &cxm, &cxp, &cym, &cyp);
            double c = AT(o, phi, i, j);
            double val = cxp * (AT(o, phi, i + 1, j) - c) - cxm * (c - AT(o, phi, i - 1, j)) +
                         cyp * (AT(o, phi, i, j + 1) - c) - cym * (c - AT(o, phi, i, j - 1));
            AT(o, Aphi, i, j) = row_weight(o, i) * val;
        }
}

static double p_inner(orc_t *o, const double *a, const double *b)
{
    double s = 0.0;
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) s += AT(o, a, i, j) * AT(o, b, i, j);
    return s;
}

/* Pressure_solve_cg (psolve_cg.c:130-293) */
static int pressure_solve_cg(orc_t *o, double *res_out)
{
    double *phi = F(o, PVOF_F_DELTAP), *rhs = F(o, PVOF_F_P_RHS);
    double *res = S(o, S_P_RES), *d = S(o, S_P_D), *Ad = S(o, S_P_AD), *M = S(o, S_P_MINV), *z = S(o, S_P_Z);
    int NXp = o->NX - 1, NYp = o->NY - 1;
    double tol = o->p.P_CG_ETOL;
    int maxit = o->p.P_CG_MAXIT;
    zero_withghost(o, z);
    bc_pressure(o, phi);
    comm(o, phi, 'c');
    pressure_operator(o, Ad, phi);
    /* the right-hand side carries the operator's row weight r_c in the
     * axisymmetric mode, as the reference's HYPRE path forms it
     * (psolve_hypre.c:184-200); its in-tree CG leaves it out and then solves
     * r_c L phi = rhs, which is not the projection's system (the oracle build
     * of the reference adds the weight too, oracle/ref/shim/axisym_rhs.c) */
    for (int j = 0; j < NYp; j++)
        for (int i = 0; i < NXp; i++) {
            double b = o->axisym ? AT(o, rhs, i, j) * row_weight(o, i) : AT(o, rhs, i, j);
            AT(o, res, i, j) = b - AT(o, Ad, i, j);
        }
    for (int j = 0; j < NYp; j++)
        for (int i = 0; i < NXp; i++) {
            AT(o, z, i, j) = AT(o, res, i, j) * AT(o, M, i, j);
            AT(o, d, i, j) = AT(o, z, i, j);
        }
    double gamma = p_inner(o, res, z), gamma_new = 0.0;
    if (sqrt(gamma) < tol) {
        *res_out = sqrt(gamma);
        return 0;
    }
    int iters;
    for (iters = 1; iters <= maxit; iters++) {
        comm(o, d, 'c');
        bc_pressure(o, d);
        pressure_operator(o, Ad, d);
        double dAd = p_inner(o, d, Ad);
        double alpha = gamma / (dAd + 1e-30);
        for (int j = 0; j < NYp; j++)
            for (int i = 0; i < NXp; i++) {
                AT(o, phi, i, j) += alpha * AT(o, d, i, j);
                AT(o, res, i, j) -= alpha * AT(o, Ad, i, j);
            }
        for (int j = 0; j < NYp; j++)
            for (int i = 0; i < NXp; i++) AT(o, z, i, j) = AT(o, res, i, j) * AT(o, M, i, j);
        gamma_new = p_inner(o, res, z);
        if (sqrt(gamma_new) < tol) break;
        double beta = gamma_new / (gamma + 1e-30);
        for (int j = 0; j < NYp; j++)
            for (int i = 0; i < NXp; i++) AT(o, d, i, j) = AT(o, z, i, j) + beta * AT(o, d, i, j);
        gamma = gamma_new;
    }
    /* remove the mean (all faces Neumann or periodic), psolve_cg.c:255-279 */
    double sum = 0.0;
    long cnt = 0;
    for (int j = 0; j < NYp; j++)
        for (int i = 0; i < NXp; i++) { sum += AT(o, phi, i, j); ++cnt; }
    double avg = sum / (double)cnt;
    for (int j = 0; j < NYp; j++)
        for (int i = 0; i < NXp; i++) AT(o, phi, i, j) -= avg;
    comm(o, phi, 'c');
    if (iters > maxit) iters = maxit;
    *res_out = sqrt(gamma_new);
    return iters;
}

/* Pressure_project_velocity (Pressure.c:218-464) */
static void pressure_project(orc_t *o)
{
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V), *pd = F(o, PVOF_F_P), *dp = F(o, PVOF_F_DELTAP), *rho = F(o, PVOF_F_RHO);
    bc_pressure(o, dp);
    comm(o, dp, 'c');
    double mdt = 2.0 * BET[o->stage] * o->dt;
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) AT(o, pd, i, j) += AT(o, dp, i, j);
    bc_pressure(o, pd);
    comm(o, pd, 'c');
    int i0, i1, j0, j1;
    u_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double inv = 2.0 / (AT(o, rho, i, j) + AT(o, rho, i - 1, j));
            AT(o, u, i, j) -= (AT(o, dp, i, j) - AT(o, dp, i - 1, j)) * (o->idx_c[i - 1] * mdt * inv);
        }
    v_range(o, &i0, &i1, &j0, &j1);
    for (int j = j0; j < j1; j++)
        for (int i = i0; i < i1; i++) {
            double inv = 2.0 / (AT(o, rho, i, j) + AT(o, rho, i, j - 1));
            AT(o, v, i, j) -= (AT(o, dp, i, j) - AT(o, dp, i, j - 1)) * (o->idy_c[j - 1] * mdt * inv);
        }
}

/* Pressure_compute_velocity_divergence (Pressure.c:475-597) */
static double pressure_divergence(orc_t *o)
{
    double *u = F(o, PVOF_F_U), *v = F(o, PVOF_F_V);
    double mx = 0.0;
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) {
            double dc = fabs(cell_center_divergence(o, u, v, i, j, o->idx_u[i], o->idy_v[j]));
            if (dc >= mx) mx = dc;
        }
    return mx;
}

/* ------------------------------------------------------------------------ */
/* public API                                                               */
/* ------------------------------------------------------------------------ */

static int is_ng(int field)
{
    return (field >= PVOF_F_U_EXPLICIT && field <= PVOF_F_FSIG_NEW_Y) ||
           (field >= PVOF_F_W_EXPLICIT && field <= PVOF_F_FSIG_NEW_Z);
}

int orc_create(const pvof_grid_desc *grid, const pvof_params *params, orc_t **out)
{
    if (!grid || !params || !out) return PVOF_EINVAL;
    if (grid->ghost_nodes != NG) return PVOF_EINVAL;
    if (grid->geometry != PVOF_GEOM_PLANAR && grid->geometry != PVOF_GEOM_AXISYM) return PVOF_EINVAL;
    if (grid->NZM != 1) return PVOF_EINVAL;
    orc_t *o = (orc_t *)calloc(1, sizeof(orc_t));
    o->g = *grid;
    o->p = *params;
    o->NX = grid->NXM + 1;
    o->NY = grid->NYM + 1;
    o->NZ = grid->NZM + 1;
    o->nk = o->NZ;
    o->SX = o->NX + 2 * NG;
    o->SY = o->NY + 2 * NG;
    o->twod = 1;
    o->planar = (grid->geometry == PVOF_GEOM_PLANAR);
    o->axisym = (grid->geometry == PVOF_GEOM_AXISYM);
    o->slab = grid->slab_thickness;
    size_t n = (size_t)o->SX * (size_t)o->SY;
    for (int q = 0; q < PVOF_F_COUNT; q++) o->f[q] = (double *)calloc(n, sizeof(double));
    for (int q = 0; q < S_COUNT; q++) o->s[q] = (double *)calloc(n, sizeof(double));
    build_metrics(o);
    *out = o;
    return PVOF_OK;
}

void orc_destroy(orc_t *o)
{
    if (!o) return;
    for (int q = 0; q < PVOF_F_COUNT; q++) free(o->f[q]);
    for (int q = 0; q < S_COUNT; q++) free(o->s[q]);
    double *m[] = {o->xu, o->xc, o->dx_u, o->dx_c, o->idx_u, o->idx_c, o->i2dx_c, o->yv, o->yc, o->dy_v,
                   o->dy_c, o->idy_v, o->idy_c, o->i2dy_c, o->r_u, o->r_c, o->inv_r_u, o->inv_r_c, o->ring_wt_c};
    for (size_t q = 0; q < sizeof(m) / sizeof(m[0]); q++) metric_free(m[q]);
    free(o);
}

size_t orc_field_block_count(const orc_t *o, int field)
{
    if (field < 0 || field >= PVOF_F_COUNT) return 0;
    if (is_ng(field)) return (size_t)o->NX * (size_t)o->NY * (size_t)o->NZ;
    return (size_t)o->SX * (size_t)o->SY * (size_t)(o->NZ + 2 * NG);
}

int orc_set_field(orc_t *o, int field, const double *block, size_t count)
{
    if (count != orc_field_block_count(o, field)) return PVOF_EINVAL;
    double *a = o->f[field];
    if (is_ng(field)) {
        for (int j = 0; j < o->NY; j++)
            for (int i = 0; i < o->NX; i++) AT(o, a, i, j) = block[(size_t)j * o->NX + i];
    } else {
        size_t plane = (size_t)o->SX * (size_t)o->SY;
        memcpy(a, block + plane * NG, plane * sizeof(double)); /* k = 0 */
    }
    return PVOF_OK;
}

int orc_get_field(const orc_t *o, int field, double *block, size_t count)
{
    if (count != orc_field_block_count(o, field)) return PVOF_EINVAL;
    const double *a = o->f[field];
    if (is_ng(field)) {
        for (int k = 0; k < o->NZ; k++)
            for (int j = 0; j < o->NY; j++)
                for (int i = 0; i < o->NX; i++)
                    block[((size_t)k * o->NY + j) * o->NX + i] = (k == 0) ? AT(o, a, i, j) : 0.0;
    } else {
        size_t plane = (size_t)o->SX * (size_t)o->SY;
        memset(block, 0, count * sizeof(double));
        for (int k = 0; k < o->NZ; k++) memcpy(block + plane * (size_t)(NG + k), a, plane * sizeof(double));
    }
    return PVOF_OK;
}

int orc_set_stage(orc_t *o, int which_stage, double dt)
{
    if (which_stage < 0 || which_stage > 2 || !(dt > 0.0)) return PVOF_EINVAL;
    o->stage = which_stage;
    o->dt = dt;
    return PVOF_OK;
}

/* Start-up sequence after the fields are injected: boundary updates of the
 * injected velocity and pressure, the VOF part of
 * Cart3d_initialize_primitive_data (Cart3d.c:1096-1130) and the cell-centred
 * velocity of the first substep. */
static void initialize(orc_t *o)
{
    bc_velocity(o, F(o, PVOF_F_U), 'u', 0);
    bc_velocity(o, F(o, PVOF_F_V), 'v', 0);
    bc_pressure(o, F(o, PVOF_F_P));
    comm(o, F(o, PVOF_F_P), 'c');
    bc_scalar(o, F(o, PVOF_F_F));
    vof_diffuse_init(o);
    update_density_viscosity(o);
    if (o->p.surface_tension) {
        compute_psi_LG(o);
        compute_f_sigma(o);
        memcpy(F(o, PVOF_F_FSIG_OLD_X), F(o, PVOF_F_FSIG_NEW_X), sizeof(double) * (size_t)o->SX * o->SY);
        memcpy(F(o, PVOF_F_FSIG_OLD_Y), F(o, PVOF_F_FSIG_NEW_Y), sizeof(double) * (size_t)o->SX * o->SY);
    }
    cell_center(o);
    o->time = 0.0;
}

int orc_routine(orc_t *o, int routine, pvof_stats *st)
{
    double tmp;
    switch (routine) {
    case ORC_VOF_DIFFUSE_INIT: initialize(o); break;
    case ORC_VOF_DIFFUSE_STEP: vof_diffuse_step(o, st); break;
    case ORC_ADVECT_WENO5: advect_weno5(o, F(o, PVOF_F_CH_RHS_CUR)); break;
    case ORC_UPDATE_DENSITY_VISCOSITY: update_density_viscosity(o); break;
    case ORC_COMPUTE_PSI_LG: compute_psi_LG(o); break;
    case ORC_COMPUTE_F_SIGMA: compute_f_sigma(o); break;
    case ORC_APPLY_F_SIGMA_OLD: apply_f_sigma_old(o); break;
    case ORC_SWAP_F_SIGMA: swap_f_sigma(o); break;
    case ORC_ADD_GRAVITY: add_gravity(o); break;
    case ORC_CELL_CENTER: cell_center(o); break;
    case ORC_U_IMPLICIT_EXPLICIT: u_implicit_explicit(o); break;
    case ORC_V_IMPLICIT_EXPLICIT: v_implicit_explicit(o); break;
    case ORC_U_SET_RHS: set_rhs(o, 'u'); break;
    case ORC_V_SET_RHS: set_rhs(o, 'v'); break;
    case ORC_U_SOLVE_CG: {
        int it = velocity_solve_cg(o, 'u', &tmp);
        if (st) { st->u_iters = it; st->u_rms = tmp; }
        return it;
    }
    case ORC_V_SOLVE_CG: {
        int it = velocity_solve_cg(o, 'v', &tmp);
        if (st) { st->v_iters = it; st->v_rms = tmp; }
        return it;
    }
    case ORC_U_UPDATE_BOUNDARIES: bc_velocity(o, F(o, PVOF_F_U), 'u', 0); break;
    case ORC_V_UPDATE_BOUNDARIES: bc_velocity(o, F(o, PVOF_F_V), 'v', 0); break;
    case ORC_PRESSURE_SET_RHS:
        zero_withghost(o, F(o, PVOF_F_DELTAP));
        pressure_set_rhs(o);
        break;
    case ORC_PRESSURE_PRECONDITIONER: pressure_preconditioner(o); break;
    case ORC_PRESSURE_SOLVE_CG: {
        int it = pressure_solve_cg(o, &tmp);
        if (st) { st->p_iters = it; st->p_res = tmp; }
        return it;
    }
    case ORC_PRESSURE_PROJECT: pressure_project(o); break;
    case ORC_PRESSURE_DIVERGENCE: {
        double d = pressure_divergence(o);
        if (st) st->div_max = d;
        break;
    }
    default: return PVOF_EINVAL;
    }
    return PVOF_OK;
}

/* Temporal_int_all_the_equations (Temporal_int.c:563-1279), no solids */
int orc_substep(orc_t *o, pvof_stats *st)
{
    pvof_stats local;
    memset(&local, 0, sizeof(local));
    if (o->stage > 0) cell_center(o);
    comm(o, F(o, PVOF_F_U_BC), 'c');
    comm(o, F(o, PVOF_F_V_BC), 'c');
    vof_diffuse_step(o, &local);
    update_density_viscosity(o);
    u_implicit_explicit(o);
    v_implicit_explicit(o);
    set_rhs(o, 'u');
    set_rhs(o, 'v');
    if (o->p.surface_tension) {
        compute_psi_LG(o);
        compute_f_sigma(o);
        apply_f_sigma_old(o);
    }
    if (o->p.gravity) add_gravity(o);
    local.u_iters = velocity_solve_cg(o, 'u', &local.u_rms);
    local.v_iters = velocity_solve_cg(o, 'v', &local.v_rms);
    bc_velocity(o, F(o, PVOF_F_U), 'u', 0);
    bc_velocity(o, F(o, PVOF_F_V), 'v', 0);
    int passes = 0;
    double div;
    int rc = PVOF_OK;
    do {
        zero_withghost(o, F(o, PVOF_F_DELTAP));
        pressure_set_rhs(o);
        pressure_preconditioner(o);
        local.p_iters = pressure_solve_cg(o, &local.p_res);
        local.p_iters_total += local.p_iters;
        pressure_project(o);
        bc_velocity(o, F(o, PVOF_F_U), 'u', 0);
        bc_velocity(o, F(o, PVOF_F_V), 'v', 0);
        div = pressure_divergence(o);
        passes++;
        if (passes > 10) { rc = PVOF_EDIVERGED; break; }
    } while (div > 1e-6);
    local.poisson_passes = passes;
    local.div_max = div;
    if (o->p.surface_tension) swap_f_sigma(o);
    if (st) *st = local;
    return rc;
}

/* Temporal_int_rk3 (Temporal_int.c:399-448) at a constant dt */
int orc_run_steps(orc_t *o, int nsteps, double dt, pvof_stats *st)
{
    for (int n = 0; n < nsteps; n++) {
        for (int rk = 0; rk < 3; rk++) {
            if (o->time != 0 && rk == 0) cell_center(o);
            orc_set_stage(o, rk, dt);
            int rc = orc_substep(o, st);
            if (rc != PVOF_OK) return rc;
            o->time += dt * BET2[rk];
        }
    }
    return PVOF_OK;
}

/* liquid mass over the physical cells of one plane (no solids) */
double orc_liquid_mass(const orc_t *o)
{
    double s = 0.0;
    const double *CL = o->f[PVOF_F_C_L];
    for (int j = 0; j < o->NY - 1; j++)
        for (int i = 0; i < o->NX - 1; i++) s += AT(o, CL, i, j) * cell_measure(o, i, j);
    return s;
}
