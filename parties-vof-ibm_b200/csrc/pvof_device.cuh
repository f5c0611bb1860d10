// Device-side stencils of the two-phase substep.
//
// Every function evaluates the reference's arithmetic expression with the
// same operands in the same order (file:line given per function; paths are
// relative to PARTIES/src).  The library is compiled without FMA
// contraction, so these stencils round exactly like the reference's C.
#pragma once

#include "pvof_internal.cuh"

namespace pvof {

#define AT_(f, i, j) ((f)[(ptrdiff_t)(j) * P + (i)])

// Value of a field at (i,j) after the ghost update of kind `m`, read from the
// interior source the update would copy (identity away from the boundaries).
__device__ __forceinline__ double remap(const BcMap &m, const double *__restrict__ f, int P,
                                        int NX, int NY, int i, int j)
{
    if (i >= 1 && i <= NX - 2 && j >= 1 && j <= NY - 2)
        return AT_(f, i, j);
    int si = m.x.src[i + NG], sj = m.y.src[j + NG];
    double mx = m.x.mul[i + NG], my = m.y.mul[j + NG];
    if (mx == 0.0 || my == 0.0) return 0.0;
    double v = AT_(f, si, sj);
    return mx * my * v;
}

// TwodOps_scalar_laplacian (Eulerian/TwodOps.c:159-199)
template <class Get>
__device__ __forceinline__ double lap_at(const Dom &d, int i, int j, Get get)
{
    const Metrics &m = d.m;
    double c = get(i, j);
    double dfdxE = (get(i + 1, j) - c) * m.idx_c[i];
    double dfdxW = (c - get(i - 1, j)) * ((i != 0) ? m.idx_c[i - 1] : m.idx_c[i]);
    double dfdyN = (get(i, j + 1) - c) * m.idy_c[j];
    double dfdyS = (c - get(i, j - 1)) * ((j != 0) ? m.idy_c[j - 1] : m.idy_c[j]);
    if (d.planar)
        return (dfdxE - dfdxW) * m.idx_u[i] + (dfdyN - dfdyS) * m.idy_v[j];
    return (m.r_u[i + 1] * dfdxE - m.r_u[i] * dfdxW) * m.idx_u[i] * m.inv_r_c[i] + (dfdyN - dfdyS) * m.idy_v[j];
}

// The same Laplacian in single precision (the FP32 stencil form): the
// operands are rounded to float on load, the metrics too.
template <class Get>
__device__ __forceinline__ float lap_at_f(const Dom &d, int i, int j, Get get)
{
    const Metrics &m = d.m;
    const float c = (float)get(i, j);
    const float dfdxE = ((float)get(i + 1, j) - c) * (float)m.idx_c[i];
    const float dfdxW = (c - (float)get(i - 1, j)) * (float)((i != 0) ? m.idx_c[i - 1] : m.idx_c[i]);
    const float dfdyN = ((float)get(i, j + 1) - c) * (float)m.idy_c[j];
    const float dfdyS = (c - (float)get(i, j - 1)) * (float)((j != 0) ? m.idy_c[j - 1] : m.idy_c[j]);
    if (d.planar)
        return (dfdxE - dfdxW) * (float)m.idx_u[i] + (dfdyN - dfdyS) * (float)m.idy_v[j];
    return ((float)m.r_u[i + 1] * dfdxE - (float)m.r_u[i] * dfdxW) * (float)m.idx_u[i] * (float)m.inv_r_c[i] +
           (dfdyN - dfdyS) * (float)m.idy_v[j];
}

// diffuse_weno5_left in single precision (the FP32 stencil form)
__device__ __forceinline__ float weno5_left_f(float v0, float v1, float v2, float v3, float v4)
{
    const float eps = 1e-6f;
    const float q0 = (2.0f * v0 - 7.0f * v1 + 11.0f * v2) * (1.0f / 6.0f);
    const float q1 = (-v1 + 5.0f * v2 + 2.0f * v3) * (1.0f / 6.0f);
    const float q2 = (2.0f * v2 + 5.0f * v3 - v4) * (1.0f / 6.0f);
    const float t0 = v0 - 2.0f * v1 + v2, t1 = v0 - 4.0f * v1 + 3.0f * v2;
    const float b0 = (13.0f / 12.0f) * (t0 * t0) + 0.25f * (t1 * t1);
    const float t2 = v1 - 2.0f * v2 + v3, t3 = v1 - v3;
    const float b1 = (13.0f / 12.0f) * (t2 * t2) + 0.25f * (t3 * t3);
    const float t4 = v2 - 2.0f * v3 + v4, t5 = 3.0f * v2 - 4.0f * v3 + v4;
    const float b2 = (13.0f / 12.0f) * (t4 * t4) + 0.25f * (t5 * t5);
    const float a0 = 0.1f / ((eps + b0) * (eps + b0));
    const float a1 = 0.6f / ((eps + b1) * (eps + b1));
    const float a2 = 0.3f / ((eps + b2) * (eps + b2));
    return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

// diffuse_weno5_left (Eulerian/VOF_DIFFUSE.c:431-451); pow(x, 2.0) is x*x
__device__ __forceinline__ double weno5_left(double v0, double v1, double v2, double v3, double v4)
{
    const double eps = 1e-6;
    double q0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
    double q1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
    double q2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
    double t0 = v0 - 2.0 * v1 + v2, t1 = v0 - 4.0 * v1 + 3.0 * v2;
    double b0 = 13.0 / 12.0 * (t0 * t0) + 0.25 * (t1 * t1);
    double t2 = v1 - 2.0 * v2 + v3, t3 = v1 - v3;
    double b1 = 13.0 / 12.0 * (t2 * t2) + 0.25 * (t3 * t3);
    double t4 = v2 - 2.0 * v3 + v4, t5 = 3.0 * v2 - 4.0 * v3 + v4;
    double b2 = 13.0 / 12.0 * (t4 * t4) + 0.25 * (t5 * t5);
    double a0 = 0.1 / ((eps + b0) * (eps + b0));
    double a1 = 0.6 / ((eps + b1) * (eps + b1));
    double a2 = 0.3 / ((eps + b2) * (eps + b2));
    double asum = a0 + a1 + a2;
    return (a0 * q0 + a1 * q1 + a2 * q2) / asum;
}

// TwodOps_u_cv_x_flux_divergence and friends (Eulerian/TwodOps.c:231-309)
__device__ __forceinline__ double u_cv_x_div(const Dom &d, int i, double fe, double fw)
{
    if (!d.axisym) return (fe - fw) * d.m.idx_c[i - 1];
    return (d.m.r_c[i] * fe - d.m.r_c[i - 1] * fw) * d.m.idx_c[i - 1] * d.m.inv_r_u[i];
}
__device__ __forceinline__ double v_cv_x_div(const Dom &d, int i, double fe, double fw)
{
    if (!d.axisym) return (fe - fw) * d.m.idx_u[i];
    return (d.m.r_u[i + 1] * fe - d.m.r_u[i] * fw) * d.m.idx_u[i] * d.m.inv_r_c[i];
}
__device__ __forceinline__ double u_cv_x_diag(const Dom &d, int i, double ce, double cw)
{
    if (!d.axisym) return (ce + cw) * d.m.idx_c[i - 1];
    return (d.m.r_c[i] * ce + d.m.r_c[i - 1] * cw) * d.m.idx_c[i - 1] * d.m.inv_r_u[i];
}
__device__ __forceinline__ double v_cv_x_diag(const Dom &d, int i, double ce, double cw)
{
    if (!d.axisym) return (ce + cw) * d.m.idx_u[i];
    return (d.m.r_u[i + 1] * ce + d.m.r_u[i] * cw) * d.m.idx_u[i] * d.m.inv_r_c[i];
}
__device__ __forceinline__ double axisym_ur_term(const Dom &d, int i, double coeff, double u)
{
    if (!d.axisym) return 0.0;
    return -2.0 * coeff * u * d.m.inv_r_u[i] * d.m.inv_r_u[i];
}
__device__ __forceinline__ double axisym_ur_coeff(const Dom &d, int i, double coeff)
{
    if (!d.axisym) return 0.0;
    return 2.0 * coeff * d.m.inv_r_u[i] * d.m.inv_r_u[i];
}

__device__ __forceinline__ double harm(double a, double b) { return 2.0 * a * b / (a + b + 1e-12); }
__device__ __forceinline__ double avg2(double a, double b) { return 0.5 * (a + b); }

// TwodOps_cell_measure_c (Eulerian/TwodOps.c:311-333)
__device__ __forceinline__ double cell_measure(const Dom &d, int i, int j)
{
    if (d.planar) return d.m.dx_u[i] * d.m.dy_v[j] * d.slab;
    return d.m.dx_u[i] * d.m.dy_v[j] * d.m.ring_wt_c[i];
}

// TwodOps_cell_center_divergence (Eulerian/TwodOps.c:12-43)
__device__ __forceinline__ double cell_div(const Dom &d, const double *__restrict__ u, const double *__restrict__ v,
                                           int i, int j, double idx_u, double idy_v)
{
    const int P = d.P;
    double dudx = (AT_(u, i + 1, j) - AT_(u, i, j)) * idx_u;
    double dvdy = (AT_(v, i, j + 1) - AT_(v, i, j)) * idy_v;
    if (d.planar) return dudx + dvdy;
    return (d.m.r_u[i + 1] * AT_(u, i + 1, j) - d.m.r_u[i] * AT_(u, i, j)) * idx_u * d.m.inv_r_c[i] + dvdy;
}

// TwodOps_build_scalar_face_coeffs (Eulerian/TwodOps.c:45-88), no z terms
__device__ __forceinline__ void face_coeffs(const Dom &d, int i, double bxm, double bxp, double bym, double byp,
                                            double &cxm, double &cxp, double &cym, double &cyp)
{
    const double idx2 = d.m.idx_c[1] * d.m.idx_c[1];
    const double idy2 = d.m.idy_c[1] * d.m.idy_c[1];
    cxm = bxm * idx2;
    cxp = bxp * idx2;
    cym = bym * idy2;
    cyp = byp * idy2;
    if (d.planar) return;
    cxm = d.m.r_u[i] * bxm * d.m.inv_r_c[i] * idx2;
    cxp = d.m.r_u[i + 1] * bxp * d.m.inv_r_c[i] * idx2;
}

__device__ __forceinline__ double row_weight(const Dom &d, int i) { return d.axisym ? d.m.r_c[i] : 1.0; }

// Pressure_operator_variableCoeff (Eulerian/lsolver/psolve_cg.c:302-344) at (i,j)
template <class Get>
__device__ __forceinline__ double pressure_op(const Dom &d, const double *__restrict__ rho, int i, int j, Get get)
{
    const int P = d.P;
    double r0 = AT_(rho, i, j);
    double bxp = 2.0 / (r0 + AT_(rho, i + 1, j));
    double bxm = 2.0 / (r0 + AT_(rho, i - 1, j));
    double byp = 2.0 / (r0 + AT_(rho, i, j + 1));
    double bym = 2.0 / (r0 + AT_(rho, i, j - 1));
    double cxm, cxp, cym, cyp;
    face_coeffs(d, i, bxm, bxp, bym, byp, cxm, cxp, cym, cyp);
    double c = get(i, j);
    double val = cxp * (get(i + 1, j) - c) - cxm * (c - get(i - 1, j)) + cyp * (get(i, j + 1) - c) - cym * (c - get(i, j - 1));
    return row_weight(d, i) * val;
}

// The face weights 2 / (rho_P + rho_N) of pressure_op, one per east face
// (bx(i,j), between cells i and i+1) and one per north face (by(i,j)).  The
// west weight of cell i is the east weight of cell i-1: the same two
// densities added in the other order, the same sum exactly.
__device__ __forceinline__ void pressure_face_weights(const Dom &d, const double *__restrict__ rho, double *bx,
                                                      double *by, int i, int j)
{
    const int P = d.P;
    const double r0 = AT_(rho, i, j);
    AT_(bx, i, j) = 2.0 / (r0 + AT_(rho, i + 1, j));
    AT_(by, i, j) = 2.0 / (r0 + AT_(rho, i, j + 1));
    if (i == 0) AT_(bx, i - 1, j) = 2.0 / (r0 + AT_(rho, i - 1, j));
    if (j == 0) AT_(by, i, j - 1) = 2.0 / (r0 + AT_(rho, i, j - 1));
}

// pressure_op with the face weights read from pressure_face_weights' planes:
// bit for bit the same value, without the four divisions
template <class Get>
__device__ __forceinline__ double pressure_op_w(const Dom &d, const double *__restrict__ bx,
                                                const double *__restrict__ by, int i, int j, Get get)
{
    const int P = d.P;
    double cxm, cxp, cym, cyp;
    face_coeffs(d, i, AT_(bx, i - 1, j), AT_(bx, i, j), AT_(by, i, j - 1), AT_(by, i, j), cxm, cxp, cym, cyp);
    double c = get(i, j);
    double val = cxp * (get(i + 1, j) - c) - cxm * (c - get(i - 1, j)) + cyp * (get(i, j + 1) - c) - cym * (c - get(i, j - 1));
    return row_weight(d, i) * val;
}

// vel_jacobi_diag (Eulerian/lsolver/msolve_cg.c:98-249), diffuse VOF
__device__ __forceinline__ double vel_diag(const Dom &d, int comp, const double *__restrict__ rho,
                                           const double *__restrict__ mu, int i, int j, double iRe, double alpha_dt)
{
    const int P = d.P;
    if (comp == 0) {
        double rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j));
        double d_time = rf / alpha_dt;
        double mu_xp = AT_(mu, i, j), mu_xm = AT_(mu, i - 1, j);
        double mu_yp = harm(avg2(AT_(mu, i - 1, j + 1), AT_(mu, i, j + 1)), avg2(AT_(mu, i - 1, j), AT_(mu, i, j)));
        double mu_ym = harm(avg2(AT_(mu, i - 1, j), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i, j - 1)));
        double dx = iRe * u_cv_x_diag(d, i, mu_xp * d.m.idx_u[i], mu_xm * d.m.idx_u[i - 1]);
        double dy = iRe * (mu_yp * d.m.idy_c[j] + mu_ym * d.m.idy_c[j - 1]) * d.m.idy_v[j];
        double da = axisym_ur_coeff(d, i, iRe * 0.5 * (mu_xp + mu_xm));
        return d_time + dx + dy + 0.0 + da;
    } else {
        double rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
        double d_time = rf / alpha_dt;
        double mu_yp = AT_(mu, i, j), mu_ym = AT_(mu, i, j - 1);
        double mu_xp = harm(avg2(AT_(mu, i + 1, j - 1), AT_(mu, i + 1, j)), avg2(AT_(mu, i, j - 1), AT_(mu, i, j)));
        double mu_xm = harm(avg2(AT_(mu, i, j - 1), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i - 1, j)));
        double dx = iRe * v_cv_x_diag(d, i, mu_xp * d.m.idx_c[i], mu_xm * d.m.idx_c[i - 1]);
        double dy = iRe * (mu_yp * d.m.idy_v[j] + mu_ym * d.m.idy_v[j - 1]) * d.m.idy_c[j - 1];
        return d_time + dx + dy + 0.0 + 0.0;
    }
}

// The quotients of vel_op, stored once per solve: the time term
// ft = 0.5 (rho_P + rho_W|S) / (alpha dt) per cell and the harmonic mean of
// the viscosity at the cell's upper corner (u: north, v: east), mc.  The
// lower corner of a cell is the upper corner of the neighbour below (u) or
// to the west (v): the same expression with the same operands, so
// mc(i, j-1) (u) and mc(i-1, j) (v) are vel_op's mu_ym and mu_xm bit for bit.
// The cell at the start of the range also stores its lower corner.
__device__ __forceinline__ void vel_weights(const Dom &d, int comp, const double *__restrict__ rho,
                                            const double *__restrict__ mu, double *ft, double *mc, int i, int j,
                                            int i0, int j0, double alpha_dt)
{
    const int P = d.P;
    if (comp == 0) {
        AT_(ft, i, j) = 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j)) / alpha_dt;
        AT_(mc, i, j) = harm(avg2(AT_(mu, i - 1, j + 1), AT_(mu, i, j + 1)), avg2(AT_(mu, i - 1, j), AT_(mu, i, j)));
        if (j == j0)
            AT_(mc, i, j - 1) =
                harm(avg2(AT_(mu, i - 1, j), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i, j - 1)));
    } else {
        AT_(ft, i, j) = 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1)) / alpha_dt;
        AT_(mc, i, j) = harm(avg2(AT_(mu, i + 1, j - 1), AT_(mu, i + 1, j)), avg2(AT_(mu, i, j - 1), AT_(mu, i, j)));
        if (i == i0)
            AT_(mc, i - 1, j) =
                harm(avg2(AT_(mu, i, j - 1), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i - 1, j)));
    }
}

// vel_op with its quotients read from vel_weights' planes: the same value
// without the three divisions
template <class Get>
__device__ __forceinline__ double vel_op_w(const Dom &d, int comp, const double *__restrict__ ft,
                                           const double *__restrict__ mc, const double *__restrict__ mu, int i,
                                           int j, double iRe, Get x)
{
    const int P = d.P;
    double op = 0.0;
    double c = x(i, j);
    double Ax = AT_(ft, i, j) * c;
    if (comp == 0) {
        double mu_xp = AT_(mu, i, j), mu_xm = AT_(mu, i - 1, j);
        double mu_yp = AT_(mc, i, j), mu_ym = AT_(mc, i, j - 1);
        double fxp = mu_xp * (x(i + 1, j) - c) * d.m.idx_u[i];
        double fxm = mu_xm * (c - x(i - 1, j)) * d.m.idx_u[i - 1];
        double fyp = mu_yp * (x(i, j + 1) - c) * d.m.idy_c[j];
        double fym = mu_ym * (c - x(i, j - 1)) * d.m.idy_c[j - 1];
        op += iRe * u_cv_x_div(d, i, fxp, fxm);
        op += iRe * (fyp - fym) * d.m.idy_v[j];
        op += axisym_ur_term(d, i, iRe * 0.5 * (mu_xp + mu_xm), c);
        return Ax - op;
    } else {
        double mu_yp = AT_(mu, i, j), mu_ym = AT_(mu, i, j - 1);
        double mu_xp = AT_(mc, i, j), mu_xm = AT_(mc, i - 1, j);
        double fxp = mu_xp * (x(i + 1, j) - c) * d.m.idx_c[i];
        double fxm = mu_xm * (c - x(i - 1, j)) * d.m.idx_c[i - 1];
        double fyp = mu_yp * (x(i, j + 1) - c) * d.m.idy_v[j];
        double fym = mu_ym * (c - x(i, j - 1)) * d.m.idy_v[j - 1];
        op += iRe * v_cv_x_div(d, i, fxp, fxm);
        op += iRe * (fyp - fym) * d.m.idy_c[j - 1];
        return Ax - op;
    }
}

// matVec (Eulerian/lsolver/msolve_cg.c:255-493), diffuse VOF, at (i,j)
template <class Get>
__device__ __forceinline__ double vel_op(const Dom &d, int comp, const double *__restrict__ rho,
                                         const double *__restrict__ mu, int i, int j, double iRe, double alpha_dt,
                                         Get x)
{
    const int P = d.P;
    double op = 0.0;
    double c = x(i, j);
    if (comp == 0) {
        double rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j));
        double ft = rf / alpha_dt;
        double Ax = ft * c;
        double mu_xp = AT_(mu, i, j), mu_xm = AT_(mu, i - 1, j);
        double mu_yp = harm(avg2(AT_(mu, i - 1, j + 1), AT_(mu, i, j + 1)), avg2(AT_(mu, i - 1, j), AT_(mu, i, j)));
        double mu_ym = harm(avg2(AT_(mu, i - 1, j), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i, j - 1)));
        double fxp = mu_xp * (x(i + 1, j) - c) * d.m.idx_u[i];
        double fxm = mu_xm * (c - x(i - 1, j)) * d.m.idx_u[i - 1];
        double fyp = mu_yp * (x(i, j + 1) - c) * d.m.idy_c[j];
        double fym = mu_ym * (c - x(i, j - 1)) * d.m.idy_c[j - 1];
        op += iRe * u_cv_x_div(d, i, fxp, fxm);
        op += iRe * (fyp - fym) * d.m.idy_v[j];
        op += axisym_ur_term(d, i, iRe * 0.5 * (mu_xp + mu_xm), c);
        return Ax - op;
    } else {
        double rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
        double ft = rf / alpha_dt;
        double Ax = ft * c;
        double mu_yp = AT_(mu, i, j), mu_ym = AT_(mu, i, j - 1);
        double mu_xp = harm(avg2(AT_(mu, i + 1, j - 1), AT_(mu, i + 1, j)), avg2(AT_(mu, i, j - 1), AT_(mu, i, j)));
        double mu_xm = harm(avg2(AT_(mu, i, j - 1), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i - 1, j)));
        double fxp = mu_xp * (x(i + 1, j) - c) * d.m.idx_c[i];
        double fxm = mu_xm * (c - x(i - 1, j)) * d.m.idx_c[i - 1];
        double fyp = mu_yp * (x(i, j + 1) - c) * d.m.idy_v[j];
        double fym = mu_ym * (c - x(i, j - 1)) * d.m.idy_v[j - 1];
        op += iRe * v_cv_x_div(d, i, fxp, fxm);
        op += iRe * (fyp - fym) * d.m.idy_c[j - 1];
        return Ax - op;
    }
}

}  // namespace pvof
