// Three-dimensional mode of the two-phase substep (no TWOD_* flag in the
// reference): x and z periodic, walls in y, no solids.
//
// Layout: every field is one padded block of (NZ + 2G) planes of (NY + 2G)
// rows with a row pitch of P doubles; the pointer handed around addresses
// element (0,0,0), element (i,j,k) is at f[k*S + j*P + i] for the reference's
// ghosted index space i in [-3, NX+3), j in [-3, NY+3), k in [-3, NZ+3)
// (PARTIES/src/Memory.c:36-89), NX = NXM+1, NY = NYM+1, NZ = NZM+1.
//
// Ghost values are never stored by the routines: every read goes through the
// source map of the ghost update the reference applies to that field
// (Map3, built once on the host from Communication.c and the boundary
// routines), so a read at a ghost or half cell returns what the reference's
// array holds there.  Kernels write the physical cells (or the owned faces of
// a velocity component) only.  Density, viscosity, C_G and the cell-centred
// velocities are functions of C_L and u, v, w at the point read and are
// evaluated where they are needed instead of being stored.
//
// The routines are written once over an executor X that runs a functor over
// a box of cells (X::cells), a weighted sum over a box (X::reduce) and a
// single-thread scalar step over the finished sums (X::scalar); the library
// instantiates them with the CUDA executor of pvof_3d.cu.  Iterative solvers
// keep their scalars in device memory and gate every launch on a device
// flag, so the host reads back one word per chunk of iterations.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "../../include/pvof.h"

namespace pvof3 {

constexpr int NG = 3;
constexpr int OX = 8;   // column of i = 0 inside a padded row

// ghost-update kinds of the 3D mode
enum Kind {
    K_SCALAR = 0,   // VOF_DIFFUSE_set_boundary_values (VOF_DIFFUSE.c:571-683)
    K_PRESSURE,     // Pressure_apply_BCs + exchange (psolve_cg.c:358-529)
    K_U,            // Velocity_update_boundaries 'u' (Velocity.c:2427-2806), both types
    K_V,            // 'v', VEL_TYPE_NORMAL (walls set to zero)
    K_V_CG,         // 'v', VEL_TYPE_CG (walls left as they are)
    K_W,            // 'w', both types
    K_WRAP_C,       // exchange only, scalar class (Communication.c:128-1118)
    K_WRAP_U,       // exchange only, x-face class (U_VELOCITY, FLUX_X)
    K_WRAP_V,       // exchange only, y-face class (FLUX_Y: no y wrap on walls)
    K_WRAP_W,       // exchange only, z-face class (W_VELOCITY, FLUX_Z)
    K_COUNT
};

struct Axis {
    const int *src;     // [i + NG]
    const double *mul;  // [i + NG]; 1 copy, -1 negated copy, 0 zero
};
struct Map3 {
    Axis x, y, z;
};

struct Dom3 {
    int NX, NY, NZ;   // G-range extents
    int P;            // row pitch (doubles)
    long long S;      // plane pitch (doubles)
    // metrics, each offset so that m[i] is valid for i in [-NG, N+NG-1)
    const double *idx_u, *idx_c, *dx_u, *dx_c;
    const double *idy_v, *idy_c, *dy_v, *dy_c;
    const double *idz_w, *idz_c, *dz_w, *dz_c;
    // inner-product weight of a physical cell: its measure plus the measures
    // of the half cells that copy it; weight = wx[i] * wy[j] * wz[k]
    const double *wx, *wy, *wz;
    double idx2, idy2, idz2;   // idx_c[1]^2, ... (TwodOps.c:45-93)
    double idx_u1;             // idx_u[1] (Pressure_set_RHS on a uniform grid), for host code
    Map3 map[K_COUNT];
};

// RK3 coefficients (PARTIES/src/Include/definitions.h:197-204)
__host__ __device__ inline double bet(int s) { return s == 0 ? 4.0 / 15.0 : (s == 1 ? 1.0 / 15.0 : 1.0 / 6.0); }
__host__ __device__ inline double bet2(int s) { return s == 0 ? 8.0 / 15.0 : (s == 1 ? 2.0 / 15.0 : 1.0 / 3.0); }
__host__ __device__ inline double gamb(int s) { return s == 0 ? 2.0 : (s == 1 ? 25.0 / 4.0 : 9.0 / 2.0); }
__host__ __device__ inline double zetb(int s) { return s == 0 ? 0.0 : (s == 1 ? -17.0 / 4.0 : -2.5); }

__host__ __device__ __forceinline__ long long at(const Dom3 &d, int i, int j, int k)
{
    return (long long)k * d.S + (long long)j * d.P + i;
}

// value of field f at (i,j,k) after the ghost update of kind K
template <int K>
__host__ __device__ __forceinline__ double rd(const Dom3 &d, const double *__restrict__ f, int i, int j, int k)
{
    if (i >= 1 && i <= d.NX - 2 && j >= 1 && j <= d.NY - 2 && k >= 1 && k <= d.NZ - 2) return f[at(d, i, j, k)];
    const Map3 &m = d.map[K];
    const double mx = m.x.mul[i + NG], my = m.y.mul[j + NG], mz = m.z.mul[k + NG];
    if (mx == 0.0 || my == 0.0 || mz == 0.0) return 0.0;
    const double v = f[at(d, m.x.src[i + NG], m.y.src[j + NG], m.z.src[k + NG])];
    return mx * my * mz * v;
}

// the stored position that a pure-copy ghost update of kind K reads (i,j,k) from
template <int K>
__host__ __device__ __forceinline__ void src(const Dom3 &d, int &i, int &j, int &k)
{
    const Map3 &m = d.map[K];
    i = m.x.src[i + NG];
    j = m.y.src[j + NG];
    k = m.z.src[k + NG];
}

// true where the reference's array holds a value at (i,j,k) for a field that
// it computes on the G range and then updates with the ghost rule of kind K:
// inside the G range, or a position that the ghost update writes
template <int K>
__host__ __device__ __forceinline__ bool written(const Dom3 &d, int i, int j, int k)
{
    const Map3 &m = d.map[K];
    const bool wx = (i >= 0 && i < d.NX) || m.x.src[i + NG] != i || m.x.mul[i + NG] != 1.0;
    const bool wy = (j >= 0 && j < d.NY) || m.y.src[j + NG] != j || m.y.mul[j + NG] != 1.0;
    const bool wz = (k >= 0 && k < d.NZ) || m.z.src[k + NG] != k || m.z.mul[k + NG] != 1.0;
    return wx && wy && wz;
}

__host__ __device__ __forceinline__ double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

// derived phase quantities of the diffuse-interface model without solids
// (C_S = 0): VOF_DIFFUSE_update_phase_cache (VOF_DIFFUSE.c:108-126) and
// VOF_DIFFUSE_update_density_viscosity (:1453-1488)
struct Phase {
    double rho_g, mu_g;
    __host__ __device__ __forceinline__ double cg(double cl) const { return clamp01(1.0 - cl - 0.0); }
    __host__ __device__ __forceinline__ double rho(double cl) const { return cl + 1.0 * 0.0 + rho_g * cg(cl); }
    __host__ __device__ __forceinline__ double mu(double cl) const { return cl + 1.0 * 0.0 + mu_g * cg(cl); }
};

// TwodOps_scalar_laplacian, full 3D branch (Eulerian/TwodOps.c:159-199);
// get(i,j,k) returns the field after its ghost update
template <class Get>
__host__ __device__ __forceinline__ double lap3(const Dom3 &d, int i, int j, int k, Get get)
{
    const double c = get(i, j, k);
    const double dfdxE = (get(i + 1, j, k) - c) * d.idx_c[i];
    const double dfdxW = (c - get(i - 1, j, k)) * ((i != 0) ? d.idx_c[i - 1] : d.idx_c[i]);
    const double dfdyN = (get(i, j + 1, k) - c) * d.idy_c[j];
    const double dfdyS = (c - get(i, j - 1, k)) * ((j != 0) ? d.idy_c[j - 1] : d.idy_c[j]);
    const double dfdzF = (get(i, j, k + 1) - c) * d.idz_c[k];
    const double dfdzB = (c - get(i, j, k - 1)) * ((k != 0) ? d.idz_c[k - 1] : d.idz_c[k]);
    return (dfdxE - dfdxW) * d.idx_u[i] + (dfdyN - dfdyS) * d.idy_v[j] + (dfdzF - dfdzB) * d.idz_w[k];
}

// diffuse_weno5_left (Eulerian/VOF_DIFFUSE.c:431-451); pow(x, 2.0) is x*x
__host__ __device__ __forceinline__ double weno5(double v0, double v1, double v2, double v3, double v4)
{
    const double eps = 1e-6;
    const double q0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
    const double q1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
    const double q2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
    const double t0 = v0 - 2.0 * v1 + v2, t1 = v0 - 4.0 * v1 + 3.0 * v2;
    const double b0 = 13.0 / 12.0 * (t0 * t0) + 0.25 * (t1 * t1);
    const double t2 = v1 - 2.0 * v2 + v3, t3 = v1 - v3;
    const double b1 = 13.0 / 12.0 * (t2 * t2) + 0.25 * (t3 * t3);
    const double t4 = v2 - 2.0 * v3 + v4, t5 = 3.0 * v2 - 4.0 * v3 + v4;
    const double b2 = 13.0 / 12.0 * (t4 * t4) + 0.25 * (t5 * t5);
    const double a0 = 0.1 / ((eps + b0) * (eps + b0));
    const double a1 = 0.6 / ((eps + b1) * (eps + b1));
    const double a2 = 0.3 / ((eps + b2) * (eps + b2));
    const double asum = a0 + a1 + a2;
    return (a0 * q0 + a1 * q1 + a2 * q2) / asum;
}

// face state of C_L upwinded by the face velocity (diffuse_face_state_{x,y,z},
// VOF_DIFFUSE.c:455-498); (di,dj,dk) is the unit step of the face's axis
template <class Get>
__host__ __device__ __forceinline__ double face_state(int weno_order, double vel, int i, int j, int k, int di,
                                                      int dj, int dk, Get c)
{
    if (weno_order == 5) {
        if (vel >= 0.0)
            return weno5(c(i - 3 * di, j - 3 * dj, k - 3 * dk), c(i - 2 * di, j - 2 * dj, k - 2 * dk),
                         c(i - di, j - dj, k - dk), c(i, j, k), c(i + di, j + dj, k + dk));
        return weno5(c(i + 2 * di, j + 2 * dj, k + 2 * dk), c(i + di, j + dj, k + dk), c(i, j, k),
                     c(i - di, j - dj, k - dk), c(i - 2 * di, j - 2 * dj, k - 2 * dk));
    }
    return (vel >= 0.0) ? c(i - di, j - dj, k - dk) : c(i, j, k);
}

// single-precision forms of the stencils above (the FP32 stencil form):
// operands and metrics rounded to float on load, arithmetic in float
__host__ __device__ __forceinline__ float weno5f(float v0, float v1, float v2, float v3, float v4)
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
template <class Get>
__host__ __device__ __forceinline__ float face_state_f(int weno_order, float vel, int i, int j, int k, int di, int dj,
                                                       int dk, Get c)
{
    if (weno_order == 5) {
        if (vel >= 0.0f)
            return weno5f(c(i - 3 * di, j - 3 * dj, k - 3 * dk), c(i - 2 * di, j - 2 * dj, k - 2 * dk),
                          c(i - di, j - dj, k - dk), c(i, j, k), c(i + di, j + dj, k + dk));
        return weno5f(c(i + 2 * di, j + 2 * dj, k + 2 * dk), c(i + di, j + dj, k + dk), c(i, j, k),
                      c(i - di, j - dj, k - dk), c(i - 2 * di, j - 2 * dj, k - 2 * dk));
    }
    return (vel >= 0.0f) ? c(i - di, j - dj, k - dk) : c(i, j, k);
}
template <class Get>
__host__ __device__ __forceinline__ float lap3f(const Dom3 &d, int i, int j, int k, Get get)
{
    const float c = get(i, j, k);
    const float dfdxE = (get(i + 1, j, k) - c) * (float)d.idx_c[i];
    const float dfdxW = (c - get(i - 1, j, k)) * (float)((i != 0) ? d.idx_c[i - 1] : d.idx_c[i]);
    const float dfdyN = (get(i, j + 1, k) - c) * (float)d.idy_c[j];
    const float dfdyS = (c - get(i, j - 1, k)) * (float)((j != 0) ? d.idy_c[j - 1] : d.idy_c[j]);
    const float dfdzF = (get(i, j, k + 1) - c) * (float)d.idz_c[k];
    const float dfdzB = (c - get(i, j, k - 1)) * (float)((k != 0) ? d.idz_c[k - 1] : d.idz_c[k]);
    return (dfdxE - dfdxW) * (float)d.idx_u[i] + (dfdyN - dfdyS) * (float)d.idy_v[j] + (dfdzF - dfdzB) * (float)d.idz_w[k];
}

// HARMONIC(AVG2, AVG2) of msolve_cg.c:78-79; the same expression as the
// edge viscosities of Velocity.c (e.g. :446-470)
__host__ __device__ __forceinline__ double harm(double a, double b) { return 2.0 * a * b / (a + b + 1e-12); }
__host__ __device__ __forceinline__ double avg2(double a, double b) { return 0.5 * (a + b); }

// ---------------------------------------------------------------------------
// host-side tables
// ---------------------------------------------------------------------------

struct HostAxis {
    std::vector<double> c, f, dc, df, idc, idf;   // centres, faces, widths and inverses
    std::vector<double> w;                        // inner-product weights
    std::vector<int> src[K_COUNT];
    std::vector<double> mul[K_COUNT];
};

// Grid.c:797-862 and :372-420 for one uniform axis of N = NM + 1 G-range
// points: faces lo + i*h, centres lo + (i + 1/2) h, widths as differences
inline void host_axis_metrics(HostAxis &a, int N, double lo, double hi, bool periodic)
{
    const int n = N + 2 * NG;
    a.c.assign(n, 0.0); a.f.assign(n, 0.0); a.dc.assign(n, 0.0); a.df.assign(n, 0.0);
    a.idc.assign(n, 0.0); a.idf.assign(n, 0.0); a.w.assign(n, 0.0);
    const double h = (hi - lo) / (double)(N - 1);
    for (int i = -NG; i < N + NG; i++) {
        a.f[i + NG] = lo + i * h;
        a.c[i + NG] = lo + (0.5 + i) * h;
    }
    for (int i = -NG; i < N + NG - 1; i++) {
        a.df[i + NG] = a.f[i + 1 + NG] - a.f[i + NG];
        a.dc[i + NG] = a.c[i + 1 + NG] - a.c[i + NG];
        a.idf[i + NG] = 1.0 / a.df[i + NG];
        a.idc[i + NG] = 1.0 / a.dc[i + NG];
    }
    // the half cell N-1 copies cell 0 (periodic) or N-2 (wall)
    for (int i = 0; i < N; i++) {
        const int s = (i == N - 1) ? (periodic ? 0 : N - 2) : i;
        a.w[s + NG] += a.df[i + NG];
    }
}

// one axis of every ghost-update kind; wall_lo/hi are PVOF_WALL_* (walled axes)
inline void host_axis_maps(HostAxis &a, int N, bool periodic, bool face_x, bool face_y, bool face_z, int axis,
                           int wall_lo, int wall_hi)
{
    (void)face_x; (void)face_y; (void)face_z;
    for (int kind = 0; kind < K_COUNT; kind++) {
        std::vector<int> &s = a.src[kind];
        std::vector<double> &m = a.mul[kind];
        s.resize(N + 2 * NG);
        m.assign(N + 2 * NG, 1.0);
        for (int i = -NG; i < N + NG; i++) s[i + NG] = i;
        auto set = [&](int i, int from, double mm) { s[i + NG] = from; m[i + NG] = mm; };
        // the face-class component of this axis
        const bool face = (axis == 0 && (kind == K_U || kind == K_WRAP_U)) ||
                          (axis == 1 && (kind == K_V || kind == K_V_CG || kind == K_WRAP_V)) ||
                          (axis == 2 && (kind == K_W || kind == K_WRAP_W));
        if (periodic) {
            // Communication_update_ghost_nodes_{x,y,z}: the scalar class sends
            // [0, N-1), the face class [1, N] with the first face aliased
            if (face) {
                for (int i = -NG; i <= 0; i++) set(i, i + (N - 1), 1.0);
                for (int i = N; i <= N + NG - 1; i++) set(i, i - (N - 1), 1.0);
            } else {
                for (int i = -NG; i <= -1; i++) set(i, i + (N - 1), 1.0);
                for (int i = N - 1; i <= N + NG - 2; i++) set(i, i - (N - 1), 1.0);
            }
            continue;
        }
        switch (kind) {
        case K_SCALAR:   // VOF_DIFFUSE.c:591-663
            for (int g = 1; g <= NG; g++) set(-g, wall_lo == PVOF_WALL_FREESLIP ? g - 1 : 0, 1.0);
            for (int g = 0; g < NG; g++) set(N - 1 + g, wall_hi == PVOF_WALL_FREESLIP ? N - 2 - g : N - 2, 1.0);
            break;
        case K_PRESSURE:   // psolve_cg.c:374-460
            set(-1, 0, 1.0);
            set(N - 1, N - 2, 1.0);
            break;
        case K_U:
        case K_V:
        case K_V_CG:
        case K_W:   // Velocity.c:2480-2700 without lid velocities
            if (face) {
                if (kind != K_V_CG) {
                    set(0, 0, 0.0);
                    set(N - 1, N - 1, 0.0);
                }
            } else {
                set(-1, 0, wall_lo == PVOF_WALL_NOSLIP ? -1.0 : 1.0);
                set(N - 1, N - 2, wall_hi == PVOF_WALL_NOSLIP ? -1.0 : 1.0);
            }
            break;
        default:   // exchange-only kinds on a walled axis: nothing
            break;
        }
    }
}

// ---------------------------------------------------------------------------
// executor-independent pieces of the solvers
// ---------------------------------------------------------------------------

struct Range {
    int i0, i1, j0, j1, k0, k1;
};

template <int N>
struct Vec {
    double v[N];
};

constexpr int NSLOT = 4;   // reduction slots between two scalar steps

// device-resident scalars of the 3D solvers
struct Sc3 {
    double sum[NSLOT][4];   // finished sums of the reductions
    // biharmonic CG (diffuse_solve_biharmonic_pcg, VOF_DIFFUSE.c:339-429)
    double ch_rhs_norm, ch_rz, ch_alpha, ch_beta, ch_rel;
    int ch_iter, ch_maxit, ch_active;
    double ch_tol;
    // velocity PCG (Velocity_solve_cg, msolve_cg.c:525-722)
    double v_rz, v_alpha, v_beta, v_rms, v_eps, v_in_tot, v_tol;
    int v_iter, v_maxit, v_active;
    // pressure PCG (Pressure_solve_cg, psolve_cg.c:130-293)
    double p_gamma, p_gamma_new, p_alpha, p_beta, p_tol, p_avg;
    int p_iter, p_maxit, p_active, p_ran;
    unsigned p_count;   // blocks of the current reduction that have written their partial sum
    // results kept for the statistics
    int ch_iters_out, v_iters_out[3], p_iters_out;
    double ch_rel_out, v_rms_out[3], p_res_out;
    double div_max, clamp_delta, mass;
};

// field slots of the 3D state
enum F3 {
    F3_CL = 0, F3_F, F3_PSI, F3_RN, F3_CUR, F3_VEC, F3_AUX, F3_CHR, F3_CHP, F3_AP,
    F3_U, F3_V, F3_W, F3_P, F3_DP, F3_PRHS, F3_PR, F3_PD, F3_PAD, F3_PM,
    F3_U_EXO, F3_U_VXO, F3_U_RHS, F3_V_EXO, F3_V_VXO, F3_V_RHS, F3_W_EXO, F3_W_VXO, F3_W_RHS,
    F3_VR, F3_VD, F3_VAD, F3_VDIAG,
    F3_FSO_X, F3_FSO_Y, F3_FSO_Z, F3_FSN_X, F3_FSN_Y, F3_FSN_Z,
    F3_PCX, F3_PCY, F3_PCZ, F3_PZ,
    F3_COUNT
};

// the owned index boxes of the reference's loops (e.g. Velocity.c:395-410,
// :1170-1185; psolve_cg.c:76-82)
inline Range cells_range(const Dom3 &d) { return Range{0, d.NX - 1, 0, d.NY - 1, 0, d.NZ - 1}; }
inline Range face_range(const Dom3 &d, int comp)
{
    // x and z periodic, walls in y
    if (comp == 0) return Range{1, d.NX, 0, d.NY - 1, 0, d.NZ - 1};
    if (comp == 1) return Range{0, d.NX - 1, 1, d.NY - 1, 0, d.NZ - 1};
    return Range{0, d.NX - 1, 0, d.NY - 1, 1, d.NZ};
}

}  // namespace pvof3

namespace pvof3 {

// The reference's viscous and convective momentum terms of one face
// (Velocity_{u,v,w}_set_implicit_explicit, Velocity.c:366-1480, diffuse-VOF
// branches): ex = explicit (convection), vx = visc_explicit (cross terms),
// im = implicit (diagonal viscous terms).  The cell-centred velocities
// data_bc of Velocity_cell_center (Velocity.c:278-357) are evaluated from
// u, v, w at the point read.
struct MomTerms {
    double ex, vx, im;
};

template <int C>
__host__ __device__ __forceinline__ MomTerms mom_terms(const Dom3 &d, const Phase &ph, double iRe, const double *CL,
                                                       const double *U, const double *V, const double *W, int i, int j,
                                                       int k)
{
    auto mu = [&](int a, int b, int e) { return ph.mu(rd<K_SCALAR>(d, CL, a, b, e)); };
    auto u = [&](int a, int b, int e) { return rd<K_U>(d, U, a, b, e); };
    auto v = [&](int a, int b, int e) { return rd<K_V>(d, V, a, b, e); };
    auto w = [&](int a, int b, int e) { return rd<K_W>(d, W, a, b, e); };
    // data_bc after its scalar-class exchange
    auto ubc = [&](int a, int b, int e) { src<K_WRAP_C>(d, a, b, e); return 0.5 * (u(a, b, e) + u(a + 1, b, e)); };
    auto vbc = [&](int a, int b, int e) { src<K_WRAP_C>(d, a, b, e); return 0.5 * (v(a, b, e) + v(a, b + 1, e)); };
    auto wbc = [&](int a, int b, int e) { src<K_WRAP_C>(d, a, b, e); return 0.5 * (w(a, b, e) + w(a, b, e + 1)); };
    MomTerms t;
    if (C == 0) {
        const double muE = mu(i, j, k), muW = mu(i - 1, j, k);
        const double mu_yp = 2.0 * (0.5 * (mu(i - 1, j + 1, k) + mu(i, j + 1, k))) * (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) /
                             ((0.5 * (mu(i - 1, j + 1, k) + mu(i, j + 1, k))) + (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) + 1e-12);
        const double mu_ym = 2.0 * (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) * (0.5 * (mu(i - 1, j - 1, k) + mu(i, j - 1, k))) /
                             ((0.5 * (mu(i - 1, j, k) + mu(i, j, k))) + (0.5 * (mu(i - 1, j - 1, k) + mu(i, j - 1, k))) + 1e-12);
        const double mu_zp = 2.0 * (0.5 * (mu(i - 1, j, k + 1) + mu(i, j, k + 1))) * (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) /
                             ((0.5 * (mu(i - 1, j, k + 1) + mu(i, j, k + 1))) + (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) + 1e-12);
        const double mu_zm = 2.0 * (0.5 * (mu(i - 1, j, k) + mu(i, j, k))) * (0.5 * (mu(i - 1, j, k - 1) + mu(i, j, k - 1))) /
                             ((0.5 * (mu(i - 1, j, k) + mu(i, j, k))) + (0.5 * (mu(i - 1, j, k - 1) + mu(i, j, k - 1))) + 1e-12);
        const double uc = u(i, j, k);
        const double dudxE = (u(i + 1, j, k) - uc) * d.idx_u[i];
        const double dudxW = (uc - u(i - 1, j, k)) * d.idx_u[i - 1];
        const double dudyN = (u(i, j + 1, k) - uc) * d.idy_c[j];
        const double dudyS = (uc - u(i, j - 1, k)) * d.idy_c[j - 1];
        const double dudzF = (u(i, j, k + 1) - uc) * d.idz_c[k];
        const double dudzB = (uc - u(i, j, k - 1)) * d.idz_c[k - 1];
        const double d2udy2 = iRe * (mu_yp * dudyN - mu_ym * dudyS) * d.idy_v[j];
        const double d2udz2 = iRe * (mu_zp * dudzF - mu_zm * dudzB) * d.idz_w[k];
        const double dvdxN = (v(i, j + 1, k) - v(i - 1, j + 1, k)) * d.idx_c[i - 1];
        const double dvdxS = (v(i, j, k) - v(i - 1, j, k)) * d.idx_c[i - 1];
        const double dwdxF = (w(i, j, k + 1) - w(i - 1, j, k + 1)) * d.idx_c[i - 1];
        const double dwdxB = (w(i, j, k) - w(i - 1, j, k)) * d.idx_c[i - 1];
        const double d2udx2 = iRe * ((muE * dudxE - muW * dudxW) * d.idx_c[i - 1]);
        const double ddydvdx = iRe * (mu_yp * dvdxN - mu_ym * dvdxS) * d.idy_v[j];
        const double ddzdwdx = iRe * (mu_zp * dwdxF - mu_zm * dwdxB) * d.idz_w[k];
        const double vCN = 0.5 * (v(i, j + 1, k) + v(i - 1, j + 1, k));
        const double vCS = 0.5 * (v(i, j, k) + v(i - 1, j, k));
        const double wCF = 0.5 * (w(i, j, k + 1) + w(i - 1, j, k + 1));
        const double wCB = 0.5 * (w(i, j, k) + w(i - 1, j, k));
        const double ue = ubc(i, j, k), uw = ubc(i - 1, j, k);
        const double uuE = ue * ue, uuW = uw * uw;
        const double uvN = 0.5 * (uc + u(i, j + 1, k)) * vCN;
        const double uvS = 0.5 * (uc + u(i, j - 1, k)) * vCS;
        const double uwF = 0.5 * (uc + u(i, j, k + 1)) * wCF;
        const double uwB = 0.5 * (uc + u(i, j, k - 1)) * wCB;
        const double duudx = (uuE - uuW) * d.idx_c[i - 1];
        const double duvdy = (uvN - uvS) * d.idy_v[j];
        const double duwdz = (uwF - uwB) * d.idz_w[k];
        t.ex = -(duudx + duvdy + duwdz);
        t.vx = d2udx2 + ddydvdx + ddzdwdx;
        t.im = d2udx2 + d2udy2 + d2udz2 + 0.0;
    } else if (C == 1) {
        const double mu_xp = 2.0 * (0.5 * (mu(i + 1, j - 1, k) + mu(i + 1, j, k))) * (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) /
                             ((0.5 * (mu(i + 1, j - 1, k) + mu(i + 1, j, k))) + (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) + 1e-12);
        const double mu_xm = 2.0 * (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) * (0.5 * (mu(i - 1, j - 1, k) + mu(i - 1, j, k))) /
                             ((0.5 * (mu(i, j - 1, k) + mu(i, j, k))) + (0.5 * (mu(i - 1, j - 1, k) + mu(i - 1, j, k))) + 1e-12);
        const double mu_yp = mu(i, j, k), mu_ym = mu(i, j - 1, k);
        const double mu_zp = 2.0 * (0.5 * (mu(i, j - 1, k + 1) + mu(i, j, k + 1))) * (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) /
                             ((0.5 * (mu(i, j - 1, k + 1) + mu(i, j, k + 1))) + (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) + 1e-12);
        const double mu_zm = 2.0 * (0.5 * (mu(i, j - 1, k) + mu(i, j, k))) * (0.5 * (mu(i, j - 1, k - 1) + mu(i, j, k - 1))) /
                             ((0.5 * (mu(i, j - 1, k) + mu(i, j, k))) + (0.5 * (mu(i, j - 1, k - 1) + mu(i, j, k - 1))) + 1e-12);
        const double vc = v(i, j, k);
        const double dvdxE = (v(i + 1, j, k) - vc) * d.idx_c[i];
        const double dvdxW = (vc - v(i - 1, j, k)) * d.idx_c[i - 1];
        const double dvdyN = (v(i, j + 1, k) - vc) * d.idy_v[j];
        const double dvdyS = (vc - v(i, j - 1, k)) * d.idy_v[j - 1];
        const double dvdzF = (v(i, j, k + 1) - vc) * d.idz_c[k];
        const double dvdzB = (vc - v(i, j, k - 1)) * d.idz_c[k - 1];
        const double d2vdx2 = iRe * ((mu_xp * dvdxE - mu_xm * dvdxW) * d.idx_u[i]);
        const double d2vdy2 = iRe * (mu_yp * dvdyN - mu_ym * dvdyS) * d.idy_c[j - 1];
        const double d2vdz2 = iRe * (mu_zp * dvdzF - mu_zm * dvdzB) * d.idz_w[k];
        const double dudyE = (u(i + 1, j, k) - u(i + 1, j - 1, k)) * d.idy_c[j - 1];
        const double dudyW = (u(i, j, k) - u(i, j - 1, k)) * d.idy_c[j - 1];
        const double dwdyF = (w(i, j, k + 1) - w(i, j - 1, k + 1)) * d.idy_c[j - 1];
        const double dwdyB = (w(i, j, k) - w(i, j - 1, k)) * d.idy_c[j - 1];
        const double ddxdudy = iRe * ((mu_xp * dudyE - mu_xm * dudyW) * d.idx_u[i]);
        const double ddydvdy = d2vdy2;
        const double ddzdwdy = iRe * (mu_zp * dwdyF - mu_zm * dwdyB) * d.idz_w[k];
        const double uCE = 0.5 * (u(i + 1, j, k) + u(i + 1, j - 1, k));
        const double uCW = 0.5 * (u(i, j, k) + u(i, j - 1, k));
        const double wCF = 0.5 * (w(i, j, k + 1) + w(i, j - 1, k + 1));
        const double wCB = 0.5 * (w(i, j, k) + w(i, j - 1, k));
        const double vuE = 0.5 * (vc + v(i + 1, j, k)) * uCE;
        const double vuW = 0.5 * (vc + v(i - 1, j, k)) * uCW;
        const double vn = vbc(i, j, k), vs = vbc(i, j - 1, k);
        const double vvN = vn * vn, vvS = vs * vs;
        const double vwF = 0.5 * (vc + v(i, j, k + 1)) * wCF;
        const double vwB = 0.5 * (vc + v(i, j, k - 1)) * wCB;
        const double dvudx = (vuE - vuW) * d.idx_u[i];
        const double dvvdy = (vvN - vvS) * d.idy_c[j - 1];
        const double dvwdz = (vwF - vwB) * d.idz_w[k];
        t.ex = -(dvudx + dvvdy + dvwdz);
        t.vx = ddxdudy + ddydvdy + ddzdwdy;
        t.im = d2vdx2 + d2vdy2 + d2vdz2;
    } else {
        const double mu_xp = 2.0 * (0.5 * (mu(i + 1, j, k - 1) + mu(i + 1, j, k))) * (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) /
                             ((0.5 * (mu(i + 1, j, k - 1) + mu(i + 1, j, k))) + (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) + 1e-12);
        const double mu_xm = 2.0 * (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) * (0.5 * (mu(i - 1, j, k - 1) + mu(i - 1, j, k))) /
                             ((0.5 * (mu(i, j, k - 1) + mu(i, j, k))) + (0.5 * (mu(i - 1, j, k - 1) + mu(i - 1, j, k))) + 1e-12);
        const double mu_yp = 2.0 * (0.5 * (mu(i, j + 1, k - 1) + mu(i, j + 1, k))) * (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) /
                             ((0.5 * (mu(i, j + 1, k - 1) + mu(i, j + 1, k))) + (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) + 1e-12);
        const double mu_ym = 2.0 * (0.5 * (mu(i, j, k - 1) + mu(i, j, k))) * (0.5 * (mu(i, j - 1, k - 1) + mu(i, j - 1, k))) /
                             ((0.5 * (mu(i, j, k - 1) + mu(i, j, k))) + (0.5 * (mu(i, j - 1, k - 1) + mu(i, j - 1, k))) + 1e-12);
        const double mu_zp = mu(i, j, k), mu_zm = mu(i, j, k - 1);
        const double wc = w(i, j, k);
        const double dwdxE = (w(i + 1, j, k) - wc) * d.idx_c[i];
        const double dwdxW = (wc - w(i - 1, j, k)) * d.idx_c[i - 1];
        const double dwdyN = (w(i, j + 1, k) - wc) * d.idy_c[j];
        const double dwdyS = (wc - w(i, j - 1, k)) * d.idy_c[j - 1];
        const double dwdzF = (w(i, j, k + 1) - wc) * d.idz_w[k];
        const double dwdzB = (wc - w(i, j, k - 1)) * d.idz_w[k - 1];
        const double d2wdx2 = iRe * (mu_xp * dwdxE - mu_xm * dwdxW) * d.idx_u[i];
        const double d2wdy2 = iRe * (mu_yp * dwdyN - mu_ym * dwdyS) * d.idy_v[j];
        const double d2wdz2 = iRe * (mu_zp * dwdzF - mu_zm * dwdzB) * d.idz_c[k - 1];
        const double dudzE = (u(i + 1, j, k) - u(i + 1, j, k - 1)) * d.idz_c[k - 1];
        const double dudzW = (u(i, j, k) - u(i, j, k - 1)) * d.idz_c[k - 1];
        const double dvdzN = (v(i, j + 1, k) - v(i, j + 1, k - 1)) * d.idz_c[k - 1];
        const double dvdzS = (v(i, j, k) - v(i, j, k - 1)) * d.idz_c[k - 1];
        const double ddxdudz = iRe * (mu_xp * dudzE - mu_xm * dudzW) * d.idx_u[i];
        const double ddydvdz = iRe * (mu_yp * dvdzN - mu_ym * dvdzS) * d.idy_v[j];
        const double ddzdwdz = d2wdz2;
        const double uCE = 0.5 * (u(i + 1, j, k) + u(i + 1, j, k - 1));
        const double uCW = 0.5 * (u(i, j, k) + u(i, j, k - 1));
        const double vCN = 0.5 * (v(i, j + 1, k) + v(i, j + 1, k - 1));
        const double vCS = 0.5 * (v(i, j, k) + v(i, j, k - 1));
        const double wuE = 0.5 * (wc + w(i + 1, j, k)) * uCE;
        const double wuW = 0.5 * (wc + w(i - 1, j, k)) * uCW;
        const double wvN = 0.5 * (wc + w(i, j + 1, k)) * vCN;
        const double wvS = 0.5 * (wc + w(i, j - 1, k)) * vCS;
        const double wf = wbc(i, j, k), wb = wbc(i, j, k - 1);
        const double wwF = wf * wf, wwB = wb * wb;
        const double dwudx = (wuE - wuW) * d.idx_u[i];
        const double dwvdy = (wvN - wvS) * d.idy_v[j];
        const double dwwdz = (wwF - wwB) * d.idz_c[k - 1];
        t.ex = -(dwudx + dwvdy + dwwdz);
        t.vx = ddxdudz + ddydvdz + ddzdwdz;
        t.im = d2wdx2 + d2wdy2 + d2wdz2;
    }
    return t;
}

// vel_jacobi_diag and one row of matVec (msolve_cg.c:103-493, VOF branch)
// of component C at (i,j,k); x is read through the ghost update KX
template <int C>
__host__ __device__ __forceinline__ double vel_diag(const Dom3 &d, const Phase &ph, double iRe, double alpha_k,
                                                    double dt, const double *CL, int i, int j, int k)
{
    auto mu = [&](int a, int b, int e) { return ph.mu(rd<K_SCALAR>(d, CL, a, b, e)); };
    auto rho = [&](int a, int b, int e) { return ph.rho(rd<K_SCALAR>(d, CL, a, b, e)); };
    const double rho_face = 0.5 * (rho(i, j, k) + rho(C == 0 ? i - 1 : i, C == 1 ? j - 1 : j, C == 2 ? k - 1 : k));
    const double d_time = rho_face / (alpha_k * dt);
    double dx, dy, dz, dax = 0.0;
    if (C == 0) {
        const double mu_xp = mu(i, j, k), mu_xm = mu(i - 1, j, k);
        const double mu_yp = harm(avg2(mu(i - 1, j + 1, k), mu(i, j + 1, k)), avg2(mu(i - 1, j, k), mu(i, j, k)));
        const double mu_ym = harm(avg2(mu(i - 1, j, k), mu(i, j, k)), avg2(mu(i - 1, j - 1, k), mu(i, j - 1, k)));
        const double mu_zp = harm(avg2(mu(i - 1, j, k + 1), mu(i, j, k + 1)), avg2(mu(i - 1, j, k), mu(i, j, k)));
        const double mu_zm = harm(avg2(mu(i - 1, j, k), mu(i, j, k)), avg2(mu(i - 1, j, k - 1), mu(i, j, k - 1)));
        dx = iRe * ((mu_xp * d.idx_u[i] + mu_xm * d.idx_u[i - 1]) * d.idx_c[i - 1]);
        dy = iRe * (mu_yp * d.idy_c[j] + mu_ym * d.idy_c[j - 1]) * d.idy_v[j];
        dz = iRe * (mu_zp * d.idz_c[k] + mu_zm * d.idz_c[k - 1]) * d.idz_w[k];
    } else if (C == 1) {
        const double mu_yp = mu(i, j, k), mu_ym = mu(i, j - 1, k);
        const double mu_xp = harm(avg2(mu(i + 1, j - 1, k), mu(i + 1, j, k)), avg2(mu(i, j - 1, k), mu(i, j, k)));
        const double mu_xm = harm(avg2(mu(i, j - 1, k), mu(i, j, k)), avg2(mu(i - 1, j - 1, k), mu(i - 1, j, k)));
        const double mu_zp = harm(avg2(mu(i, j - 1, k + 1), mu(i, j, k + 1)), avg2(mu(i, j - 1, k), mu(i, j, k)));
        const double mu_zm = harm(avg2(mu(i, j - 1, k), mu(i, j, k)), avg2(mu(i, j - 1, k - 1), mu(i, j, k - 1)));
        dx = iRe * ((mu_xp * d.idx_c[i] + mu_xm * d.idx_c[i - 1]) * d.idx_u[i]);
        dy = iRe * (mu_yp * d.idy_v[j] + mu_ym * d.idy_v[j - 1]) * d.idy_c[j - 1];
        dz = iRe * (mu_zp * d.idz_c[k] + mu_zm * d.idz_c[k - 1]) * d.idz_w[k];
    } else {
        const double mu_zp = mu(i, j, k), mu_zm = mu(i, j, k - 1);
        const double mu_xp = harm(avg2(mu(i + 1, j, k - 1), mu(i + 1, j, k)), avg2(mu(i, j, k - 1), mu(i, j, k)));
        const double mu_xm = harm(avg2(mu(i, j, k - 1), mu(i, j, k)), avg2(mu(i - 1, j, k - 1), mu(i - 1, j, k)));
        const double mu_yp = harm(avg2(mu(i, j + 1, k - 1), mu(i, j + 1, k)), avg2(mu(i, j, k - 1), mu(i, j, k)));
        const double mu_ym = harm(avg2(mu(i, j, k - 1), mu(i, j, k)), avg2(mu(i, j - 1, k - 1), mu(i, j - 1, k)));
        dx = iRe * (mu_xp * d.idx_c[i] + mu_xm * d.idx_c[i - 1]) * d.idx_u[i];
        dy = iRe * (mu_yp * d.idy_c[j] + mu_ym * d.idy_c[j - 1]) * d.idy_v[j];
        dz = iRe * (mu_zp * d.idz_w[k] + mu_zm * d.idz_w[k - 1]) * d.idz_c[k - 1];
    }
    return d_time + dx + dy + dz + dax;
}

template <int C, int KX>
__host__ __device__ __forceinline__ double vel_op(const Dom3 &d, const Phase &ph, double iRe, double alpha_k, double dt,
                                                  const double *CL, const double *X, int i, int j, int k)
{
    auto mu = [&](int a, int b, int e) { return ph.mu(rd<K_SCALAR>(d, CL, a, b, e)); };
    auto rho = [&](int a, int b, int e) { return ph.rho(rd<K_SCALAR>(d, CL, a, b, e)); };
    auto x = [&](int a, int b, int e) { return rd<KX>(d, X, a, b, e); };
    const double rho_face = 0.5 * (rho(i, j, k) + rho(C == 0 ? i - 1 : i, C == 1 ? j - 1 : j, C == 2 ? k - 1 : k));
    const double factor_time = rho_face / (alpha_k * dt);
    const double xc = x(i, j, k);
    const double Ax = factor_time * xc;
    double op = 0.0;
    if (C == 0) {
        const double mu_xp = mu(i, j, k), mu_xm = mu(i - 1, j, k);
        const double mu_yp = harm(avg2(mu(i - 1, j + 1, k), mu(i, j + 1, k)), avg2(mu(i - 1, j, k), mu(i, j, k)));
        const double mu_ym = harm(avg2(mu(i - 1, j, k), mu(i, j, k)), avg2(mu(i - 1, j - 1, k), mu(i, j - 1, k)));
        const double mu_zp = harm(avg2(mu(i - 1, j, k + 1), mu(i, j, k + 1)), avg2(mu(i - 1, j, k), mu(i, j, k)));
        const double mu_zm = harm(avg2(mu(i - 1, j, k), mu(i, j, k)), avg2(mu(i - 1, j, k - 1), mu(i, j, k - 1)));
        const double fxp = mu_xp * (x(i + 1, j, k) - xc) * d.idx_u[i];
        const double fxm = mu_xm * (xc - x(i - 1, j, k)) * d.idx_u[i - 1];
        const double fyp = mu_yp * (x(i, j + 1, k) - xc) * d.idy_c[j];
        const double fym = mu_ym * (xc - x(i, j - 1, k)) * d.idy_c[j - 1];
        op += iRe * ((fxp - fxm) * d.idx_c[i - 1]);
        op += iRe * (fyp - fym) * d.idy_v[j];
        const double fzp = mu_zp * (x(i, j, k + 1) - xc) * d.idz_c[k];
        const double fzm = mu_zm * (xc - x(i, j, k - 1)) * d.idz_c[k - 1];
        op += iRe * (fzp - fzm) * d.idz_w[k];
        op += 0.0;
    } else if (C == 1) {
        const double mu_yp = mu(i, j, k), mu_ym = mu(i, j - 1, k);
        const double mu_xp = harm(avg2(mu(i + 1, j - 1, k), mu(i + 1, j, k)), avg2(mu(i, j - 1, k), mu(i, j, k)));
        const double mu_xm = harm(avg2(mu(i, j - 1, k), mu(i, j, k)), avg2(mu(i - 1, j - 1, k), mu(i - 1, j, k)));
        const double mu_zp = harm(avg2(mu(i, j - 1, k + 1), mu(i, j, k + 1)), avg2(mu(i, j - 1, k), mu(i, j, k)));
        const double mu_zm = harm(avg2(mu(i, j - 1, k), mu(i, j, k)), avg2(mu(i, j - 1, k - 1), mu(i, j, k - 1)));
        const double fxp = mu_xp * (x(i + 1, j, k) - xc) * d.idx_c[i];
        const double fxm = mu_xm * (xc - x(i - 1, j, k)) * d.idx_c[i - 1];
        const double fyp = mu_yp * (x(i, j + 1, k) - xc) * d.idy_v[j];
        const double fym = mu_ym * (xc - x(i, j - 1, k)) * d.idy_v[j - 1];
        op += iRe * ((fxp - fxm) * d.idx_u[i]);
        op += iRe * (fyp - fym) * d.idy_c[j - 1];
        const double fzp = mu_zp * (x(i, j, k + 1) - xc) * d.idz_c[k];
        const double fzm = mu_zm * (xc - x(i, j, k - 1)) * d.idz_c[k - 1];
        op += iRe * (fzp - fzm) * d.idz_w[k];
    } else {
        const double mu_zp = mu(i, j, k), mu_zm = mu(i, j, k - 1);
        const double mu_xp = harm(avg2(mu(i + 1, j, k - 1), mu(i + 1, j, k)), avg2(mu(i, j, k - 1), mu(i, j, k)));
        const double mu_xm = harm(avg2(mu(i, j, k - 1), mu(i, j, k)), avg2(mu(i - 1, j, k - 1), mu(i - 1, j, k)));
        const double mu_yp = harm(avg2(mu(i, j + 1, k - 1), mu(i, j + 1, k)), avg2(mu(i, j, k - 1), mu(i, j, k)));
        const double mu_ym = harm(avg2(mu(i, j, k - 1), mu(i, j, k)), avg2(mu(i, j - 1, k - 1), mu(i, j - 1, k)));
        const double fxp = mu_xp * (x(i + 1, j, k) - xc) * d.idx_c[i];
        const double fxm = mu_xm * (xc - x(i - 1, j, k)) * d.idx_c[i - 1];
        const double fyp = mu_yp * (x(i, j + 1, k) - xc) * d.idy_c[j];
        const double fym = mu_ym * (xc - x(i, j - 1, k)) * d.idy_c[j - 1];
        op += iRe * (fxp - fxm) * d.idx_u[i];
        op += iRe * (fyp - fym) * d.idy_v[j];
        const double fzp = mu_zp * (x(i, j, k + 1) - xc) * d.idz_w[k];
        const double fzm = mu_zm * (xc - x(i, j, k - 1)) * d.idz_w[k - 1];
        op += iRe * (fzp - fzm) * d.idz_c[k - 1];
    }
    return Ax - op;
}

// Pressure_operator_variableCoeff / Pressure_compute_preconditioner
// (psolve_cg.c:63-101, :302-344) with TwodOps_build_scalar_face_coeffs
// (TwodOps.c:45-93); rho from C_L through its scalar ghost update
struct PFaces {
    double cxm, cxp, cym, cyp, czm, czp;
};
__host__ __device__ __forceinline__ PFaces p_faces(const Dom3 &d, const Phase &ph, const double *CL, int i, int j, int k)
{
    auto rho = [&](int a, int b, int e) { return ph.rho(rd<K_SCALAR>(d, CL, a, b, e)); };
    const double r0 = rho(i, j, k);
    const double bxp = 2.0 / (r0 + rho(i + 1, j, k));
    const double bxm = 2.0 / (r0 + rho(i - 1, j, k));
    const double byp = 2.0 / (r0 + rho(i, j + 1, k));
    const double bym = 2.0 / (r0 + rho(i, j - 1, k));
    const double bzp = 2.0 / (r0 + rho(i, j, k + 1));
    const double bzm = 2.0 / (r0 + rho(i, j, k - 1));
    PFaces c;
    c.cxm = bxm * d.idx2; c.cxp = bxp * d.idx2;
    c.cym = bym * d.idy2; c.cyp = byp * d.idy2;
    c.czm = bzm * d.idz2; c.czp = bzp * d.idz2;
    return c;
}
__host__ __device__ __forceinline__ double p_apply(const Dom3 &d, const PFaces &c, const double *X, int i, int j, int k)
{
    auto x = [&](int a, int b, int e) { return rd<K_PRESSURE>(d, X, a, b, e); };
    const double xc = x(i, j, k);
    const double val = c.cxp * (x(i + 1, j, k) - xc) - c.cxm * (xc - x(i - 1, j, k)) + c.cyp * (x(i, j + 1, k) - xc) -
                       c.cym * (xc - x(i, j - 1, k)) + c.czp * (x(i, j, k + 1) - xc) - c.czm * (xc - x(i, j, k - 1));
    return 1.0 * val;
}

// the same operator with the face coefficients of one solve stored: CX at
// (i,j,k) is cxp of that cell and cxm of cell i+1 (2/(rho_i + rho_i+1) is the
// same number seen from either side); CX, CY, CZ hold one layer below the
// physical cells too
__host__ __device__ __forceinline__ double p_apply_st(const Dom3 &d, const double *CX, const double *CY,
                                                      const double *CZ, const double *X, int i, int j, int k)
{
    auto x = [&](int a, int b, int e) { return rd<K_PRESSURE>(d, X, a, b, e); };
    const long long q = at(d, i, j, k);
    const double xc = x(i, j, k);
    const double val = CX[q] * (x(i + 1, j, k) - xc) - CX[q - 1] * (xc - x(i - 1, j, k)) + CY[q] * (x(i, j + 1, k) - xc) -
                       CY[q - d.P] * (xc - x(i, j - 1, k)) + CZ[q] * (x(i, j, k + 1) - xc) - CZ[q - d.S] * (xc - x(i, j, k - 1));
    return 1.0 * val;
}

// TwodOps_cell_center_divergence, 3D branch (TwodOps.c:12-43)
__host__ __device__ __forceinline__ double cc_div(const Dom3 &d, const double *U, const double *V, const double *W, int i,
                                                  int j, int k, double ix, double iy, double iz)
{
    const double dudx = (rd<K_U>(d, U, i + 1, j, k) - rd<K_U>(d, U, i, j, k)) * ix;
    const double dvdy = (rd<K_V>(d, V, i, j + 1, k) - rd<K_V>(d, V, i, j, k)) * iy;
    const double dwdz = (rd<K_W>(d, W, i, j, k + 1) - rd<K_W>(d, W, i, j, k)) * iz;
    return dudx + dvdy + dwdz;
}

// VOF_DIFFUSE_compute_f_sigma of one face of component C (VOF_DIFFUSE.c:1364-1445)
template <int C>
__host__ __device__ __forceinline__ double f_sigma(const Dom3 &d, const Phase &ph, double scale, const double *CL,
                                                   const double *PSI, int i, int j, int k)
{
    const int a = C == 0 ? i - 1 : i, b = C == 1 ? j - 1 : j, e = C == 2 ? k - 1 : k;
    const double c0 = rd<K_SCALAR>(d, CL, i, j, k), c1 = rd<K_SCALAR>(d, CL, a, b, e);
    const double cl = 0.5 * (c0 + c1);
    const double cg = 0.5 * (ph.cg(c0) + ph.cg(c1));
    const double cs = 0.5 * (0.0 + 0.0);
    if (cl < 0.005 || cl > 0.995 || cg < 0.005 || cg > 0.995 || cs > 0.05) return 0.0;
    const double psi_f = 0.5 * (rd<K_SCALAR>(d, PSI, i, j, k) + rd<K_SCALAR>(d, PSI, a, b, e));
    const double id = C == 0 ? d.idx_c[i - 1] : (C == 1 ? d.idy_c[j - 1] : d.idz_c[k - 1]);
    const double gradC = (c0 - c1) * id;
    return scale * psi_f * gradC;
}

// the same face force in single precision (the FP32 stencil form)
template <int C>
__host__ __device__ __forceinline__ double f_sigma_f(const Dom3 &d, const Phase &ph, float scale, const double *CL,
                                                     const double *PSI, int i, int j, int k)
{
    const int a = C == 0 ? i - 1 : i, b = C == 1 ? j - 1 : j, e = C == 2 ? k - 1 : k;
    const float c0 = (float)rd<K_SCALAR>(d, CL, i, j, k), c1 = (float)rd<K_SCALAR>(d, CL, a, b, e);
    const float cl = 0.5f * (c0 + c1);
    const float cg = 0.5f * ((float)ph.cg(c0) + (float)ph.cg(c1));
    if (cl < 0.005f || cl > 0.995f || cg < 0.005f || cg > 0.995f) return 0.0;
    const float psi_f = 0.5f * ((float)rd<K_SCALAR>(d, PSI, i, j, k) + (float)rd<K_SCALAR>(d, PSI, a, b, e));
    const float id = (float)(C == 0 ? d.idx_c[i - 1] : (C == 1 ? d.idy_c[j - 1] : d.idz_c[k - 1]));
    return (double)(scale * psi_f * ((c0 - c1) * id));
}

__host__ __device__ __forceinline__ double weight(const Dom3 &d, int i, int j, int k) { return d.wx[i] * d.wy[j] * d.wz[k]; }

// ---------------------------------------------------------------------------
// the substep over an executor
// ---------------------------------------------------------------------------

template <class X>
struct Box3 {
    X x;
    Dom3 d;
    Phase ph;
    pvof_grid_desc g;
    pvof_params p;
    double *f[F3_COUNT] = {};
    double *vd[3] = {};       // velocity CG directions, one per component
    int stage = 0;
    double dt = 0.0, time = 0.0, clamp_total = 0.0;
    bool initialized = false;
    static constexpr int CHUNK = 8;   // CG iterations issued between two reads of the device flag
    // solver counters (PVOF_SOLVER_BIHARMONIC, _VELOCITY, _PRESSURE): solves,
    // iterations, cell-iterations since the context was created
    long long sol_launches[3] = {}, sol_iters[3] = {}, sol_cell_iters[3] = {};

    // ---- VOF_DIFFUSE_step (VOF_DIFFUSE.c:1262-1359), no solids ------------
    void vof_step(double a_dt)
    {
        const Dom3 d = this->d;
        const double *CL = f[F3_CL], *U = f[F3_U], *V = f[F3_V], *W = f[F3_W], *RN = f[F3_RN];
        double *CUR = f[F3_CUR], *VEC = f[F3_VEC], *AUX = f[F3_AUX];
        const int wo = p.weno_order, s = stage;
        const double pe = p.Pe_CH, gs = gamb(s), zs = zetb(s);
        if (p.stencil_fp32) {
            // the FP32 stencil form: fluxes, their divergence and L S in float;
            // each face flux is the same float number seen from both cells, so
            // the advection still telescopes
            x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
                auto c = [&](int a, int b, int e) { return (float)rd<K_SCALAR>(d, CL, a, b, e); };
                auto fx = [&](int a, int b, int e) {
                    src<K_WRAP_U>(d, a, b, e);
                    const float vel = (float)rd<K_U>(d, U, a, b, e);
                    return vel * face_state_f(wo, vel, a, b, e, 1, 0, 0, c);
                };
                auto fy = [&](int a, int b, int e) {
                    src<K_WRAP_V>(d, a, b, e);
                    const float vel = (float)rd<K_V>(d, V, a, b, e);
                    return vel * face_state_f(wo, vel, a, b, e, 0, 1, 0, c);
                };
                auto fz = [&](int a, int b, int e) {
                    src<K_WRAP_W>(d, a, b, e);
                    const float vel = (float)rd<K_W>(d, W, a, b, e);
                    return vel * face_state_f(wo, vel, a, b, e, 0, 0, 1, c);
                };
                const float div = (fx(i + 1, j, k) - fx(i, j, k)) / (float)d.dx_c[i] +
                                  (fy(i, j + 1, k) - fy(i, j, k)) / (float)d.dy_c[j] +
                                  (fz(i, j, k + 1) - fz(i, j, k)) / (float)d.dz_c[k];
                auto bulk = [&](int a, int b, int e) {
                    const float cc = c(a, b, e);
                    return 0.5f * cc - 1.5f * cc * cc + cc * cc * cc;
                };
                const double tmp = (double)lap3f(d, i, j, k, bulk) / pe;
                const double cu = -(double)div + tmp;
                const long long q = at(d, i, j, k);
                CUR[q] = cu;
                const double cl = CL[q];
                VEC[q] = (s == 0) ? a_dt * cl + gs * cu : a_dt * cl + gs * cu + zs * RN[q];
            });
        } else
        // VOF_DIFFUSE_advect_WENO5 (:931-996) + compute_bulk_S / explicit_diffusion
        // (:865-885, :998-1016) + the rhs assembly (:1290-1310): the face fluxes
        // after their exchange are evaluated at the face the exchange copies
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            auto c = [&](int a, int b, int e) { return rd<K_SCALAR>(d, CL, a, b, e); };
            auto fx = [&](int a, int b, int e) {
                src<K_WRAP_U>(d, a, b, e);
                const double vel = rd<K_U>(d, U, a, b, e);
                return vel * face_state(wo, vel, a, b, e, 1, 0, 0, c);
            };
            auto fy = [&](int a, int b, int e) {
                src<K_WRAP_V>(d, a, b, e);
                const double vel = rd<K_V>(d, V, a, b, e);
                return vel * face_state(wo, vel, a, b, e, 0, 1, 0, c);
            };
            auto fz = [&](int a, int b, int e) {
                src<K_WRAP_W>(d, a, b, e);
                const double vel = rd<K_W>(d, W, a, b, e);
                return vel * face_state(wo, vel, a, b, e, 0, 0, 1, c);
            };
            const double div = (fx(i + 1, j, k) - fx(i, j, k)) / d.dx_c[i] + (fy(i, j + 1, k) - fy(i, j, k)) / d.dy_c[j] +
                               (fz(i, j, k + 1) - fz(i, j, k)) / d.dz_c[k];
            auto bulk = [&](int a, int b, int e) {
                const double cc = c(a, b, e), cs = 0.0;
                return 0.5 * cc - 1.5 * cc * cc + cc * cc * cc - cc * cs * (1.0 - cc - cs);
            };
            const double tmp = lap3(d, i, j, k, bulk) / pe;
            const double cu = -div + tmp;
            const long long q = at(d, i, j, k);
            CUR[q] = cu;
            const double cl = CL[q];
            VEC[q] = (s == 0) ? a_dt * cl + gs * cu : a_dt * cl + gs * cu + zs * RN[q];
        });
        // VOF_DIFFUSE_solve_implicit_biharmonic (:1018-1069): aux = L C
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            AUX[at(d, i, j, k)] = lap3(d, i, j, k, [&](int a, int b, int e) { return rd<K_SCALAR>(d, CL, a, b, e); });
        });
    }

    // diffuse_solve_biharmonic_pcg (VOF_DIFFUSE.c:339-429) on x = C_L,
    // b = rhs_vec - (Cn^2/Pe) L L C (the first operator application is the
    // same L L C, so r0 = b - a_dt C - (Cn^2/Pe) L L C comes with it)
    void biharmonic(double a_dt)
    {
        const Dom3 d = this->d;
        Sc3 *sc = x.sc;
        double *CL = f[F3_CL], *VEC = f[F3_VEC], *AUX = f[F3_AUX], *R = f[F3_CHR], *PP = f[F3_CHP], *AP = f[F3_AP];
        const double bih = p.Cn * p.Cn / p.Pe_CH;
        const int maxit = (p.ch_iter_max > 0) ? p.ch_iter_max : p.CG_MAXIT;
        const double tol = (p.ch_tol > 0.0) ? p.ch_tol : p.CG_ETOL;
        const Range cr = cells_range(d);
        x.template reduce<2>(cr, nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            const double L = lap3(d, i, j, k, [&](int a, int b, int e) { return rd<K_SCALAR>(d, AUX, a, b, e); });
            const long long q = at(d, i, j, k);
            const double b = VEC[q] - bih * L;
            VEC[q] = b;
            const double ap = a_dt * CL[q] + bih * L;
            const double r = b - ap;
            R[q] = r;
            PP[q] = r;
            const double w = weight(d, i, j, k);
            return Vec<2>{{w * b * b, w * r * r}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            double rn = sqrt(s->sum[0][0]);
            if (rn < 1e-30) rn = 1.0;
            s->ch_rhs_norm = rn;
            s->ch_rz = s->sum[0][1];
            s->ch_rel = sqrt(s->sum[0][1]) / rn;
            s->ch_iter = 0;
            s->ch_maxit = maxit;
            s->ch_tol = tol;
            s->ch_active = (s->ch_rel < tol || maxit <= 0) ? 0 : 1;
        });
        const int *gate = &sc->ch_active;
        for (int it = 0; it < maxit; it += CHUNK) {
            for (int q = 0; q < CHUNK && it + q < maxit; q++) {
                x.cells(cr, gate, [=] __host__ __device__(int i, int j, int k) {
                    AUX[at(d, i, j, k)] =
                        lap3(d, i, j, k, [&](int a, int b, int e) { return rd<K_SCALAR>(d, PP, a, b, e); });
                });
                x.template reduce<1>(cr, gate, 0, [=] __host__ __device__(int i, int j, int k) {
                    const double L = lap3(d, i, j, k, [&](int a, int b, int e) { return rd<K_SCALAR>(d, AUX, a, b, e); });
                    const long long q = at(d, i, j, k);
                    const double pv = PP[q];
                    const double ap = a_dt * pv + bih * L;
                    AP[q] = ap;
                    return Vec<1>{{weight(d, i, j, k) * pv * ap}};
                });
                x.scalar(gate, [=] __host__ __device__(Sc3 * s) {
                    const double pAp = s->sum[0][0];
                    if (fabs(pAp) < 1e-30) s->ch_active = 0;
                    else s->ch_alpha = s->ch_rz / pAp;
                });
                x.template reduce<1>(cr, gate, 0, [=] __host__ __device__(int i, int j, int k) {
                    const double alpha = sc->ch_alpha;
                    const long long q = at(d, i, j, k);
                    CL[q] += alpha * PP[q];
                    const double r = R[q] - alpha * AP[q];
                    R[q] = r;
                    return Vec<1>{{weight(d, i, j, k) * r * r}};
                });
                x.scalar(gate, [=] __host__ __device__(Sc3 * s) {
                    const double rr = s->sum[0][0];
                    s->ch_iter++;
                    s->ch_rel = sqrt(rr) / s->ch_rhs_norm;
                    if (s->ch_rel < s->ch_tol) {
                        s->ch_active = 0;
                    } else {
                        s->ch_beta = rr / (s->ch_rz + 1e-30);
                        s->ch_rz = rr;
                        if (s->ch_iter >= s->ch_maxit) s->ch_active = 0;
                    }
                });
                x.cells(cr, gate, [=] __host__ __device__(int i, int j, int k) {
                    const long long q = at(d, i, j, k);
                    PP[q] = R[q] + sc->ch_beta * PP[q];
                });
            }
            if (!x.read_int(gate)) break;
        }
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->ch_iters_out = s->ch_iter;
            s->ch_rel_out = s->ch_rel;
        });
    }

    // diffuse_bound_liquid_fraction (VOF_DIFFUSE.c:1093-1127) without solids;
    // the mass change is summed over the physical cells (the reference's sum
    // also counts the half cells, which copy physical ones), the cells that
    // pvof_liquid_mass sums
    void clamp()
    {
        const Dom3 d = this->d;
        double *CL = f[F3_CL];
        x.template reduce<1>(cells_range(d), nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            const double old_cl = CL[q], cs = 0.0;
            double max_cl = 1.0 - cs;
            if (max_cl < 0.0) max_cl = 0.0;
            if (max_cl > 1.0) max_cl = 1.0;
            double new_cl = old_cl;
            if (new_cl < 0.0) new_cl = 0.0;
            if (new_cl > max_cl) new_cl = max_cl;
            CL[q] = new_cl;
            return Vec<1>{{(new_cl - old_cl) * (d.dx_u[i] * d.dy_v[j] * d.dz_w[k])}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) { s->clamp_delta = s->sum[0][0]; });
    }

    // VOF_DIFFUSE_compute_psi_LG (VOF_DIFFUSE.c:907-929)
    void psi_LG()
    {
        const Dom3 d = this->d;
        const double *CL = f[F3_CL];
        double *PSI = f[F3_PSI];
        const double cn2 = p.Cn * p.Cn;
        if (p.stencil_fp32) {
            const float cn2f = (float)cn2;
            x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
                const float L = lap3f(d, i, j, k, [&](int a, int b, int e) { return (float)rd<K_SCALAR>(d, CL, a, b, e); });
                const long long q = at(d, i, j, k);
                const float c = (float)CL[q];
                PSI[q] = (double)(c * c * c - 1.5f * c * c + 0.5f * c - cn2f * L);
            });
            return;
        }
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const double L = lap3(d, i, j, k, [&](int a, int b, int e) { return rd<K_SCALAR>(d, CL, a, b, e); });
            const long long q = at(d, i, j, k);
            const double c = CL[q];
            PSI[q] = c * c * c - 1.5 * c * c + 0.5 * c - cn2 * L;
        });
    }

    double fsig_scale() const { return 2.0 * 6.0 * std::sqrt(2.0) / (p.Cn * p.We + 1e-30); }

    // f_sigma of the start-up (Cart3d.c:1124-1130): new and old forces equal
    template <int C>
    void f_sigma_init()
    {
        const Dom3 d = this->d;
        const Phase ph = this->ph;
        const double *CL = f[F3_CL], *PSI = f[F3_PSI];
        double *FN = f[F3_FSN_X + C], *FO = f[F3_FSO_X + C];
        const double scale = fsig_scale();
        const int f32 = p.stencil_fp32;
        x.cells(face_range(d, C), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const double v = f32 ? f_sigma_f<C>(d, ph, (float)scale, CL, PSI, i, j, k) : f_sigma<C>(d, ph, scale, CL, PSI, i, j, k);
            FN[at(d, i, j, k)] = v;
            FO[at(d, i, j, k)] = v;
        });
    }

    // one momentum component: Velocity_*_set_implicit_explicit, _set_RHS
    // (Velocity.c:1494-2160), then in the substep's order f_sigma (new),
    // VOF_apply_f_sigma_old and Velocity_add_gravity_2_RHS
    // (VOF_SurfaceTension.c:1983-2154) at the same face
    template <int C>
    void momentum_rhs(double a_dt, double gdir)
    {
        const Dom3 d = this->d;
        const Phase ph = this->ph;
        const double *CL = f[F3_CL], *U = f[F3_U], *V = f[F3_V], *W = f[F3_W], *PR = f[F3_P], *PSI = f[F3_PSI];
        const double *DATA = f[F3_U + C], *FO = f[F3_FSO_X + C];
        double *EXO = f[F3_U_EXO + 3 * C], *VXO = f[F3_U_VXO + 3 * C], *RHS = f[F3_U_RHS + 3 * C], *FN = f[F3_FSN_X + C];
        const double iRe = 1.0 / p.Re, gs = gamb(stage), zs = zetb(stage);
        const double dpdx_src = (C == 0) ? 2.0 * (-p.dp_dx) : 0.0;
        const int st = p.surface_tension, grav = p.gravity;
        const double scale = fsig_scale(), Ri = p.richardson;
        const int f32 = p.stencil_fp32;
        x.cells(face_range(d, C), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const MomTerms t = mom_terms<C>(d, ph, iRe, CL, U, V, W, i, j, k);
            const int a = C == 0 ? i - 1 : i, b = C == 1 ? j - 1 : j, e = C == 2 ? k - 1 : k;
            const double id = C == 0 ? d.idx_c[i - 1] : (C == 1 ? d.idy_c[j - 1] : d.idz_c[k - 1]);
            const double dp = (rd<K_PRESSURE>(d, PR, i, j, k) - rd<K_PRESSURE>(d, PR, a, b, e)) * id;
            const double rf = 0.5 * (ph.rho(rd<K_SCALAR>(d, CL, i, j, k)) + ph.rho(rd<K_SCALAR>(d, CL, a, b, e)));
            const long long q = at(d, i, j, k);
            double conv = gs * t.ex + zs * EXO[q];
            conv *= rf;
            double r = rf * a_dt * DATA[q] + conv + t.im + (gs * t.vx + zs * VXO[q]) - 2.0 * dp;
            if (C == 0) r += dpdx_src;
            EXO[q] = t.ex;
            VXO[q] = t.vx;
            if (st) {
                FN[q] = f32 ? f_sigma_f<C>(d, ph, (float)scale, CL, PSI, i, j, k) : f_sigma<C>(d, ph, scale, CL, PSI, i, j, k);
                r += FO[q];
            }
            if (grav) r += 2.0 * rf * Ri * gdir;
            RHS[q] = r;
        });
    }

    // Velocity_solve_cg (msolve_cg.c:525-722) of component C
    template <int C>
    void velocity_solve()
    {
        constexpr int KN = C == 0 ? K_U : (C == 1 ? K_V : K_W);
        constexpr int KC = C == 0 ? K_U : (C == 1 ? K_V_CG : K_W);
        const Dom3 d = this->d;
        const Phase ph = this->ph;
        Sc3 *sc = x.sc;
        const double *CL = f[F3_CL], *RHS = f[F3_U_RHS + 3 * C];
        double *DATA = f[F3_U + C], *R = f[F3_VR], *AD = f[F3_VAD], *DG = f[F3_VDIAG], *DD = vd[C];
        const double iRe = 1.0 / p.Re, alpha_k = bet(stage), dt = this->dt;
        const double EPS = p.velocity_cg_unregularized ? 0.0 : 1e-14;
        const int NX = d.NX, NY = d.NY, NZ = d.NZ;
        const double in_tot = (C == 1) ? 1.0 / (double)((NX - 1) * (NY - 2) * (NZ - 1))
                                       : 1.0 / (double)((NX - 1) * (NY - 1) * (NZ - 1));
        const double tol = p.CG_ETOL;
        const int maxit = p.CG_MAXIT;
        const Range fr = face_range(d, C);
        x.template reduce<1>(fr, nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            const double dg = vel_diag<C>(d, ph, iRe, alpha_k, dt, CL, i, j, k);
            const double ad = vel_op<C, KN>(d, ph, iRe, alpha_k, dt, CL, DATA, i, j, k);
            const long long q = at(d, i, j, k);
            DG[q] = dg;
            const double r = RHS[q] - ad;
            R[q] = r;
            const double dd = r / (dg + EPS);
            DD[q] = dd;
            return Vec<1>{{r * dd}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->v_rz = s->sum[0][0];
            s->v_iter = 0;
            s->v_maxit = maxit;
            s->v_rms = 0.0;
            s->v_eps = EPS;
            s->v_in_tot = in_tot;
            s->v_tol = tol;
            s->v_active = maxit > 0 ? 1 : 0;
        });
        const int *gate = &sc->v_active;
        for (int it = 0; it < maxit; it += CHUNK) {
            for (int q = 0; q < CHUNK && it + q < maxit; q++) {
                x.template reduce<1>(fr, gate, 0, [=] __host__ __device__(int i, int j, int k) {
                    const double ad = vel_op<C, KC>(d, ph, iRe, alpha_k, dt, CL, DD, i, j, k);
                    const long long q = at(d, i, j, k);
                    AD[q] = ad;
                    return Vec<1>{{DD[q] * ad}};
                });
                x.scalar(gate, [=] __host__ __device__(Sc3 * s) {
                    s->v_iter++;
                    s->v_alpha = s->v_rz / (s->sum[0][0] + s->v_eps);
                });
                x.template reduce<2>(fr, gate, 0, [=] __host__ __device__(int i, int j, int k) {
                    const double alpha = sc->v_alpha, eps = sc->v_eps;
                    const long long q = at(d, i, j, k);
                    DATA[q] += alpha * DD[q];
                    const double r = R[q] - alpha * AD[q];
                    R[q] = r;
                    return Vec<2>{{r * r / (DG[q] + eps), r * r}};
                });
                x.scalar(gate, [=] __host__ __device__(Sc3 * s) {
                    const double rz_new = s->sum[0][0], rr = s->sum[0][1];
                    s->v_rms = sqrt(s->v_in_tot * rr);
                    if (s->v_rms < s->v_tol) {
                        s->v_active = 0;
                    } else {
                        s->v_beta = rz_new / (s->v_rz + s->v_eps);
                        s->v_rz = rz_new;
                        if (s->v_iter >= s->v_maxit) s->v_active = 0;
                    }
                });
                x.cells(fr, gate, [=] __host__ __device__(int i, int j, int k) {
                    const long long q = at(d, i, j, k);
                    DD[q] = R[q] / (DG[q] + sc->v_eps) + sc->v_beta * DD[q];
                });
            }
            if (!x.read_int(gate)) break;
        }
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->v_iters_out[C] = s->v_iter;
            s->v_rms_out[C] = s->v_rms;
        });
    }

    // Pressure_set_RHS (Pressure.c:100-196) and Pressure_compute_preconditioner
    void pressure_rhs_precond()
    {
        const Dom3 d = this->d;
        const Phase ph = this->ph;
        const double *U = f[F3_U], *V = f[F3_V], *W = f[F3_W], *CL = f[F3_CL];
        double *RHS = f[F3_PRHS], *M = f[F3_PM], *CX = f[F3_PCX], *CY = f[F3_PCY], *CZ = f[F3_PCZ];
        const double a_dt = 1.0 / (dt * 2.0 * bet(stage));
        const double ihdt = d.idx_u1 * a_dt;
        // the +x, +y, +z face coefficients of the cells and of one layer below
        x.cells(Range{-1, d.NX - 1, -1, d.NY - 1, -1, d.NZ - 1}, nullptr, [=] __host__ __device__(int i, int j, int k) {
            auto rho = [&](int a, int b, int e) { return ph.rho(rd<K_SCALAR>(d, CL, a, b, e)); };
            const long long q = at(d, i, j, k);
            const double r0 = rho(i, j, k);
            CX[q] = 2.0 / (r0 + rho(i + 1, j, k)) * d.idx2;
            CY[q] = 2.0 / (r0 + rho(i, j + 1, k)) * d.idy2;
            CZ[q] = 2.0 / (r0 + rho(i, j, k + 1)) * d.idz2;
        });
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            RHS[q] = cc_div(d, U, V, W, i, j, k, ihdt, ihdt, ihdt);
            const double aii = CX[q - 1] + CX[q] + CY[q - d.P] + CY[q] + CZ[q - d.S] + CZ[q];
            M[q] = 1.0 / (1.0 * aii + 1e-12);
        });
    }

    // the same solve preconditioned by z = s (-L)^-1 (s r), L the operator at
    // density one and s the square root of the Jacobi weights
    // (pressure_preconditioner = 1, no counterpart in the reference); the
    // stopping test stays the reference's sqrt(r.Mr) < P_CG_ETOL, M the
    // Jacobi weights, so the result moves within that tolerance
    void pressure_solve_spectral()
    {
        const Dom3 d = this->d;
        Sc3 *sc = x.sc;
        const double *B = f[F3_PRHS], *M = f[F3_PM], *CX = f[F3_PCX], *CY = f[F3_PCY], *CZ = f[F3_PCZ];
        double *PHI = f[F3_DP], *R = f[F3_PR], *DD = f[F3_PD], *AD = f[F3_PAD], *Z = f[F3_PZ];
        const double tol = p.P_CG_ETOL;
        const int maxit = p.P_CG_MAXIT;
        const Range cr = cells_range(d);
        x.template reduce<1>(cr, nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            const double r = B[q] - p_apply_st(d, CX, CY, CZ, PHI, i, j, k);
            R[q] = r;
            return Vec<1>{{r * (r * M[q])}};
        });
        // z = P r and gamma = r.z, then d = z
        x.spec_apply(d, R, M, Z, nullptr, [=] __host__ __device__(Sc3 * s, double rz) {
            s->p_gamma = rz;
            s->p_beta = 0.0;
        });
        x.p_dir_z(d, Z, DD, nullptr);
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->p_gamma_new = s->sum[0][0];   // r.Mr: the stopping quantity
            s->p_iter = 0;
            s->p_maxit = maxit;
            s->p_tol = tol;
            const int conv = sqrt(s->p_gamma_new) < tol;
            s->p_ran = conv ? 0 : 1;
            s->p_active = (conv || maxit <= 0) ? 0 : 1;
        });
        const int *gate = &sc->p_active;
        for (int it = 0; it < maxit; it += CHUNK) {
            for (int q = 0; q < CHUNK && it + q < maxit; q++) {
                x.p_apply(d, CX, CY, CZ, DD, AD, gate, [=] __host__ __device__(Sc3 * s, double dAd) {
                    s->p_alpha = s->p_gamma / (dAd + 1e-300);
                });
                x.p_update(d, PHI, R, DD, AD, M, gate, [=] __host__ __device__(Sc3 * s, double rMr) {
                    s->p_iter++;
                    s->p_gamma_new = rMr;
                    if (sqrt(rMr) < s->p_tol) s->p_active = 0;
                });
                // z = P r, r.z and the direction's coefficient, then d = z + beta d
                x.spec_apply(d, R, M, Z, gate, [=] __host__ __device__(Sc3 * s, double g) {
                    s->p_beta = g / (s->p_gamma + 1e-300);
                    s->p_gamma = g;
                    if (s->p_iter >= s->p_maxit) s->p_active = 0;
                });
                x.p_dir_z(d, Z, DD, gate);
            }
            if (!x.read_int(gate)) break;
        }
        const int *ran = &sc->p_ran;
        const double count = (double)((long long)(d.NX - 1) * (d.NY - 1) * (d.NZ - 1));
        x.template reduce<1>(cr, ran, 0, [=] __host__ __device__(int i, int j, int k) {
            return Vec<1>{{PHI[at(d, i, j, k)]}};
        });
        x.scalar(ran, [=] __host__ __device__(Sc3 * s) { s->p_avg = s->sum[0][0] / count; });
        x.cells(cr, ran, [=] __host__ __device__(int i, int j, int k) { PHI[at(d, i, j, k)] -= sc->p_avg; });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->p_iters_out = s->p_iter;
            s->p_res_out = sqrt(s->p_gamma_new);
        });
    }

    // Pressure_solve_cg (psolve_cg.c:130-293) for deltap from zero
    void pressure_solve()
    {
        if (p.pressure_preconditioner) {
            pressure_solve_spectral();
            return;
        }
        const Dom3 d = this->d;
        Sc3 *sc = x.sc;
        const double *B = f[F3_PRHS], *M = f[F3_PM], *CX = f[F3_PCX], *CY = f[F3_PCY], *CZ = f[F3_PCZ];
        double *PHI = f[F3_DP], *R = f[F3_PR], *DD = f[F3_PD], *AD = f[F3_PAD];
        const double tol = p.P_CG_ETOL;
        const int maxit = p.P_CG_MAXIT;
        const Range cr = cells_range(d);
        x.template reduce<1>(cr, nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            const double r = B[q] - p_apply_st(d, CX, CY, CZ, PHI, i, j, k);
            R[q] = r;
            const double z = r * M[q];
            DD[q] = z;
            return Vec<1>{{r * z}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->p_gamma = s->sum[0][0];
            s->p_gamma_new = s->p_gamma;
            s->p_iter = 0;
            s->p_maxit = maxit;
            s->p_tol = tol;
            const int conv = sqrt(s->p_gamma) < tol;
            s->p_ran = conv ? 0 : 1;
            s->p_active = (conv || maxit <= 0) ? 0 : 1;
        });
        const int *gate = &sc->p_active;
        for (int it = 0; it < maxit; it += CHUNK) {
            for (int q = 0; q < CHUNK && it + q < maxit; q++) {
                // AD = A d and d.AD (the executor's streaming form of p_apply_st),
                // then the step length from the finished sum
                x.p_apply(d, CX, CY, CZ, DD, AD, gate, [=] __host__ __device__(Sc3 * s, double dAd) {
                    s->p_alpha = s->p_gamma / (dAd + 1e-30);
                });
                // phi += alpha d, r -= alpha AD and r.(M r), then the stopping test
                // and the direction's coefficient
                x.p_update(d, PHI, R, DD, AD, M, gate, [=] __host__ __device__(Sc3 * s, double rz) {
                    s->sum[0][0] = rz;
                    s->p_iter++;
                    s->p_gamma_new = s->sum[0][0];
                    if (sqrt(s->p_gamma_new) < s->p_tol) {
                        s->p_active = 0;
                    } else {
                        s->p_beta = s->p_gamma_new / (s->p_gamma + 1e-30);
                        s->p_gamma = s->p_gamma_new;
                        if (s->p_iter >= s->p_maxit) s->p_active = 0;
                    }
                });
                // d = M r + beta d
                x.p_dir(d, R, M, DD, gate);
            }
            if (!x.read_int(gate)) break;
        }
        // mean removal (psolve_cg.c:255-279), only after the iteration ran
        const int *ran = &sc->p_ran;
        const double count = (double)((long long)(d.NX - 1) * (d.NY - 1) * (d.NZ - 1));
        x.template reduce<1>(cr, ran, 0, [=] __host__ __device__(int i, int j, int k) {
            return Vec<1>{{PHI[at(d, i, j, k)]}};
        });
        x.scalar(ran, [=] __host__ __device__(Sc3 * s) { s->p_avg = s->sum[0][0] / count; });
        x.cells(cr, ran, [=] __host__ __device__(int i, int j, int k) { PHI[at(d, i, j, k)] -= sc->p_avg; });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) {
            s->p_iters_out = s->p_iter;
            s->p_res_out = sqrt(s->p_ran ? s->p_gamma_new : s->p_gamma);
        });
    }

    // Pressure_project_velocity (Pressure.c:218-464)
    void project()
    {
        const Dom3 d = this->d;
        const double *DP = f[F3_DP], *CL = f[F3_CL];
        double *P = f[F3_P];
        const double mdt = 2.0 * bet(stage) * dt;
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            P[q] += DP[q];
        });
        project_comp<0>(mdt, DP, CL);
        project_comp<1>(mdt, DP, CL);
        project_comp<2>(mdt, DP, CL);
    }
    template <int C>
    void project_comp(double mdt, const double *DP, const double *CL)
    {
        const Dom3 d = this->d;
        const Phase ph = this->ph;
        double *DATA = f[F3_U + C];
        x.cells(face_range(d, C), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const int a = C == 0 ? i - 1 : i, b = C == 1 ? j - 1 : j, e = C == 2 ? k - 1 : k;
            const double inv = 2.0 / (ph.rho(rd<K_SCALAR>(d, CL, i, j, k)) + ph.rho(rd<K_SCALAR>(d, CL, a, b, e)));
            const double id = C == 0 ? d.idx_c[i - 1] : (C == 1 ? d.idy_c[j - 1] : d.idz_c[k - 1]);
            DATA[at(d, i, j, k)] -= (rd<K_PRESSURE>(d, DP, i, j, k) - rd<K_PRESSURE>(d, DP, a, b, e)) * (id * mdt * inv);
        });
    }

    // Pressure_compute_velocity_divergence (Pressure.c:475-597)
    void divergence()
    {
        const Dom3 d = this->d;
        const double *U = f[F3_U], *V = f[F3_V], *W = f[F3_W];
        x.template reduce<1, true>(cells_range(d), nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            return Vec<1>{{fabs(cc_div(d, U, V, W, i, j, k, d.idx_u[i], d.idy_v[j], d.idz_w[k]))}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) { s->div_max = s->sum[0][0]; });
    }

    // ---- start-up (Cart3d.c:1096-1130 and the boundary updates before it)
    int initialize()
    {
        const Dom3 d = this->d;
        const double *FF = f[F3_F];
        double *CL = f[F3_CL];
        // VOF_DIFFUSE_init (VOF_DIFFUSE.c:524-568): C_L = clamp(F); the clamp
        // and phase-cache passes after it change nothing without solids
        x.cells(cells_range(d), nullptr, [=] __host__ __device__(int i, int j, int k) {
            const long long q = at(d, i, j, k);
            CL[q] = clamp01(FF[q]);
        });
        if (p.surface_tension) {
            psi_LG();
            f_sigma_init<0>();
            f_sigma_init<1>();
            f_sigma_init<2>();
        }
        time = 0.0;
        clamp_total = 0.0;
        initialized = true;
        return x.status();
    }

    // Temporal_int_all_the_equations (Temporal_int.c:563-1279), no solids
    int substep(pvof_stats *st)
    {
        if (!(dt > 0.0)) return PVOF_EINVAL;
        const double a_dt = 1.0 / (dt * bet(stage));
        const Range cr = cells_range(d);
        const long long ncell = (long long)(cr.i1 - cr.i0) * (cr.j1 - cr.j0) * (cr.k1 - cr.k0);
        long long nface[3];
        for (int c = 0; c < 3; c++) {
            const Range fr = face_range(d, c);
            nface[c] = (long long)(fr.i1 - fr.i0) * (fr.j1 - fr.j0) * (fr.k1 - fr.k0);
        }
        vof_step(a_dt);
        x.tic();
        biharmonic(a_dt);
        x.toc(0);
        clamp();
        std::swap(f[F3_RN], f[F3_CUR]);
        // momentum right-hand sides; psi_LG first, as f_sigma reads it
        if (p.surface_tension) psi_LG();
        double gx = 0.0, gy = 0.0, gz = 0.0;
        const double gm = std::sqrt(p.grav[0] * p.grav[0] + p.grav[1] * p.grav[1] + p.grav[2] * p.grav[2]);
        if (gm > 0.0) {
            gx = p.grav[0] / gm;
            gy = p.grav[1] / gm;
            gz = p.grav[2] / gm;
        }
        momentum_rhs<0>(a_dt, gx);
        momentum_rhs<1>(a_dt, gy);
        momentum_rhs<2>(a_dt, gz);
        x.tic();
        velocity_solve<0>();
        velocity_solve<1>();
        velocity_solve<2>();
        x.toc(1);
        // the outer Poisson loop (Temporal_int.c:1052-1107)
        int passes = 0, rc = PVOF_OK, p_total = 0;
        double div = 0.0;
        Sc3 s;
        do {
            x.zero(f[F3_DP]);
            pressure_rhs_precond();
            x.tic();
            pressure_solve();
            x.toc(2);
            project();
            divergence();
            s = x.read_scalars();
            const int xs = x.status();
            if (xs < 0) return xs;
            div = s.div_max;
            p_total += s.p_iters_out;
            sol_launches[2]++;
            sol_iters[2] += s.p_iters_out;
            sol_cell_iters[2] += s.p_iters_out * ncell;
            passes++;
            if (passes > 10) {
                rc = PVOF_EDIVERGED;
                break;
            }
        } while (div > 1e-6);
        if (p.surface_tension)
            for (int c = 0; c < 3; c++) std::swap(f[F3_FSO_X + c], f[F3_FSN_X + c]);
        clamp_total += s.clamp_delta;
        sol_launches[0]++;
        sol_iters[0] += s.ch_iters_out;
        sol_cell_iters[0] += s.ch_iters_out * ncell;
        for (int c = 0; c < 3; c++) {
            sol_launches[1]++;
            sol_iters[1] += s.v_iters_out[c];
            sol_cell_iters[1] += s.v_iters_out[c] * nface[c];
        }
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->ch_iters = s.ch_iters_out;
            st->ch_rel_res = s.ch_rel_out;
            st->u_iters = s.v_iters_out[0];
            st->v_iters = s.v_iters_out[1];
            st->w_iters = s.v_iters_out[2];
            st->u_rms = s.v_rms_out[0];
            st->v_rms = s.v_rms_out[1];
            st->w_rms = s.v_rms_out[2];
            st->p_iters = s.p_iters_out;
            st->p_iters_total = p_total;
            st->p_res = s.p_res_out;
            st->poisson_passes = passes;
            st->div_max = div;
            st->clamp_mass = s.clamp_delta;
        }
        return rc;
    }

    int run_steps(int nsteps, double step_dt, pvof_stats *st)
    {
        pvof_stats local;
        std::memset(&local, 0, sizeof(local));
        for (int n = 0; n < nsteps; n++)
            for (int rk = 0; rk < 3; rk++) {
                stage = rk;
                dt = step_dt;
                int rc = substep(&local);
                if (st) *st = local;
                if (rc < 0) return rc;
                time += step_dt * bet2(rk);
            }
        return PVOF_OK;
    }

    // liquid volume: sum of C_L times the cell measure over the physical cells
    int liquid_mass(double *out)
    {
        const Dom3 d = this->d;
        const double *CL = f[F3_CL];
        x.template reduce<1>(cells_range(d), nullptr, 0, [=] __host__ __device__(int i, int j, int k) {
            return Vec<1>{{d.dx_u[i] * d.dy_v[j] * d.dz_w[k] * CL[at(d, i, j, k)]}};
        });
        x.scalar(nullptr, [=] __host__ __device__(Sc3 * s) { s->mass = s->sum[0][0]; });
        *out = x.read_double(&x.sc->mass);
        return x.status();
    }
};

}  // namespace pvof3
