// Immersed-boundary routines of the diffuse-interface substep for resolved
// solid particles in the planar 2D mode (the reference's VOF_IBM +
// LAG_PARTICLE_RESOLVED + TWOD_CARTESIAN build):
//
//   particle lists at the start of a substep   Particle_MPI_update (single rank,
//                                              Lagrangian/Particle.c:2042-2500)
//   markers and their flags                    Lagrangian_flag_points,
//                                              Lagrangian_generate_points_2d
//                                              (Lagrangian/Lagrangian.c:2515-2800, :2900-2995)
//   solid fraction C_S                         VOF_DIFFUSE_compute_C_S (Eulerian/VOF_DIFFUSE.c:685-813)
//   explicit momentum predictor                Velocity_solve_explicit (lsolver/msolve_direct.c:146-260)
//   direct forcing                             Lagrangian_force, Lagrangian_force_individual
//                                              (Lagrangian/Lagrangian.c:1724-2505), with
//                                              Interpolate_Eul_to_Lag_twod / _Lag_to_Eul_uniform_twod
//                                              and delta (Lagrangian/Interpolate.c:390-560)
//
// Particle bookkeeping (lists, periodic copies, markers, flags) is host work on
// a few hundred markers; the gathers, the per-particle force and torque sums
// and the spreads run on the device.  The spread is written as a gather: each
// cell adds the contributions of a particle's markers in marker order, which
// is the order in which the reference's scatter adds them, so the result is
// the reference's to the last bit.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

constexpr double IBM_PI = 3.14159265358979323846;   // PI, Include/definitions.h:7
constexpr double DELTA_FUNC_RADIUS = 1.5;           // Include/definitions.h:58
constexpr double LAG_FLAG_RANGE = 3.0;              // Include/definitions.h:61
constexpr double LUB_RANGE = 2.0;                   // [particle] lub_range default (IO/default.inp)

// ---------------------------------------------------------------------------
// host: particle lists, markers and flags
// ---------------------------------------------------------------------------

// Particle_calc_derived_data (Lagrangian/Particle.c:663-733), planar branch
static void derived_data(IbmEntry &e, const IbmGrid &g)
{
    const double h = g.dy_min;
    const double R2 = e.R * e.R;
    double slab = g.slab > 0.0 ? g.slab : g.twod_slab;
    if (slab <= 0.0) slab = h;
    int N_L = (int)ceil(2.0 * IBM_PI * e.R / h);
    e.N_L = N_L > 8 ? N_L : 8;
    e.M = e.rho_s * IBM_PI * R2 * slab;
    e.I_p = e.rho_s * 0.5 * IBM_PI * R2 * R2 * slab;
    e.Vol_L = (2.0 * IBM_PI * e.R / e.N_L) * slab * h;
}

// Particle_ibm_exchange_range (Lagrangian/Particle.c:26-47) plus the marker-flag
// and lubrication ranges added in Particle_MPI_update (:2052-2060)
static double exchange_range(const IbmGrid &g, double Cn)
{
    const double h = g.h;
    double range = DELTA_FUNC_RADIUS * h;
    const double h_ref = (g.dy_min > 0.0) ? g.dy_min : h;
    const double cn = (Cn > 0.0) ? Cn : 0.0;
    const double wetting = 8.0 * ((cn > h_ref) ? cn : h_ref);
    if (wetting > range) range = wetting;
    range += LAG_FLAG_RANGE * h;
    const double lub = 0.5 * LUB_RANGE * h;
    return range > lub ? range : lub;
}

// One list of Particle_MPI_update on a single rank: local -> local + periodic
// copies; copies are prepended in the order the exchanges add them.
static std::vector<IbmEntry> update_list(const std::vector<IbmEntry> &local, const IbmGrid &g, double Cn)
{
    std::vector<IbmEntry> list = local;
    const double range = exchange_range(g, Cn);
    for (int axis = 0; axis < 2; axis++) {
        if (!g.periodic[axis]) continue;
        const double lo = (axis == 0 ? g.xu[0] : g.yv[0]) + range;
        const double hi = (axis == 0 ? g.xu[g.NX - 1] : g.yv[g.NY - 1]) - range;
        const double L = axis == 0 ? g.Lx : g.Ly;
        std::vector<IbmEntry> low, high;
        for (const IbmEntry &p : list)
            if (p.X[axis] - p.R < lo) { IbmEntry c = p; c.X[axis] += L; c.copy = 1; low.push_back(c); }
        for (const IbmEntry &p : list)
            if (p.X[axis] + p.R > hi) { IbmEntry c = p; c.X[axis] -= L; c.copy = 1; high.push_back(c); }
        std::vector<IbmEntry> out = high;
        out.insert(out.end(), low.begin(), low.end());
        out.insert(out.end(), list.begin(), list.end());
        list.swap(out);
    }
    return list;
}

// Lagrangian_near_point_2d (Lagrangian/Lagrangian.c:86-96)
static bool near_point(double x, double y, double range, const IbmGrid &g)
{
    const double xs = g.xu[0], xe = g.xu[g.NX - 1], ys = g.yv[0], ye = g.yv[g.NY - 1];
    return xs - x < range && x - xe < range && ys - y < range && y - ye < range;
}

// Lagrangian_generate_points_2d, planar branch (Lagrangian/Lagrangian.c:2900-2947)
static void generate_points(IbmEntry &e, const IbmGrid &g, IbmMarkers &m)
{
    const double h = g.h;
    const double range = DELTA_FUNC_RADIUS * h;
    const double dtheta = 2.0 * IBM_PI / e.N_L;
    const double ds = e.R * dtheta;
    double slab = g.slab;
    if (slab <= 0.0) slab = h;
    e.moff = (int)m.x.size();
    for (int mv = 0; mv < e.N_L; mv++) {
        const double theta = (mv + 0.5) * dtheta;
        const double nx = cos(theta), ny = sin(theta);
        const double x = e.X[0] + e.R * nx;
        const double y = e.X[1] + e.R * ny;
        if (near_point(x, y, range, g)) {
            m.x.push_back(x);
            m.y.push_back(y);
            m.vol.push_back(ds * slab * h);
            m.flag.push_back(1);
        }
    }
    e.mcount = (int)m.x.size() - e.moff;
}

// Lagrangian_flag_points_individual (Lagrangian/Lagrangian.c:2629-2690), 2D
static void flag_individual(const IbmEntry &p, const IbmEntry &p2, const IbmGrid &g, IbmMarkers &m)
{
    const double h = g.h;
    double dpp = p.R + p2.R + LAG_FLAG_RANGE * h;
    dpp = dpp * dpp;
    double dlp = p2.R + LAG_FLAG_RANGE * h;
    dlp = dlp * dlp;
    double r0 = p2.X[0] - p.X[0], r1 = p2.X[1] - p.X[1];
    if (!(r0 * r0 + r1 * r1 < dpp)) return;
    for (int q = p.moff; q < p.moff + p.mcount; q++) {
        r0 = p2.X[0] - m.x[q];
        r1 = p2.X[1] - m.y[q];
        const double d2 = r0 * r0 + r1 * r1;
        if (m.flag[q] == 1 && d2 < dlp) m.flag[q] = 0;
    }
}

// Lagrangian_flag_points_wall (Lagrangian/Lagrangian.c:2697-2795), x and y walls
static void flag_walls(const IbmEntry &p, const IbmGrid &g, IbmMarkers &m)
{
    const double h = g.h;
    const double dpw = p.R + 0.5 * LAG_FLAG_RANGE * h;
    const double dlw = 0.5 * LAG_FLAG_RANGE * h;
    auto wall = [&](int axis, double pos) {
        const double c = axis == 0 ? p.X[0] : p.X[1];
        if (!(fabs(c - pos) < dpw)) return;
        for (int q = p.moff; q < p.moff + p.mcount; q++) {
            const double v = axis == 0 ? m.x[q] : m.y[q];
            if (m.flag[q] == 1 && fabs(v - pos) < dlw) m.flag[q] = 0;
        }
    };
    if (!g.periodic[0]) {
        wall(0, g.xu[0]);
        wall(0, g.xu[g.NX - 1]);
    }
    if (!g.periodic[1]) {
        wall(1, g.yv[0]);
        wall(1, g.yv[g.NY - 1]);
    }
}

void ibm_build(const std::vector<IbmEntry> &mobile_local, const std::vector<IbmEntry> &fixed_local, const IbmGrid &g,
               double Cn, std::vector<IbmEntry> &entries, IbmMarkers &m)
{
    std::vector<IbmEntry> mob = update_list(mobile_local, g, Cn);
    std::vector<IbmEntry> fix = update_list(fixed_local, g, Cn);
    for (IbmEntry &e : mob) { e.mobile = 1; derived_data(e, g); }
    for (IbmEntry &e : fix) { e.mobile = 0; derived_data(e, g); }
    m = IbmMarkers();
    // Lagrangian_flag_points: mobile list first, then fixed
    for (IbmEntry &p : mob) {
        generate_points(p, g, m);
        for (const IbmEntry &p2 : mob)
            if (p2.id != p.id) flag_individual(p, p2, g, m);
        for (const IbmEntry &p2 : fix) flag_individual(p, p2, g, m);
        flag_walls(p, g, m);
    }
    for (IbmEntry &p : fix) {
        generate_points(p, g, m);
        for (const IbmEntry &p2 : mob) flag_individual(p, p2, g, m);
        for (const IbmEntry &p2 : fix)
            if (p2.id != p.id) flag_individual(p, p2, g, m);
        flag_walls(p, g, m);
    }
    entries = mob;
    entries.insert(entries.end(), fix.begin(), fix.end());
    // cell box of every particle's marker supports (3 x 3 stencils), for the spread
    for (IbmEntry &e : entries) {
        e.box[0] = e.box[2] = 1 << 30;
        e.box[1] = e.box[3] = -(1 << 30);
        for (int q = e.moff; q < e.moff + e.mcount; q++) {
            const int i = (int)floor((m.x[q] - g.xu[0]) / g.h), j = (int)floor((m.y[q] - g.yv[0]) / g.h);
            e.box[0] = std::min(e.box[0], i - 3);
            e.box[1] = std::max(e.box[1], i + 4);
            e.box[2] = std::min(e.box[2], j - 3);
            e.box[3] = std::max(e.box[3], j + 4);
        }
    }
}

// VOF_DIFFUSE_compute_C_S geometry (VOF_DIFFUSE.c:57-85 through
// Particle_collect_owned_overlaps, Lagrangian/Particle.c:1697-1786): on one
// rank every particle whose centre the rank owns, unshifted -- the overlap
// test takes the first shift that overlaps and the unshifted one always does
// -- so a particle crossing a periodic boundary has no copy in C_S.  The
// maximum over particles does not depend on their order.
void ibm_solid_geometry(const std::vector<IbmEntry> &mobile_local, const std::vector<IbmEntry> &fixed_local,
                        const IbmGrid &g, std::vector<double> &geo)
{
    geo.clear();
    const double x0 = g.xu[0], x1 = g.xu[g.NX - 1], y0 = g.yv[0], y1 = g.yv[g.NY - 1];
    for (const std::vector<IbmEntry> *l : {&mobile_local, &fixed_local})
        for (const IbmEntry &p : *l) {
            if (!(p.X[0] >= x0 && p.X[0] <= x1 && p.X[1] >= y0 && p.X[1] <= y1)) continue;
            geo.push_back(p.X[0]);
            geo.push_back(p.X[1]);
            geo.push_back(p.R);
        }
}

// diffuse_solid_support_extra (Eulerian/VOF_DIFFUSE.c:42-55) and the profile constants
void ibm_solid_constants(double cn, double &shift, double &denom, double &extra)
{
    shift = sqrt(2.0) * log(19.0) * cn;
    denom = 2.0 * sqrt(2.0) * cn;
    extra = 0.0;
    if (cn <= 0.0) return;
    const double eps = 1.0e-12;   // DIFFUSE_SOLID_GEOM_CUTOFF (VOF_DIFFUSE.c:23)
    const double x = 1.0 - 2.0 * eps;
    const double atanh_x = 0.5 * log((1.0 + x) / (1.0 - x));
    const double e = -shift + denom * atanh_x;
    extra = e > 0.0 ? e : 0.0;
}

// ---------------------------------------------------------------------------
// device
// ---------------------------------------------------------------------------

// delta (Lagrangian/Interpolate.c:551-560)
__device__ __forceinline__ double ibm_delta(double r)
{
    r = fabs(r);
    if (r <= 0.5) return (1 + sqrt(-3 * r * r + 1)) / 3;
    else if (r <= 1.5) return (5 - 3 * r - sqrt(-3 * (1 - r) * (1 - r) + 1)) / 6;
    return 0;
}

// Interpolate_Eul_to_Lag_twod (Interpolate.c:477-529): one marker per thread
__global__ void k_ibm_interp(Dom d, const double *__restrict__ a, const double *__restrict__ xs,
                             const double *__restrict__ ys, double h, const double *__restrict__ XL,
                             const double *__restrict__ YL, int nm, double *__restrict__ out)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nm) return;
    const int P = d.P;
    int i_start = (int)round((XL[m] - xs[0]) / h) - 1;
    int j_start = (int)round((YL[m] - ys[0]) / h) - 1;
    int i_end = i_start + 3, j_end = j_start + 3;
    i_start = max(i_start, -NG);
    j_start = max(j_start, -NG);
    i_end = min(i_end, d.NX + NG);
    j_end = min(j_end, d.NY + NG);
    double A = 0.0;
    for (int j = j_start; j < j_end; j++) {
        const double r1 = YL[m] - ys[j];
        for (int i = i_start; i < i_end; i++) {
            const double r0 = XL[m] - xs[i];
            A += 1 * AT_(a, i, j) * (ibm_delta(r0 / h) * ibm_delta(r1 / h));
        }
    }
    out[m] = A;
}

// Marker forces of one velocity component and the particle reaction force
// and torque (Lagrangian.c:2119-2170 for u, :2280-2335 for v): one thread per
// particle, its markers in order.
__global__ void k_ibm_marker_force(IbmDev D, int comp, int nentries, double idt2beta, int reset)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nentries) return;
    const IbmEntryDev &p = D.ent[e];
    double *F = D.FT + 6 * e, *T = F + 3;
    if (reset) { F[0] = F[1] = F[2] = T[0] = T[1] = T[2] = 0.0; }
    for (int q = p.moff; q < p.moff + p.mcount; q++) {
        if (D.flag[q] == 0) { D.FL[q] = 0.0; continue; }
        const double r0 = D.XL[q] - p.X[0], r1 = D.YL[q] - p.X[1], r2 = p.Zs - p.X[2];
        const double Ud = comp == 0 ? p.U[0] + p.Omega[1] * r2 - p.Omega[2] * r1
                                    : p.U[1] + p.Omega[2] * r0 - p.Omega[0] * r2;
        const double rho_L = D.rhoL[q];
        const double FL = idt2beta * (Ud - D.UL[q]);
        const double x = D.XL[q], y = D.YL[q];
        if (x >= D.xlo && x < D.xhi && y >= D.ylo && y < D.yhi) {   // Lagrangian_local_point_2d
            const double M = D.vol[q];
            if (comp == 0) {
                F[0] -= rho_L * M * FL;
                T[2] += rho_L * M * r1 * FL;
            } else {
                F[1] -= rho_L * M * FL;
                T[2] -= rho_L * M * r0 * FL;
            }
        }
        D.FL[q] = FL;
    }
}

// Interpolate_Lag_to_Eul_uniform_twod (Interpolate.c:390-475) of one particle
// as a gather, then rhs += 2 rho_face temp (Lagrangian.c:2176-2190, :2338-2350)
__global__ void k_ibm_spread(Dom d, IbmDev D, int e, int comp, const double *__restrict__ xs,
                             const double *__restrict__ ys, const double *__restrict__ rho, double *__restrict__ rhs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= d.NX || j >= d.NY) return;
    const int P = d.P;
    const IbmEntryDev &p = D.ent[e];
    const double h = D.h;
    double temp = 0.0;
    if (i >= p.box[0] && i < p.box[1] && j >= p.box[2] && j < p.box[3]) {
        const double cellv = D.dxu1 * D.dyv[j] * D.slab;   // Interpolate_twod_cell_volume, planar
        for (int q = p.moff; q < p.moff + p.mcount; q++) {
            int i_start = (int)round((D.XL[q] - xs[0]) / h) - 1;
            int j_start = (int)round((D.YL[q] - ys[0]) / h) - 1;
            int i_end = i_start + 3, j_end = j_start + 3;
            i_start = max(i_start, 0);
            i_end = min(max(i_end, 0), d.NX);
            j_start = min(max(j_start, 0), d.NY);
            j_end = min(max(j_end, 0), d.NY);
            if (i < i_start || i >= i_end || j < j_start || j >= j_end) continue;
            const double r1 = D.YL[q] - ys[j];
            const double r0 = D.XL[q] - xs[i];
            const double dV = D.vol[q] / cellv;
            temp += 1 * D.FL[q] * (ibm_delta(r0 / h) * ibm_delta(r1 / h)) * dV;
        }
    }
    const double rho_face = comp == 0 ? 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j)) : 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
    AT_(rhs, i, j) += 2.0 * rho_face * temp;
}

// corrector update u += beta dt rhs / rho_face over the G range (Lagrangian.c:1832-1851)
__global__ void k_ibm_correct(Dom d, int comp, double dtbeta, const double *__restrict__ rhs,
                              const double *__restrict__ rho, double *__restrict__ vel)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= d.NX || j >= d.NY) return;
    const int P = d.P;
    const double rf = comp == 0 ? 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j)) : 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
    AT_(vel, i, j) += dtbeta * AT_(rhs, i, j) / rf;
}

// a = 0 (reset == 1) or a -= b over the G range
__global__ void k_ibm_ng_update(Dom d, double *__restrict__ a, const double *__restrict__ b, int reset)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= d.NX || j >= d.NY) return;
    const int P = d.P;
    if (reset) AT_(a, i, j) = 0.0;
    else AT_(a, i, j) -= AT_(b, i, j);
}

// Velocity_solve_explicit (msolve_direct.c:146-260), VOF branch, over the solve range
__global__ void k_vel_explicit(Dom d, int comp, int i0, int i1, int j0, int j1, double dtimeb,
                               const double *__restrict__ rhs, const double *__restrict__ rho, double *__restrict__ vel)
{
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = j0 + blockIdx.y;
    if (i >= i1 || j >= j1) return;
    const int P = d.P;
    double rho_face = comp == 0 ? 0.5 * (AT_(rho, i - 1, j) + AT_(rho, i, j)) : 0.5 * (AT_(rho, i, j - 1) + AT_(rho, i, j));
    if (rho_face <= 0.0) rho_face = 1.0;
    AT_(vel, i, j) = (AT_(rhs, i, j) * dtimeb) / rho_face;
}

// VOF_DIFFUSE_compute_C_S cell loop (VOF_DIFFUSE.c:714-770), planar: every cell
// of the ghosted plane starts at 0 and takes the maximum over the particles
__global__ void k_compute_C_S(Dom d, const double *__restrict__ xc, const double *__restrict__ yc,
                              const double *__restrict__ geo, int ngeo, double shift, double denom, double extra,
                              double *__restrict__ CS)
{
    const int i = -NG + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = -NG + (int)blockIdx.y;
    if (i >= d.NX + NG || j >= d.NY + NG) return;
    const int P = d.P;
    double cs_max = 0.0;
    for (int n = 0; n < ngeo; n++) {
        const double X0 = geo[3 * n], X1 = geo[3 * n + 1], R = geo[3 * n + 2];
        const double support = R + extra;
        const double dx = xc[i] - X0, dy = yc[j] - X1;
        const double dist = sqrt(dx * dx + dy * dy);
        if (dist > support) continue;
        const double arg = (dist - (R - shift)) / (denom + 1.0e-30);
        const double cs = 0.5 - 0.5 * tanh(arg);
        if (cs > cs_max) cs_max = cs;
    }
    AT_(CS, i, j) = cs_max;
}

}  // namespace pvof
