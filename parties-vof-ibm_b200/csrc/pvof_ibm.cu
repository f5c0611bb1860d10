// Immersed-boundary routines of the diffuse-interface substep for resolved
// solid particles in the 2D modes (the reference's VOF_IBM +
// LAG_PARTICLE_RESOLVED build with TWOD_CARTESIAN: cylinders; with AXISYM_RZ:
// spheres on the symmetry axis, their markers full rings):
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
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <string>

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

// Particle_calc_derived_data (Lagrangian/Particle.c:663-733): planar
// cylinders per slab thickness; axisymmetric spheres keep the sphere's mass
// and moment of inertia, with one ring marker per ceil(pi R / h) (at least 4)
static void derived_data(IbmEntry &e, const IbmGrid &g)
{
    const double h = g.dy_min;
    const double R = e.R, R2 = R * R;
    if (g.axisym) {
        e.M = e.rho_s * 4.0 / 3.0 * IBM_PI * R2 * R;
        e.I_p = e.rho_s * 8.0 / 15.0 * IBM_PI * R2 * R2 * R;
        int N_L = (int)ceil(IBM_PI * R / h);
        e.N_L = N_L > 4 ? N_L : 4;
        e.Vol_L = 4.0 * IBM_PI * R2 * h / e.N_L;
        return;
    }
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
        // a copy carries the whole particle, its previous position shifted too
        for (const IbmEntry &p : list)
            if (p.X[axis] - p.R < lo) {
                IbmEntry c = p;
                c.X[axis] += L;
                c.X_old[axis] += L;
                c.copy = 1;
                low.push_back(c);
            }
        for (const IbmEntry &p : list)
            if (p.X[axis] + p.R > hi) {
                IbmEntry c = p;
                c.X[axis] -= L;
                c.X_old[axis] -= L;
                c.copy = 1;
                high.push_back(c);
            }
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

// Lagrangian_generate_points_2d (Lagrangian/Lagrangian.c:2900-2991): planar
// markers on the circle, line segment x slab x h each; axisymmetric markers on
// the meridian of a sphere centred on the axis, midpoints in the polar angle,
// each the spherical band 2 pi R^2 (cos theta_m - cos theta_p) times h
static void generate_points(IbmEntry &e, const IbmGrid &g, IbmMarkers &m)
{
    const double h = g.h;
    const double range = DELTA_FUNC_RADIUS * h;
    if (g.axisym) {
        const double dtheta = IBM_PI / e.N_L;
        e.moff = (int)m.x.size();
        for (int mv = 0; mv < e.N_L; mv++) {
            const double theta = (mv + 0.5) * dtheta;
            const double theta_m = mv * dtheta;
            const double theta_p = (mv + 1) * dtheta;
            const double r_ring = e.R * sin(theta);
            const double z_axial = e.X[1] + e.R * cos(theta);
            const double ring_volume = (2.0 * IBM_PI) * e.R * e.R * (cos(theta_m) - cos(theta_p)) * h;
            if (near_point(r_ring, z_axial, range, g)) {
                m.x.push_back(r_ring);
                m.y.push_back(z_axial);
                m.vol.push_back(ring_volume);
                m.flag.push_back(1);
            }
        }
        e.mcount = (int)m.x.size() - e.moff;
        return;
    }
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
        if (!g.axisym) wall(0, g.xu[0]);   // the axis is no wall (Lagrangian.c:2723)
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

void ibm_derive(IbmEntry &e, const IbmGrid &g) { derived_data(e, g); }

// cell ranges of Interpolate_integrate_momentum_twod and
// Interpolate_paint_rigid_body_velocity_twod (Lagrangian/Interpolate.c:644-800):
// u faces have cell edges at xc[i-1] and yv[j], v faces at xu[i] and yc[j-1]
void ibm_momentum_boxes(const IbmEntry &e, const IbmGrid &g, const double *xc, const double *yc, int box[2][4])
{
    const double h = g.h;
    for (int comp = 0; comp < 2; comp++) {
        const double xe0 = comp == 0 ? xc[-1] : g.xu[0];
        const double ye0 = comp == 0 ? g.yv[0] : yc[-1];
        int i_start = (int)floor((e.X[0] - e.R - xe0) / h);
        int j_start = (int)floor((e.X[1] - e.R - ye0) / h);
        int i_end = (int)ceil((e.X[0] + e.R - xe0) / h);
        int j_end = (int)ceil((e.X[1] + e.R - ye0) / h);
        i_start = std::max(i_start, 0);
        j_start = std::max(j_start, 0);
        i_end = std::min(std::min(i_end, g.NX), g.NX - 1);
        j_end = std::min(std::min(j_end, g.NY), g.NY - 1);
        box[comp][0] = i_start;
        box[comp][1] = i_end;
        box[comp][2] = j_start;
        box[comp][3] = j_end;
    }
}

// Particle_list_remove (Lagrangian/Particle.c:991-1090), 2D: a centre outside
// [xu[0], xu[NX-1]) x [yv[0], yv[NY-1]) belongs to a periodic copy
static bool outside(const IbmEntry &p, const IbmGrid &g)
{
    return p.X[0] < g.xu[0] || p.X[0] >= g.xu[g.NX - 1] || p.X[1] < g.yv[0] || p.X[1] >= g.yv[g.NY - 1];
}

std::vector<IbmEntry> ibm_collect(const std::vector<IbmEntry> &both, const IbmGrid &g)
{
    std::vector<IbmEntry> local;
    std::vector<const IbmEntry *> foreign;
    for (const IbmEntry &p : both) {
        if (outside(p, g)) foreign.push_back(&p);
        else local.push_back(p);
    }
    for (IbmEntry &p : local) {
        p.copy = 0;
        for (const IbmEntry *pf : foreign) {
            if (pf->id != p.id) continue;
            for (int i = 0; i < 3; i++) p.F[i] += pf->F[i];
            for (int i = 0; i < 3; i++) p.T[i] += pf->T[i];
            for (int i = 0; i < 3; i++) p.F_CCF[i] += pf->F_CCF[i];
            for (int i = 0; i < 3; i++) p.T_CCF[i] += pf->T_CCF[i];
            for (int i = 0; i < 3; i++) p.Int_U[i] += pf->Int_U[i];
            for (int i = 0; i < 3; i++) p.Int_Omega[i] += pf->Int_Omega[i];
        }
    }
    return local;
}

namespace {

// RK3 coefficients (Include/definitions.h:197-204)
const double RK_BET[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
const double RK_GAM[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double RK_ZET[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

// Lagrangian_apply_twod_particle_constraints (Lagrangian/Lagrangian.c:105-129):
// planar cylinders keep the spin about z only; axisymmetric spheres stay on
// the axis and do not rotate
void twod_constraints(IbmEntry &p, double zs, bool axisym)
{
    p.X[2] = zs;
    p.X_old[2] = p.X[2];
    p.U[2] = 0.0;
    p.U_old[2] = 0.0;
    if (axisym) {
        p.X[0] = 0.0;
        p.X_old[0] = 0.0;
        p.U[0] = 0.0;
        p.U_old[0] = 0.0;
        for (int i = 0; i < 3; i++) p.Omega[i] = 0.0;
        for (int i = 0; i < 3; i++) p.Omega_old[i] = 0.0;
        return;
    }
    p.Omega[0] = 0.0;
    p.Omega[1] = 0.0;
    p.Omega_old[0] = 0.0;
    p.Omega_old[1] = 0.0;
}

// The ranges at which Collision_particle / Collision_wall
// (Lagrangian/Collision.c:277-720) start to act: contact, or a surface gap
// within lub_range * h (LUBRICATION_NORMAL).  Returns false if any pair or
// wall is that close.
bool out_of_contact(const std::vector<IbmEntry> &mob_both, const std::vector<IbmEntry> &fix_both, const IbmGrid &g,
                    std::string &err)
{
    const double range = LUB_RANGE * g.h;
    char msg[256];
    for (size_t a = 0; a < mob_both.size(); a++) {
        const IbmEntry &p = mob_both[a];
        auto check = [&](const IbmEntry &q) {
            if (q.id == p.id) return true;
            const double c = p.R + q.R + range;
            const double d0 = p.X[0] - q.X[0], d1 = p.X[1] - q.X[1];
            if (d0 * d0 + d1 * d1 <= c * c) {
                snprintf(msg, sizeof(msg),
                         "particles %d and %d within the lubrication range: the collision models are not built", p.id,
                         q.id);
                err = msg;
                return false;
            }
            return true;
        };
        for (size_t b = 0; b < mob_both.size(); b++)
            if (!check(mob_both[b])) return false;
        for (const IbmEntry &q : fix_both)
            if (!check(q)) return false;
        for (int axis = 0; axis < 2; axis++) {
            if (g.periodic[axis]) continue;
            const double lo = axis == 0 ? g.xu[0] : g.yv[0];
            const double hi = axis == 0 ? g.xu[g.NX - 1] : g.yv[g.NY - 1];
            if (fabs(p.X[axis] - lo) - p.R <= range || fabs(hi - p.X[axis]) - p.R <= range) {
                snprintf(msg, sizeof(msg),
                         "particle %d within the lubrication range of a wall: the collision models are not built",
                         p.id);
                err = msg;
                return false;
            }
        }
    }
    return true;
}

// the list updates and removals around Collision_evaluate
// (Lagrangian/Lagrangian.c:1291-1303): copies across the periodic
// boundaries, then the entries whose centre is in the domain, so a particle
// that left through one side continues as its copy from the other
bool relist(std::vector<IbmEntry> &mobile, std::vector<IbmEntry> &fixed, const IbmGrid &g, double Cn, std::string &err)
{
    std::vector<IbmEntry> mob = update_list(mobile, g, Cn), fix = update_list(fixed, g, Cn);
    if (!out_of_contact(mob, fix, g, err)) return false;
    mobile.clear();
    for (const IbmEntry &p : mob)
        if (!outside(p, g)) mobile.push_back(p);
    fixed.clear();
    for (const IbmEntry &p : fix)
        if (!outside(p, g)) fixed.push_back(p);
    for (IbmEntry &p : mobile) p.copy = 0;
    for (IbmEntry &p : fixed) p.copy = 0;
    return true;
}

}  // namespace

bool ibm_advance(std::vector<IbmEntry> &mobile, std::vector<IbmEntry> &fixed, const IbmGrid &g, double Cn, int stage,
                 double dt, const double grav[3], std::string &err)
{
    // Lagrangian_evaluate_fluid_forces (Lagrangian/Lagrangian.c:338-957), after
    // the hydrodynamic collection; the diagnostic accumulators (F_IBM, F_rigid,
    // F_CCF_cum, ...) change nothing downstream and are not kept
    const double bt = RK_BET[stage];
    const double idt2beta = 1.0 / (2.0 * bt * dt);
    // axisymmetric: markers are full rings, so on an on-axis sphere the radial
    // and azimuthal components and every torque cancel (Lagrangian.c:525-543,
    // :819-837); only the axial force moves it
    if (g.axisym)
        for (std::vector<IbmEntry> *l : {&mobile, &fixed})
            for (IbmEntry &p : *l) {
                p.F[0] = 0.0;
                p.F[2] = 0.0;
                for (int i = 0; i < 3; i++) p.T[i] = 0.0;
                p.Int_U[0] = 0.0;
                p.Int_U[2] = 0.0;
                for (int i = 0; i < 3; i++) p.Int_Omega[i] = 0.0;
                p.F_CCF[0] = 0.0;
                p.F_CCF[2] = 0.0;
                for (int i = 0; i < 3; i++) p.T_CCF[i] = 0.0;
            }
    for (IbmEntry &p : mobile) {
        const double int_rho = (p.rho_s > 0.0) ? p.M / p.rho_s : 0.0;   // Lagrangian_set_exact_solid_body_mass
        for (int i = 0; i < 3; i++) p.F[i] += p.F_CCF[i];
        for (int i = 0; i < 3; i++) p.T[i] += p.T_CCF[i];
        for (int i = 0; i < 3; i++) p.F[i] += idt2beta * (p.Int_U[i] - p.Int_U_old[i]);
        for (int i = 0; i < 3; i++) p.T[i] += idt2beta * (p.Int_Omega[i] - p.Int_Omega_old[i]);
        for (int i = 0; i < 3; i++) p.Int_U_old[i] = p.Int_U[i];
        for (int i = 0; i < 3; i++) p.Int_Omega_old[i] = p.Int_Omega[i];
        for (int i = 0; i < 3; i++) p.F[i] += (p.M - int_rho) * grav[i];
    }
    for (IbmEntry &p : fixed) {
        const double int_rho = (p.rho_s > 0.0) ? p.M / p.rho_s : 0.0;
        for (int i = 0; i < 3; i++) p.F[i] += p.F_CCF[i];
        for (int i = 0; i < 3; i++) p.T[i] += p.T_CCF[i];
        for (int i = 0; i < 3; i++) p.Int_U_old[i] = p.Int_U[i];
        for (int i = 0; i < 3; i++) p.Int_Omega_old[i] = p.Int_Omega[i];
        for (int i = 0; i < 3; i++) p.F[i] += (p.M - int_rho) * grav[i];
    }
    // SUBSTEP (Lagrangian.c:293-318): 8, 2, 5 particle steps of dt / 15 per
    // fluid stage, each a full RK3 of Lagrangian_integrate_particle_motion
    // (Lagrangian.c:967-1640).  Out of contact range the collision forces and
    // torques Fc, Tc are zero; the fixed particles keep their place.
    const int nsub[3] = {8, 2, 5};
    const double dts = dt / 15.0;
    const double zs = mobile.empty() ? 0.0 : mobile[0].X[2];
    for (int n = 0; n < nsub[stage]; n++)
        for (int rk = 0; rk < 3; rk++) {
            const double b = RK_BET[rk], gm = RK_GAM[rk], zt = RK_ZET[rk];
            const double Fc = 0.0, Fc_old = 0.0;
            for (IbmEntry &p : mobile) {   // predictor
                const double dt_iM = dts / p.M, dt_iI = dts / p.I_p;
                for (int i = 0; i < 3; i++) p.X_old[i] = p.X[i];
                for (int i = 0; i < 3; i++) p.U_old[i] = p.U[i];
                for (int i = 0; i < 3; i++) p.U[i] = p.U_old[i] + dt_iM * (2.0 * b * p.F[i] + gm * Fc + zt * Fc_old);
                for (int i = 0; i < 3; i++) p.Omega_old[i] = p.Omega[i];
                for (int i = 0; i < 3; i++)
                    p.Omega[i] = p.Omega_old[i] + dt_iI * (2.0 * b * p.T[i] + gm * Fc + zt * Fc_old);
                for (int i = 0; i < 3; i++) p.X[i] = p.X_old[i] + dts * b * (p.U[i] + p.U_old[i]);
                twod_constraints(p, zs, g.axisym != 0);
            }
            if (!relist(mobile, fixed, g, Cn, err)) return false;
            for (IbmEntry &p : mobile) {   // corrector
                const double dt_iM = dts / p.M, dt_iI = dts / p.I_p;
                for (int i = 0; i < 3; i++) p.U[i] = p.U_old[i] + dt_iM * b * (2.0 * p.F[i] + Fc + Fc_old);
                for (int i = 0; i < 3; i++) p.Omega[i] = p.Omega_old[i] + dt_iI * b * (2.0 * p.T[i] + Fc + Fc_old);
                for (int i = 0; i < 3; i++) p.X[i] = p.X_old[i] + dts * b * (p.U[i] + p.U_old[i]);
                twod_constraints(p, zs, g.axisym != 0);
            }
        }
    return true;
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

// Interpolate_axis_index_for_sample / _for_spread (Interpolate.c:334-388):
// across the symmetry axis (axis == IBM_AXIS_ODD for u faces, radial parity
// odd; IBM_AXIS_EVEN for every other quantity) an index left of the axis
// folds back onto its mirror cell, u with the sign flipped; the u face on the
// axis itself maps to -1.  axis == IBM_AXIS_NONE: the identity.
__device__ __forceinline__ int axis_fold(int i, int axis, int &sign)
{
    sign = 1;
    if (axis == IBM_AXIS_NONE) return i;
    if (i < 0) {
        if (axis == IBM_AXIS_ODD) {
            sign = -1;
            return -i;
        }
        return -1 - i;
    }
    if (axis == IBM_AXIS_ODD && i == 0) return -1;
    return i;
}

// Interpolate_Eul_to_Lag_twod (Interpolate.c:477-529): one marker per thread
__global__ void k_ibm_interp(Dom d, const double *__restrict__ a, const double *__restrict__ xs,
                             const double *__restrict__ ys, double h, const double *__restrict__ XL,
                             const double *__restrict__ YL, int nm, int axis, double *__restrict__ out)
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
            int parity;
            const int ii = axis_fold(i, axis, parity);
            if (ii < -NG || ii >= d.NX + NG) continue;
            const double r0 = XL[m] - xs[i];
            A += parity * AT_(a, ii, j) * (ibm_delta(r0 / h) * ibm_delta(r1 / h));
        }
    }
    out[m] = A;
}

// Marker forces of one velocity component and the particle reaction force
// and torque (Lagrangian.c:2119-2170 for u, :2280-2335 for v): one block per
// particle, its markers in chunks across the threads.  Each marker's force is
// its own; its terms of the particle's force and torque go to shared memory
// and one thread adds them in marker order, as the reference does.  The lower
// corner of each marker's 3 x 3 spreading support on this component's grid is
// stored for k_ibm_spread.
__global__ void __launch_bounds__(IBM_FORCE_THREADS) k_ibm_marker_force(IbmDev D, int comp, double xs0, double ys0,
                                                                       double idt2beta, int reset)
{
    __shared__ double sh_f[IBM_FORCE_THREADS], sh_t[IBM_FORCE_THREADS];
    __shared__ int sh_ok[IBM_FORCE_THREADS];
    const int e = blockIdx.x, tid = threadIdx.x;
    const IbmEntryDev &p = D.ent[e];
    const double h = D.h;
    double *Fp = D.FT + 6 * e, *Tp = Fp + 3;
    double Fa = 0.0, Ta = 0.0;
    if (tid == 0) {
        if (reset) { Fp[0] = Fp[1] = Fp[2] = Tp[0] = Tp[1] = Tp[2] = 0.0; }
        Fa = Fp[comp];
        Ta = Tp[2];
    }
    const int end = p.moff + p.mcount;
    for (int base = p.moff; base < end; base += IBM_FORCE_THREADS) {
        const int q = base + tid;
        int ok = 0;
        if (q < end) {
            const double x = D.XL[q], y = D.YL[q];
            D.sup_i[q] = (int)round((x - xs0) / h) - 1;
            D.sup_j[q] = (int)round((y - ys0) / h) - 1;
            if (D.flag[q] == 0) {
                D.FL[q] = 0.0;
            } else {
                const double r0 = x - p.X[0], r1 = y - p.X[1], r2 = p.Zs - p.X[2];
                const double Ud = comp == 0 ? p.U[0] + p.Omega[1] * r2 - p.Omega[2] * r1
                                            : p.U[1] + p.Omega[2] * r0 - p.Omega[0] * r2;
                const double rho_L = D.rhoL[q];
                const double FL = idt2beta * (Ud - D.UL[q]);
                if (x >= D.xlo && x < D.xhi && y >= D.ylo && y < D.yhi) {   // Lagrangian_local_point_2d
                    const double M = D.vol[q];
                    sh_f[tid] = rho_L * M * FL;
                    sh_t[tid] = rho_L * M * (comp == 0 ? r1 : r0) * FL;
                    ok = 1;
                }
                D.FL[q] = FL;
            }
        }
        sh_ok[tid] = ok;
        __syncthreads();
        if (tid == 0) {
            const int n = min(IBM_FORCE_THREADS, end - base);
            for (int k = 0; k < n; k++) {
                if (!sh_ok[k]) continue;
                Fa -= sh_f[k];
                if (D.axisym) continue;   // the torque is the planar spin's only (Lagrangian.c:2157-2159)
                if (comp == 0) Ta += sh_t[k];
                else Ta -= sh_t[k];
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        Fp[comp] = Fa;
        Tp[2] = Ta;
    }
}

// Interpolate_Lag_to_Eul_uniform_twod (Interpolate.c:390-475) of every
// particle as a gather, then rhs += 2 rho_face temp per particle, in list
// order (Lagrangian.c:2176-2190, :2338-2350).  A cell takes a marker when it
// lies in the marker's 3 x 3 support (the support's corner from
// k_ibm_marker_force; the reference clips the support to the interior, which
// the cell already is); a cell outside a particle's box gets zero from it,
// which leaves its sum as it is.
// Interpolate_twod_cell_volume (Interpolate.c:288-312): the planar cell times
// the slab; in the axisymmetric mode the full ring, dx dy theta_span r with r
// the face radius for u and the cell-centre radius otherwise (xs), 2 pi times
// half a cell on the axis
__device__ __forceinline__ double ibm_cell_volume(const IbmDev &D, int comp, const double *xs, int i, int j)
{
    if (!D.axisym) return D.dxu1 * D.dyv[j] * D.slab;
    (void)comp;
    double radius = fabs(xs[i]);
    if (radius < 1.0e-14) radius = 0.5 * D.dxu1;
    double ring = D.theta_span * fabs(xs[i]);
    if (ring < 1.0e-14) ring = (2.0 * 3.14159265358979323846) * radius;
    return D.dxu1 * D.dyv[j] * ring;
}

__global__ void k_ibm_spread(Dom d, IbmDev D, int ne, int comp, const double *__restrict__ xs,
                             const double *__restrict__ ys, const double *__restrict__ rho, double *__restrict__ rhs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= d.NX || j >= d.NY) return;
    const int P = d.P;
    const double h = D.h;
    // axisymmetric: the cell also takes the supports of its mirror index left
    // of the axis, which the reference's scatter visits first (ascending i)
    const int axis = D.axisym ? (comp == 0 ? IBM_AXIS_ODD : IBM_AXIS_EVEN) : IBM_AXIS_NONE;
    const int im = axis == IBM_AXIS_ODD ? (i >= 1 ? -i : 1 << 30) : (axis == IBM_AXIS_EVEN ? -1 - i : 1 << 30);
    const bool direct = !(axis == IBM_AXIS_ODD && i == 0);   // the axis face takes nothing
    double r = 0.0;
    bool touched = false;
    for (int e = 0; e < ne; e++) {
        const IbmEntryDev &p = D.ent[e];
        if (!(i >= p.box[0] && i < p.box[1] && j >= p.box[2] && j < p.box[3])) continue;
        if (!touched) {
            r = AT_(rhs, i, j);
            touched = true;
        }
        double temp = 0.0;
        const double cellv = ibm_cell_volume(D, comp, xs, i, j);
        for (int q = p.moff; q < p.moff + p.mcount; q++) {
            if ((unsigned)(j - D.sup_j[q]) >= 3u) continue;
            const double r1 = D.YL[q] - ys[j];
            const double dV = D.vol[q] / cellv;
            if (axis != IBM_AXIS_NONE && (unsigned)(im - D.sup_i[q]) < 3u && im >= -NG) {
                const double r0 = D.XL[q] - xs[im];
                const double sgn = axis == IBM_AXIS_ODD ? -1.0 : 1.0;
                temp += sgn * D.FL[q] * (ibm_delta(r0 / h) * ibm_delta(r1 / h)) * dV;
            }
            if (!direct || (unsigned)(i - D.sup_i[q]) >= 3u) continue;
            const double r0 = D.XL[q] - xs[i];
            temp += 1 * D.FL[q] * (ibm_delta(r0 / h) * ibm_delta(r1 / h)) * dV;
        }
        const double rho_face = comp == 0 ? 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j))
                                          : 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
        r += 2.0 * rho_face * temp;
    }
    if (touched) AT_(rhs, i, j) = r;
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

// Interpolate_twod_level_set (Interpolate.c:314-320)
__device__ __forceinline__ double twod_level_set(double x, double y, double X0, double X1, double R)
{
    return sqrt((x - X0) * (x - X0) + (y - X1) * (y - X1)) / R - 1.0;
}

// Interpolate_twod_volume_fraction_from_phi (Interpolate.c:531-542)
__device__ __forceinline__ double vf_from_phi(double phi00, double phi10, double phi01, double phi11)
{
    double vf_cell = 0.0;
    const double sum_phi = fabs(phi00) + fabs(phi10) + fabs(phi01) + fabs(phi11);
    if (phi00 < 0.0) vf_cell -= phi00;
    if (phi10 < 0.0) vf_cell -= phi10;
    if (phi01 < 0.0) vf_cell -= phi01;
    if (phi11 < 0.0) vf_cell -= phi11;
    return (sum_phi > 0.0) ? vf_cell / sum_phi : 0.0;
}

// solid fraction of face cell (i, j) of component comp from the level set at
// its corners: u faces have corners at (xc[i-1..i], yv[j..j+1]), v faces at
// (xu[i..i+1], yc[j-1..j]) (Interpolate.c:690-706)
__device__ __forceinline__ double face_solid_fraction(int comp, int i, int j, double X0, double X1, double R,
                                                      const double *xu, const double *xc, const double *yv,
                                                      const double *yc)
{
    const double xa = comp == 0 ? xc[i - 1] : xu[i], xb = comp == 0 ? xc[i] : xu[i + 1];
    const double ya = comp == 0 ? yv[j] : yc[j - 1], yb = comp == 0 ? yv[j + 1] : yc[j];
    const double p00 = twod_level_set(xa, ya, X0, X1, R), p01 = twod_level_set(xb, ya, X0, X1, R);
    const double p10 = twod_level_set(xa, yb, X0, X1, R), p11 = twod_level_set(xb, yb, X0, X1, R);
    return vf_from_phi(p00, p01, p10, p11);
}

// mcl_particle_owns_diffuse_support (Eulerian/VOF_IBM_wetting.c:72-116): the
// entry with ID `id` has the smallest surface gap among the list entries
// whose support reaches (x, y), ties to the lower ID
__device__ __forceinline__ bool owns_support(const double *plist, int np, double id, double x, double y,
                                             double support_width)
{
    double best_gap = DBL_MAX, best_id = id;
    bool found = false;
    for (int q = 0; q < np; q++) {
        const double *pq = plist + 4 * q;
        const double support = pq[2] + support_width;
        const double dx = x - pq[0], dy = y - pq[1], dz = 0.0;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 > support * support) continue;
        const double gap = sqrt(d2) - pq[2];
        if (!found || gap < best_gap - 1.0e-12 || (fabs(gap - best_gap) <= 1.0e-12 && pq[3] < best_id)) {
            best_gap = gap;
            best_id = pq[3];
            found = true;
        }
    }
    return !found || best_id == id;
}

// One block per list entry, at the end of a substep:
//   Interpolate_integrate_momentum_twod (Interpolate.c:644-725) of u and v:
//     Int_U[c] = sum vf * vel * dV, Int_Omega[2] = -sum_u dP r_y + sum_v dP r_x
//   VOF_accumulate_solid_capillary_force (Eulerian/VOF_IBM_wetting.c:198-372),
//     Washino's contact-line force sigma t_c (grad C_L . t_s)(grad C_S . n_s)
//     over the cells of every G-range k plane within R + support of the centre
//     that the entry owns; F_CCF and T_CCF[2]
// The sums run as block reductions in a fixed order (run to run
// reproducible); the reference adds the cells one by one, so the sums agree
// to rounding.
__global__ void __launch_bounds__(256) k_ibm_particle_sums(Dom d, IbmSumArgs A)
{
    const IbmEntryDev &E = A.ent[blockIdx.x];
    const double X0 = E.X[0], X1 = E.X[1], R = E.R;
    const int P = d.P;
    double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int comp = 0; comp < 2; comp++) {
        const int *b = E.mbox[comp];
        const int w = b[1] - b[0], hgt = b[3] - b[2];
        if (w <= 0 || hgt <= 0) continue;
        const double *vel = comp == 0 ? A.U : A.V;
        const double *xn = comp == 0 ? A.xu : A.xc, *yn = comp == 0 ? A.yc : A.yv;
        for (int t = threadIdx.x; t < w * hgt; t += blockDim.x) {
            const int i = b[0] + t % w, j = b[2] + t / w;
            const double vf = face_solid_fraction(comp, i, j, X0, X1, R, A.xu, A.xc, A.yv, A.yc);
            double ring = A.slab;   // Interpolate_twod_cell_volume: slab, or the ring at the face radius
            if (A.axisym) {
                double radius = fabs(xn[i]);
                if (radius < 1.0e-14) radius = 0.5 * A.h;
                ring = A.theta_span * fabs(xn[i]);
                if (ring < 1.0e-14) ring = (2.0 * 3.14159265358979323846) * radius;
            }
            const double dV = A.h * d.m.dy_v[j] * ring;
            const double dP = vf * AT_(vel, i, j) * dV;
            acc[comp] += dP;
            if (comp == 0) acc[2] += dP * (yn[j] - X1);
            else acc[3] += dP * (xn[i] - X0);
        }
    }
    if (A.ccf) {
        const double sr = R + A.support_width, sr2 = sr * sr;
        const double hx = A.xc[1] - A.xc[0], hy = A.yc[1] - A.yc[0];
        const int i0 = max(0, (int)floor((X0 - sr - A.xc[0]) / hx) - 1);
        const int i1 = min(d.NX, (int)ceil((X0 + sr - A.xc[0]) / hx) + 2);
        const int j0 = max(0, (int)floor((X1 - sr - A.yc[0]) / hy) - 1);
        const int j1 = min(d.NY, (int)ceil((X1 + sr - A.yc[0]) / hy) + 2);
        const int w = i1 - i0, hgt = j1 - j0;
        const int ncell = (w > 0 && hgt > 0) ? w * hgt : 0;
        const double eps = 1.0e-14;
        for (int t = threadIdx.x; t < ncell * A.nk; t += blockDim.x) {
            const int c = t % ncell;
            const int i = i0 + c % w, j = j0 + c / w;
            const double r0 = A.xc[i] - X0, r1 = A.yc[j] - X1, r2 = 0.0;
            const double dist2 = r0 * r0 + r1 * r1 + r2 * r2;
            if (dist2 > sr2) continue;
            if (!owns_support(A.plist, A.np, E.id, A.xc[i], A.yc[j], A.support_width)) continue;
            const double i2dx = 1.0 / (A.xc[i + 1] - A.xc[i - 1]), i2dy = 1.0 / (A.yc[j + 1] - A.yc[j - 1]);
            const double gl[3] = {(AT_(A.CL, i + 1, j) - AT_(A.CL, i - 1, j)) * i2dx,
                                  (AT_(A.CL, i, j + 1) - AT_(A.CL, i, j - 1)) * i2dy, 0.0};
            const double gs[3] = {(AT_(A.CS, i + 1, j) - AT_(A.CS, i - 1, j)) * i2dx,
                                  (AT_(A.CS, i, j + 1) - AT_(A.CS, i, j - 1)) * i2dy, 0.0};
            const double mag_l = sqrt(gl[0] * gl[0] + gl[1] * gl[1] + gl[2] * gl[2]);
            const double mag_s = sqrt(gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2]);
            if (mag_l < eps || mag_s < eps) continue;
            const double ns[3] = {gs[0] / mag_s, gs[1] / mag_s, gs[2] / mag_s};
            const double gl_ns = gl[0] * ns[0] + gl[1] * ns[1] + gl[2] * ns[2];
            double ts[3] = {gl[0] - gl_ns * ns[0], gl[1] - gl_ns * ns[1], gl[2] - gl_ns * ns[2]};
            const double ts_len = sqrt(ts[0] * ts[0] + ts[1] * ts[1] + ts[2] * ts[2]);
            if (ts_len < eps) continue;
            ts[0] /= ts_len;
            ts[1] /= ts_len;
            ts[2] /= ts_len;
            double tc[3] = {A.ct * ts[0] - A.st * ns[0], A.ct * ts[1] - A.st * ns[1], A.ct * ts[2] - A.st * ns[2]};
            const double tc_len = sqrt(tc[0] * tc[0] + tc[1] * tc[1] + tc[2] * tc[2]);
            if (tc_len < eps) continue;
            tc[0] /= tc_len;
            tc[1] /= tc_len;
            const double term_l = gl[0] * ts[0] + gl[1] * ts[1] + gl[2] * ts[2];
            const double term_s = gs[0] * ns[0] + gs[1] * ns[1] + gs[2] * ns[2];
            const double f0 = A.sigma * term_l * term_s * tc[0], f1 = A.sigma * term_l * term_s * tc[1];
            // TwodOps_cell_measure_c (TwodOps.c:326-347)
            const double dV = A.axisym ? d.m.dx_u[i] * d.m.dy_v[j] * d.m.ring_wt_c[i]
                                       : d.m.dx_u[i] * d.m.dy_v[j] * A.slab;
            const double dF0 = f0 * dV, dF1 = f1 * dV;
            acc[4] += dF0;
            acc[5] += dF1;
            acc[6] += (dF0 * r1 - dF1 * r0);
        }
    }
    // block reduction: warps, then the warp totals
    __shared__ double red[8][7];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 7; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int k = threadIdx.x;
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += red[q][k];
        red[0][k] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double *o = A.out + 6 * blockIdx.x;
        o[0] = red[0][0];
        o[1] = red[0][1];
        o[2] = (0.0 - red[0][2]) + red[0][3];
        o[3] = red[0][4];
        o[4] = red[0][5];
        o[5] = red[0][6];
    }
}

// Interpolate_paint_rigid_body_velocity_twod (Interpolate.c:734-800) of one
// entry: vel = vf (U + Omega_z x r) + (1 - vf) vel on the face cells it covers
__global__ void k_ibm_paint(Dom d, IbmEntryDev e, int comp, const double *__restrict__ xu,
                            const double *__restrict__ xc, const double *__restrict__ yv,
                            const double *__restrict__ yc, double *__restrict__ vel)
{
    const int *b = e.mbox[comp];
    const int i = b[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = b[2] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    if (i >= b[1] || j >= b[3]) return;
    const double X0 = e.X[0], X1 = e.X[1];
    const double vf = face_solid_fraction(comp, i, j, X0, X1, e.R, xu, xc, yv, yc);
    if (vf <= 0.0) return;
    const int P = d.P;
    const double om = e.Omega[2];
    const double u_rigid = comp == 0 ? e.U[0] - om * (yc[j] - X1) : e.U[1] + om * (xc[i] - X0);
    AT_(vel, i, j) = vf * u_rigid + (1.0 - vf) * AT_(vel, i, j);
}

}  // namespace pvof
