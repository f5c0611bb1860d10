// Device-resident particle bookkeeping of the resolved-solid substep: the
// particle lists and their periodic copies, the markers and their flags, and
// the rigid-body motion live in device memory, so a substep with resolved
// particles needs no host round trip and replays from a CUDA graph like the
// plain one.
//
//   Particle_MPI_update on one rank          ps_update_list (periodic copies,
//                                            Lagrangian/Particle.c:2042-2500)
//   Lagrangian_flag_points,                  k_ps_markers (Lagrangian/Lagrangian.c:2515-2800,
//   Lagrangian_generate_points_2d            :2900-2991)
//   Lagrangian_collect_forces,               ps_collect, ps_advance
//   Lagrangian_evaluate_fluid_forces and the (Lagrangian.c:283-1640)
//   substepped rigid-body motion
//
// The list logic runs in one device thread (a handful of particles).  It is
// written once, as host-and-device functions, in the order of the reference's
// list operations, so the markers and sums are the reference's to the last
// bit (the library is compiled without FMA contraction, so device arithmetic
// rounds like the host's).  The unit-circle tables of the markers (cos and
// sin of the marker angles, and the ring volumes) are computed on the host
// once per particle, so the marker positions round like the reference's.
#pragma once

#include "pvof_kernels.cuh"

namespace pvof {

constexpr double PS_PI = 3.14159265358979323846;   // PI, Include/definitions.h:7
constexpr double PS_DELTA_FUNC_RADIUS = 1.5;       // Include/definitions.h:58
constexpr double PS_LAG_FLAG_RANGE = 3.0;          // Include/definitions.h:61
constexpr double PS_LUB_RANGE = 2.0;               // [particle] lub_range default (IO/default.inp)
constexpr int PS_TRIG = 4;                         // table doubles per marker: two unit components, volume, pad

// one particle: an owned one, or a list entry after an update (an owned
// particle or one of its periodic copies)
struct PEnt {
    int mobile, id, copy;
    int N_L;                  // markers of the whole circle (planar) or meridian (axisymmetric)
    int moff, mcount;         // this entry's markers near the domain
    int box[4];               // cells [i0, i1) x [j0, j1) its marker supports can reach
    int mbox[2][4];           // cells of Interpolate_integrate_momentum_twod for u and v
    double X[3], U[3], Omega[3], R, rho_s;
    double M, I_p, Vol_L;     // Particle_calc_derived_data
    // rigid-body state (the Particle fields of Include/DataTypes.h:1327-1527
    // that the motion of a cylinder reads)
    double X_old[3], U_old[3], Omega_old[3];
    double Int_U[3], Int_Omega[3], Int_U_old[3], Int_Omega_old[3];
    double F[3], T[3], F_CCF[3], T_CCF[3];
};

// the grid data the bookkeeping reads
struct PGrid {
    int NX, NY;
    int periodic[2];
    int axisym;                      // AXISYM_RZ: spheres on the axis, ring markers
    double h, dy_min, Lx, Ly, Cn, zs;
    double slab, twod_slab;          // the plane's slab thickness and the configured one (host use)
    double xu0, xuN, yv0, yvN;       // xu[0], xu[NX-1], yv[0], yv[NY-1]
    double xcm1, ycm1;               // xc[-1], yc[-1]: the momentum boxes' u and v cell edges
    double grav[3];
};

// The particle state of a context.  One copy lives in device memory (the
// kernels read and write its counts); the host keeps one with the same
// pointers and capacities.
struct PSet {
    int nmob, nfix;           // owned particles, list order
    int ne;                   // list entries after the last update (mobile first)
    int nm;                   // markers of the entries
    int np;                   // entries of the contact-line particle list
    int ngeo;                 // particles of the solid-fraction field
    int err;                  // 1: within the lubrication range; 2: a list beyond its capacity
    int err_a, err_b;         // the IDs of err 1 (err_b -1: a wall)
    int cap_own, cap_ent, cap_mk;
    PEnt *mob, *fix;          // owned lists [cap_own] each
    PEnt *ent;                // entries [cap_ent]
    PEnt *tmp;                // scratch of the list updates [3 cap_ent]
    IbmEntryDev *dent;        // the entries as the force and sum kernels read them [cap_ent]
    double *mk;               // markers: x, y, vol, UL, rhoL, FL, each [cap_mk]
    int *mflag;               // flag, support corner i, j, owning entry, each [cap_mk]
    const double *trig;       // marker tables, PS_TRIG doubles per marker, particle after particle by ID
    const int *trig_off;      // first marker of each ID in trig
    double *plist;            // x, y, R, ID per contact-line list entry [cap_ent]
    double *geo;              // x, y, R of the solid-fraction particles [3 cap_own]
    double *FT;               // F[3], T[3] per entry (Lagrangian_force)
    double *sums;             // k_ibm_particle_sums, 6 per entry
    PGrid g;
};

// Particle_ibm_exchange_range (Lagrangian/Particle.c:26-47) plus the marker-flag
// and lubrication ranges added in Particle_MPI_update (:2052-2060)
__host__ __device__ inline double ps_exchange_range(const PGrid &g)
{
    const double h = g.h;
    double range = PS_DELTA_FUNC_RADIUS * h;
    const double h_ref = (g.dy_min > 0.0) ? g.dy_min : h;
    const double cn = (g.Cn > 0.0) ? g.Cn : 0.0;
    const double wetting = 8.0 * ((cn > h_ref) ? cn : h_ref);
    if (wetting > range) range = wetting;
    range += PS_LAG_FLAG_RANGE * h;
    const double lub = 0.5 * PS_LUB_RANGE * h;
    return range > lub ? range : lub;
}

// One list of Particle_MPI_update on a single rank: in[0..n) -> out with the
// periodic copies prepended in the order the exchanges add them (per
// periodic axis: the copies shifted down, the copies shifted up, then the
// list).  A copy carries the whole particle, its previous position shifted
// too.  work: room for cap entries, distinct from in and out.  Returns the
// new count, or -1 when cap is too small.
__host__ __device__ inline int ps_update_list(const PEnt *in, int n, PEnt *out, PEnt *work, int cap, const PGrid &g)
{
    const double range = ps_exchange_range(g);
    const PEnt *src = in;
    int ns = n;
    PEnt *dst = work;
    for (int axis = 0; axis < 2; axis++) {
        if (!g.periodic[axis]) continue;
        const double lo = (axis == 0 ? g.xu0 : g.yv0) + range;
        const double hi = (axis == 0 ? g.xuN : g.yvN) - range;
        const double L = axis == 0 ? g.Lx : g.Ly;
        int k = 0;
        for (int q = 0; q < ns; q++)
            if (src[q].X[axis] + src[q].R > hi) {
                if (k >= cap) return -1;
                dst[k] = src[q];
                dst[k].X[axis] -= L;
                dst[k].X_old[axis] -= L;
                dst[k].copy = 1;
                k++;
            }
        for (int q = 0; q < ns; q++)
            if (src[q].X[axis] - src[q].R < lo) {
                if (k >= cap) return -1;
                dst[k] = src[q];
                dst[k].X[axis] += L;
                dst[k].X_old[axis] += L;
                dst[k].copy = 1;
                k++;
            }
        for (int q = 0; q < ns; q++) {
            if (k >= cap) return -1;
            dst[k++] = src[q];
        }
        src = dst;
        ns = k;
        dst = (dst == work) ? out : work;
    }
    if (ns > cap) return -1;
    if (src != out)
        for (int q = 0; q < ns; q++) out[q] = src[q];
    return ns;
}

// Particle_list_remove (Lagrangian/Particle.c:991-1090), 2D: a centre outside
// [xu[0], xu[NX-1]) x [yv[0], yv[NY-1]) belongs to a periodic copy
__host__ __device__ inline bool ps_outside(const PEnt &p, const PGrid &g)
{
    return p.X[0] < g.xu0 || p.X[0] >= g.xuN || p.X[1] < g.yv0 || p.X[1] >= g.yvN;
}

// Lagrangian_near_point_2d (Lagrangian/Lagrangian.c:86-96)
__host__ __device__ inline bool ps_near_point(double x, double y, double range, const PGrid &g)
{
    return g.xu0 - x < range && x - g.xuN < range && g.yv0 - y < range && y - g.yvN < range;
}

// Lagrangian_collect_forces (LAG_COLLECT_HYDRO) after
// Particle_list_foreign_create: the entries of a list whose centre lies in
// the domain, in order, each with the F, T, capillary and momentum sums of the
// out-of-domain entries of its ID added.  At most cap are kept; returns the
// count, or -1 beyond cap.
__host__ __device__ inline int ps_collect(const PEnt *both, int n, PEnt *local, int cap, const PGrid &g)
{
    int k = 0;
    for (int q = 0; q < n; q++) {
        if (ps_outside(both[q], g)) continue;
        if (k >= cap) return -1;
        PEnt &p = local[k++];
        p = both[q];
        p.copy = 0;
        for (int f = 0; f < n; f++) {
            const PEnt &pf = both[f];
            if (!ps_outside(pf, g) || pf.id != p.id) continue;
            for (int i = 0; i < 3; i++) p.F[i] += pf.F[i];
            for (int i = 0; i < 3; i++) p.T[i] += pf.T[i];
            for (int i = 0; i < 3; i++) p.F_CCF[i] += pf.F_CCF[i];
            for (int i = 0; i < 3; i++) p.T_CCF[i] += pf.T_CCF[i];
            for (int i = 0; i < 3; i++) p.Int_U[i] += pf.Int_U[i];
            for (int i = 0; i < 3; i++) p.Int_Omega[i] += pf.Int_Omega[i];
        }
    }
    return k;
}

// cell ranges of Interpolate_integrate_momentum_twod and
// Interpolate_paint_rigid_body_velocity_twod (Lagrangian/Interpolate.c:644-800):
// u faces have cell edges at xc[i-1] and yv[j], v faces at xu[i] and yc[j-1]
__host__ __device__ inline void ps_momentum_boxes(PEnt &e, const PGrid &g)
{
    const double h = g.h;
    for (int comp = 0; comp < 2; comp++) {
        const double xe0 = comp == 0 ? g.xcm1 : g.xu0;
        const double ye0 = comp == 0 ? g.yv0 : g.ycm1;
        int i_start = (int)floor((e.X[0] - e.R - xe0) / h);
        int j_start = (int)floor((e.X[1] - e.R - ye0) / h);
        int i_end = (int)ceil((e.X[0] + e.R - xe0) / h);
        int j_end = (int)ceil((e.X[1] + e.R - ye0) / h);
        i_start = i_start > 0 ? i_start : 0;
        j_start = j_start > 0 ? j_start : 0;
        i_end = i_end < g.NX ? i_end : g.NX;
        i_end = i_end < g.NX - 1 ? i_end : g.NX - 1;
        j_end = j_end < g.NY ? j_end : g.NY;
        j_end = j_end < g.NY - 1 ? j_end : g.NY - 1;
        e.mbox[comp][0] = i_start;
        e.mbox[comp][1] = i_end;
        e.mbox[comp][2] = j_start;
        e.mbox[comp][3] = j_end;
    }
}

// RK3 coefficients (Include/definitions.h:197-204)
__host__ __device__ inline double ps_bet(int s) { return s == 0 ? 4.0 / 15.0 : (s == 1 ? 1.0 / 15.0 : 1.0 / 6.0); }
__host__ __device__ inline double ps_gam(int s) { return s == 0 ? 8.0 / 15.0 : (s == 1 ? 5.0 / 12.0 : 3.0 / 4.0); }
__host__ __device__ inline double ps_zet(int s) { return s == 0 ? 0.0 : (s == 1 ? -17.0 / 60.0 : -5.0 / 12.0); }

// Lagrangian_apply_twod_particle_constraints (Lagrangian/Lagrangian.c:105-129):
// planar cylinders keep the spin about z only; axisymmetric spheres stay on
// the axis and do not rotate
__host__ __device__ inline void ps_constraints(PEnt &p, double zs, bool axisym)
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
// within lub_range * h (LUBRICATION_NORMAL).  False if any pair or wall is
// that close; who[0], who[1] the IDs (who[1] = -1: a wall).
__host__ __device__ inline bool ps_out_of_contact(const PEnt *mob, int nm, const PEnt *fix, int nf, const PGrid &g,
                                                  int *who)
{
    const double range = PS_LUB_RANGE * g.h;
    for (int a = 0; a < nm; a++) {
        const PEnt &p = mob[a];
        for (int b = 0; b < nm + nf; b++) {
            const PEnt &q = b < nm ? mob[b] : fix[b - nm];
            if (q.id == p.id) continue;
            const double c = p.R + q.R + range;
            const double d0 = p.X[0] - q.X[0], d1 = p.X[1] - q.X[1];
            if (d0 * d0 + d1 * d1 <= c * c) {
                who[0] = p.id;
                who[1] = q.id;
                return false;
            }
        }
        for (int axis = 0; axis < 2; axis++) {
            if (g.periodic[axis]) continue;
            const double lo = axis == 0 ? g.xu0 : g.yv0;
            const double hi = axis == 0 ? g.xuN : g.yvN;
            if (fabs(p.X[axis] - lo) - p.R <= range || fabs(hi - p.X[axis]) - p.R <= range) {
                who[0] = p.id;
                who[1] = -1;
                return false;
            }
        }
    }
    return true;
}

// the list updates and removals around Collision_evaluate
// (Lagrangian/Lagrangian.c:1291-1303): copies across the periodic boundaries,
// then the entries whose centre is in the domain, so a particle that left
// through one side continues as its copy from the other.  work: room for
// 3 cap entries; the owned lists hold cap_own each.  Returns 0, 1 on contact
// (who set), 2 when a list outgrows its room.
__host__ __device__ inline int ps_relist(PEnt *mob, int &nm, PEnt *fix, int &nf, PEnt *work, int cap, int cap_own,
                                         const PGrid &g, int *who)
{
    PEnt *mb = work, *fb = work + cap, *scratch = work + 2 * cap;
    const int m = ps_update_list(mob, nm, mb, scratch, cap, g);
    const int f = ps_update_list(fix, nf, fb, scratch, cap, g);
    if (m < 0 || f < 0) return 2;
    if (!ps_out_of_contact(mb, m, fb, f, g, who)) return 1;
    int k = 0;
    for (int q = 0; q < m; q++)
        if (!ps_outside(mb[q], g)) {
            if (k >= cap_own) return 2;
            mob[k] = mb[q];
            mob[k].copy = 0;
            k++;
        }
    nm = k;
    k = 0;
    for (int q = 0; q < f; q++)
        if (!ps_outside(fb[q], g)) {
            if (k >= cap_own) return 2;
            fix[k] = fb[q];
            fix[k].copy = 0;
            k++;
        }
    nf = k;
    return 0;
}

// Lagrangian_evaluate_fluid_forces (Lagrangian/Lagrangian.c:338-957), after
// the hydrodynamic collection, then SUBSTEP (Lagrangian.c:293-318): 8, 2, 5
// particle steps of dt / 15 per fluid stage, each a full RK3 of
// Lagrangian_integrate_particle_motion (Lagrangian.c:967-1640).  Out of
// contact range the collision forces and torques are zero; the fixed
// particles keep their place.  The diagnostic accumulators (F_IBM, F_rigid,
// F_CCF_cum, ...) change nothing downstream and are not kept.  Returns as
// ps_relist.
__host__ __device__ inline int ps_advance(PEnt *mob, int &nm, PEnt *fix, int &nf, PEnt *work, int cap, int cap_own,
                                          const PGrid &g, int stage, double dt, int *who)
{
    const double bt = ps_bet(stage);
    const double idt2beta = 1.0 / (2.0 * bt * dt);
    // axisymmetric: markers are full rings, so on an on-axis sphere the radial
    // and azimuthal components and every torque cancel (Lagrangian.c:525-543,
    // :819-837); only the axial force moves it
    if (g.axisym)
        for (int q = 0; q < nm + nf; q++) {
            PEnt &p = q < nm ? mob[q] : fix[q - nm];
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
    for (int q = 0; q < nm; q++) {
        PEnt &p = mob[q];
        const double int_rho = (p.rho_s > 0.0) ? p.M / p.rho_s : 0.0;   // Lagrangian_set_exact_solid_body_mass
        for (int i = 0; i < 3; i++) p.F[i] += p.F_CCF[i];
        for (int i = 0; i < 3; i++) p.T[i] += p.T_CCF[i];
        for (int i = 0; i < 3; i++) p.F[i] += idt2beta * (p.Int_U[i] - p.Int_U_old[i]);
        for (int i = 0; i < 3; i++) p.T[i] += idt2beta * (p.Int_Omega[i] - p.Int_Omega_old[i]);
        for (int i = 0; i < 3; i++) p.Int_U_old[i] = p.Int_U[i];
        for (int i = 0; i < 3; i++) p.Int_Omega_old[i] = p.Int_Omega[i];
        for (int i = 0; i < 3; i++) p.F[i] += (p.M - int_rho) * g.grav[i];
    }
    for (int q = 0; q < nf; q++) {
        PEnt &p = fix[q];
        const double int_rho = (p.rho_s > 0.0) ? p.M / p.rho_s : 0.0;
        for (int i = 0; i < 3; i++) p.F[i] += p.F_CCF[i];
        for (int i = 0; i < 3; i++) p.T[i] += p.T_CCF[i];
        for (int i = 0; i < 3; i++) p.Int_U_old[i] = p.Int_U[i];
        for (int i = 0; i < 3; i++) p.Int_Omega_old[i] = p.Int_Omega[i];
        for (int i = 0; i < 3; i++) p.F[i] += (p.M - int_rho) * g.grav[i];
    }
    const int nsub = stage == 0 ? 8 : (stage == 1 ? 2 : 5);
    const double dts = dt / 15.0;
    const double zs = nm == 0 ? 0.0 : mob[0].X[2];
    const bool axi = g.axisym != 0;
    for (int n = 0; n < nsub; n++)
        for (int rk = 0; rk < 3; rk++) {
            const double b = ps_bet(rk), gm = ps_gam(rk), zt = ps_zet(rk);
            const double Fc = 0.0, Fc_old = 0.0;
            for (int q = 0; q < nm; q++) {   // predictor
                PEnt &p = mob[q];
                const double dt_iM = dts / p.M, dt_iI = dts / p.I_p;
                for (int i = 0; i < 3; i++) p.X_old[i] = p.X[i];
                for (int i = 0; i < 3; i++) p.U_old[i] = p.U[i];
                for (int i = 0; i < 3; i++) p.U[i] = p.U_old[i] + dt_iM * (2.0 * b * p.F[i] + gm * Fc + zt * Fc_old);
                for (int i = 0; i < 3; i++) p.Omega_old[i] = p.Omega[i];
                for (int i = 0; i < 3; i++)
                    p.Omega[i] = p.Omega_old[i] + dt_iI * (2.0 * b * p.T[i] + gm * Fc + zt * Fc_old);
                for (int i = 0; i < 3; i++) p.X[i] = p.X_old[i] + dts * b * (p.U[i] + p.U_old[i]);
                ps_constraints(p, zs, axi);
            }
            const int rc = ps_relist(mob, nm, fix, nf, work, cap, cap_own, g, who);
            if (rc) return rc;
            for (int q = 0; q < nm; q++) {   // corrector
                PEnt &p = mob[q];
                const double dt_iM = dts / p.M, dt_iI = dts / p.I_p;
                for (int i = 0; i < 3; i++) p.U[i] = p.U_old[i] + dt_iM * b * (2.0 * p.F[i] + Fc + Fc_old);
                for (int i = 0; i < 3; i++) p.Omega[i] = p.Omega_old[i] + dt_iI * b * (2.0 * p.T[i] + Fc + Fc_old);
                for (int i = 0; i < 3; i++) p.X[i] = p.X_old[i] + dts * b * (p.U[i] + p.U_old[i]);
                ps_constraints(p, zs, axi);
            }
        }
    return 0;
}

// host: Particle_calc_derived_data, and a particle's marker table (pvof_ibm.cu)
void ps_derived(PEnt &e, const PGrid &g);
void ps_marker_table(const PEnt &e, const PGrid &g, std::vector<double> &tab);

// kernels of the bookkeeping (pvof_ibm.cu); ps points at the device copy
constexpr int PS_MARKER_THREADS = 1024;
// entries: the owned lists updated with their periodic copies, their
// momentum boxes, the contact-line list (one thread)
__global__ void k_ps_update(PSet *ps);
// markers, flags and boxes of the entries, the entries as the force kernels
// read them, F and T zeroed (one block of PS_MARKER_THREADS)
__global__ void k_ps_markers(PSet *ps);
// the solid-fraction particles: owned centres inside the domain (one thread)
__global__ void k_ps_geo(PSet *ps);
// the end-of-substep sums into the entries, collected into the owned lists,
// then: PS_COLLECT nothing more, PS_INIT_VELOCITY the velocities from the
// momentum integrals (Particle_initialize_velocities), PS_INIT_MOMENTUM the
// momentum integrals as the previous ones, PS_ADVANCE the rigid-body motion
// of the stage (one thread)
constexpr int PS_COLLECT = 0, PS_INIT_VELOCITY = 1, PS_INIT_MOMENTUM = 2, PS_ADVANCE = 3;
__global__ void k_ps_collect(PSet *ps, int mode, int ccf, int stage, double dt);
// Interpolate_paint_rigid_body_velocity_twod of every mobile entry, in list order
__global__ void k_ps_paint(Dom d, const PSet *ps, int comp, const double *xu, const double *xc, const double *yv,
                           const double *yc, double *vel);

}  // namespace pvof
