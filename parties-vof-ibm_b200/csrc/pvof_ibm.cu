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
// Everything runs on the device: the particle bookkeeping (lists, periodic
// copies, markers, flags, rigid-body motion; the list logic is shared with
// the host in pvof_particles.cuh) in one-thread or one-block kernels over a
// handful of particles and a few hundred markers, the gathers, the
// per-particle force and torque sums and the spreads.  Only the marker
// tables of each particle are made on the host, once.  The spread is written as a gather: each
// cell adds the contributions of a particle's markers in marker order, which
// is the order in which the reference's scatter adds them, so the result is
// the reference's to the last bit.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <string>

#include "pvof_device.cuh"
#include "pvof_particles.cuh"

namespace pvof {

constexpr double IBM_PI = PS_PI;

// ---------------------------------------------------------------------------
// host: per-particle constants
// ---------------------------------------------------------------------------

// Particle_calc_derived_data (Lagrangian/Particle.c:663-733): planar
// cylinders per slab thickness; axisymmetric spheres keep the sphere's mass
// and moment of inertia, with one ring marker per ceil(pi R / h) (at least 4)
void ps_derived(PEnt &e, const PGrid &g)
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

// The marker table of one particle for k_ps_markers, after
// Lagrangian_generate_points_2d (Lagrangian/Lagrangian.c:2900-2991): planar
// markers on the circle at the angle midpoints, (cos, sin, segment x slab x h);
// axisymmetric markers on the meridian at the polar-angle midpoints,
// (sin, cos, the spherical band 2 pi R^2 (cos theta_m - cos theta_p) times h)
void ps_marker_table(const PEnt &e, const PGrid &g, std::vector<double> &tab)
{
    const double h = g.h;
    if (g.axisym) {
        const double dtheta = IBM_PI / e.N_L;
        for (int mv = 0; mv < e.N_L; mv++) {
            const double theta = (mv + 0.5) * dtheta;
            const double theta_m = mv * dtheta;
            const double theta_p = (mv + 1) * dtheta;
            tab.push_back(sin(theta));
            tab.push_back(cos(theta));
            tab.push_back((2.0 * IBM_PI) * e.R * e.R * (cos(theta_m) - cos(theta_p)) * h);
            tab.push_back(0.0);
        }
        return;
    }
    const double dtheta = 2.0 * IBM_PI / e.N_L;
    const double ds = e.R * dtheta;
    double slab = g.slab;
    if (slab <= 0.0) slab = h;
    for (int mv = 0; mv < e.N_L; mv++) {
        const double theta = (mv + 0.5) * dtheta;
        tab.push_back(cos(theta));
        tab.push_back(sin(theta));
        tab.push_back(ds * slab * h);
        tab.push_back(0.0);
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
// device: particle bookkeeping
// ---------------------------------------------------------------------------

// Particle_MPI_update of both lists (mobile, then fixed), the entries'
// momentum boxes, and the contact-line list (mcl_nearest_particle_normal,
// VOF_IBM_wetting.c:118-182, reads the lists as they stand after the update)
__global__ void k_ps_update(PSet *ps)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PSet &S = *ps;
    const PGrid &g = S.g;
    const int m = ps_update_list(S.mob, S.nmob, S.ent, S.tmp, S.cap_ent, g);
    const int f = m < 0 ? -1 : ps_update_list(S.fix, S.nfix, S.ent + m, S.tmp, S.cap_ent - m, g);
    if (m < 0 || f < 0) {
        S.err = 2;
        S.ne = S.np = 0;
        return;
    }
    S.ne = m + f;
    for (int q = 0; q < S.ne; q++) {
        PEnt &e = S.ent[q];
        e.mobile = q < m ? 1 : 0;
        ps_momentum_boxes(e, g);
        double *pl = S.plist + 4 * q;
        pl[0] = e.X[0];
        pl[1] = e.X[1];
        pl[2] = e.R;
        pl[3] = (double)e.id;
    }
    S.np = S.ne;
}

// Lagrangian_flag_points (Lagrangian/Lagrangian.c:2515-2800) for the entries
// in list order: each entry's markers near the domain
// (Lagrangian_generate_points_2d), compacted in marker order by a block scan;
// then every marker's flag, cleared within LAG_FLAG_RANGE h of another
// particle (Lagrangian_flag_points_individual, :2629-2690) or of an x or y
// wall (Lagrangian_flag_points_wall, :2697-2795; the axis is no wall) -- the
// flags only go from 1 to 0, so the order of the tests does not matter; then
// each entry's cell box of its marker supports (3 x 3 stencils, for the
// spread) and the entry as the force kernels read it.
__global__ void __launch_bounds__(PS_MARKER_THREADS) k_ps_markers(PSet *ps)
{
    __shared__ int s_cnt[PS_MARKER_THREADS / 32];
    __shared__ int s_total, s_over;
    __shared__ int s_box[4];
    PSet &S = *ps;
    const PGrid &g = S.g;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int ne = S.ne, cap = S.cap_mk;
    double *mx = S.mk, *my = S.mk + cap, *mvol = S.mk + 2 * cap;
    int *mflag = S.mflag, *mown = S.mflag + 3 * cap;
    const double h = g.h, range = PS_DELTA_FUNC_RADIUS * h;
    if (tid == 0) s_over = 0;
    int base = 0;
    for (int e = 0; e < ne; e++) {
        const PEnt &E = S.ent[e];
        const double *tab = S.trig + (size_t)S.trig_off[E.id] * PS_TRIG;
        const int start = base;
        for (int c0 = 0; c0 < E.N_L; c0 += blockDim.x) {
            const int mv = c0 + tid;
            bool near = false;
            double x = 0.0, y = 0.0, vol = 0.0;
            if (mv < E.N_L) {
                const double *t = tab + (size_t)mv * PS_TRIG;
                x = g.axisym ? E.R * t[0] : E.X[0] + E.R * t[0];
                y = E.X[1] + E.R * t[1];
                vol = t[2];
                near = ps_near_point(x, y, range, g);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, near);
            if (lane == 0) s_cnt[warp] = __popc(bal);
            __syncthreads();
            if (tid == 0) {
                int run = 0;
                for (int w = 0; w < nw; w++) {
                    const int n = s_cnt[w];
                    s_cnt[w] = run;
                    run += n;
                }
                s_total = run;
            }
            __syncthreads();
            if (near) {
                const int pos = base + s_cnt[warp] + __popc(bal & ((1u << lane) - 1u));
                if (pos < cap) {
                    mx[pos] = x;
                    my[pos] = y;
                    mvol[pos] = vol;
                    mflag[pos] = 1;
                    mown[pos] = e;
                } else {
                    s_over = 1;
                }
            }
            base += s_total;
            __syncthreads();
        }
        if (tid == 0) {
            S.ent[e].moff = start;
            S.ent[e].mcount = base - start;
        }
    }
    __syncthreads();
    if (s_over || base > cap) {
        if (tid == 0) {
            S.err = 2;
            S.nm = 0;
            for (int e = 0; e < ne; e++) S.ent[e].mcount = 0;
        }
        base = 0;
    }
    __syncthreads();
    const int nm = base;
    for (int q = tid; q < nm; q += blockDim.x) {
        const PEnt &P = S.ent[mown[q]];
        int flag = mflag[q];
        for (int e2 = 0; e2 < ne; e2++) {
            const PEnt &P2 = S.ent[e2];
            if (P2.id == P.id) continue;
            double dpp = P.R + P2.R + PS_LAG_FLAG_RANGE * h;
            dpp = dpp * dpp;
            double dlp = P2.R + PS_LAG_FLAG_RANGE * h;
            dlp = dlp * dlp;
            double r0 = P2.X[0] - P.X[0], r1 = P2.X[1] - P.X[1];
            if (!(r0 * r0 + r1 * r1 < dpp)) continue;
            r0 = P2.X[0] - mx[q];
            r1 = P2.X[1] - my[q];
            const double d2 = r0 * r0 + r1 * r1;
            if (flag == 1 && d2 < dlp) flag = 0;
        }
        const double dpw = P.R + 0.5 * PS_LAG_FLAG_RANGE * h;
        const double dlw = 0.5 * PS_LAG_FLAG_RANGE * h;
        for (int w = 0; w < 4; w++) {
            const int axis = w >> 1;
            if (g.periodic[axis]) continue;
            if (w == 0 && g.axisym) continue;   // the axis is no wall (Lagrangian.c:2723)
            const double pos = w == 0 ? g.xu0 : (w == 1 ? g.xuN : (w == 2 ? g.yv0 : g.yvN));
            const double c = axis == 0 ? P.X[0] : P.X[1];
            if (!(fabs(c - pos) < dpw)) continue;
            const double v = axis == 0 ? mx[q] : my[q];
            if (flag == 1 && fabs(v - pos) < dlw) flag = 0;
        }
        mflag[q] = flag;
    }
    for (int e = 0; e < ne; e++) {
        if (tid == 0) {
            s_box[0] = s_box[2] = 1 << 30;
            s_box[1] = s_box[3] = -(1 << 30);
        }
        __syncthreads();
        const PEnt &E = S.ent[e];
        int b0 = 1 << 30, b1 = -(1 << 30), b2 = 1 << 30, b3 = -(1 << 30);
        for (int q = E.moff + tid; q < E.moff + E.mcount; q += blockDim.x) {
            const int i = (int)floor((mx[q] - g.xu0) / h), j = (int)floor((my[q] - g.yv0) / h);
            b0 = min(b0, i - 3);
            b1 = max(b1, i + 4);
            b2 = min(b2, j - 3);
            b3 = max(b3, j + 4);
        }
        atomicMin(&s_box[0], b0);
        atomicMax(&s_box[1], b1);
        atomicMin(&s_box[2], b2);
        atomicMax(&s_box[3], b3);
        __syncthreads();
        if (tid == 0)
            for (int k = 0; k < 4; k++) S.ent[e].box[k] = s_box[k];
        __syncthreads();
    }
    for (int e = tid; e < ne; e += blockDim.x) {
        const PEnt &E = S.ent[e];
        IbmEntryDev &o = S.dent[e];
        for (int k = 0; k < 3; k++) { o.X[k] = E.X[k]; o.U[k] = E.U[k]; o.Omega[k] = E.Omega[k]; }
        o.X[2] = g.zs;
        o.Zs = g.zs;
        o.moff = E.moff;
        o.mcount = E.mcount;
        for (int k = 0; k < 4; k++) o.box[k] = E.box[k];
        o.R = E.R;
        o.id = (double)E.id;
        for (int c = 0; c < 2; c++)
            for (int k = 0; k < 4; k++) o.mbox[c][k] = E.mbox[c][k];
        for (int k = 0; k < 6; k++) S.FT[6 * e + k] = 0.0;
    }
    if (tid == 0) S.nm = nm;
}

// VOF_DIFFUSE_compute_C_S geometry (VOF_DIFFUSE.c:57-85 through
// Particle_collect_owned_overlaps, Lagrangian/Particle.c:1697-1786): on one
// rank every particle whose centre the rank owns, unshifted -- the overlap
// test takes the first shift that overlaps and the unshifted one always does
// -- so a particle crossing a periodic boundary has no copy in C_S.  The
// maximum over particles does not depend on their order.
__global__ void k_ps_geo(PSet *ps)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PSet &S = *ps;
    const PGrid &g = S.g;
    int n = 0;
    for (int q = 0; q < S.nmob + S.nfix; q++) {
        const PEnt &p = q < S.nmob ? S.mob[q] : S.fix[q - S.nmob];
        if (!(p.X[0] >= g.xu0 && p.X[0] <= g.xuN && p.X[1] >= g.yv0 && p.X[1] <= g.yvN)) continue;
        S.geo[3 * n] = p.X[0];
        S.geo[3 * n + 1] = p.X[1];
        S.geo[3 * n + 2] = p.R;
        n++;
    }
    S.ngeo = n;
}

// The end of a substep (Temporal_int.c:1186-1238) after k_ibm_particle_sums:
// every entry takes its direct-forcing reaction (F, T of Lagrangian_force),
// its momentum integrals (Int_U[0..1], Int_Omega[2]) and, with ccf, its
// capillary contact force (F_CCF[0..1], T_CCF[2]); the two lists are
// collected into the owned particles (the mobile entries come first); then
// the mode's step.
__global__ void k_ps_collect(PSet *ps, int mode, int ccf, int stage, double dt)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PSet &S = *ps;
    const PGrid &g = S.g;
    if (S.err) return;
    const int ne = S.ne;
    int nmob_e = 0;
    for (int q = 0; q < ne; q++) {
        PEnt &e = S.ent[q];
        const double *o = S.sums + 6 * q;
        for (int k = 0; k < 3; k++) {
            e.F[k] = S.FT[6 * q + k];
            e.T[k] = S.FT[6 * q + 3 + k];
            e.Int_U[k] = e.Int_Omega[k] = e.F_CCF[k] = e.T_CCF[k] = 0.0;
        }
        e.Int_U[0] = o[0];
        e.Int_U[1] = o[1];
        e.Int_Omega[2] = o[2];
        if (ccf) {
            e.F_CCF[0] = o[3];
            e.F_CCF[1] = o[4];
            e.T_CCF[2] = o[5];
        }
        if (e.mobile) nmob_e = q + 1;
    }
    const int m = ps_collect(S.ent, nmob_e, S.mob, S.cap_own, g);
    const int f = ps_collect(S.ent + nmob_e, ne - nmob_e, S.fix, S.cap_own, g);
    if (m < 0 || f < 0) {
        S.err = 2;
        return;
    }
    S.nmob = m;
    S.nfix = f;
    if (mode == PS_INIT_VELOCITY) {
        for (int q = 0; q < m; q++) {
            PEnt &p = S.mob[q];
            for (int i = 0; i < 3; i++) p.U[i] = p.Int_U[i] * p.rho_s / p.M;
            for (int i = 0; i < 3; i++) p.Omega[i] = p.Int_Omega[i] * p.rho_s / p.I_p;
            for (int i = 0; i < 3; i++) p.U_old[i] = p.U[i];
            for (int i = 0; i < 3; i++) p.Omega_old[i] = p.Omega[i];
        }
    } else if (mode == PS_INIT_MOMENTUM) {
        for (int q = 0; q < m; q++) {
            PEnt &p = S.mob[q];
            for (int i = 0; i < 3; i++) p.Int_U_old[i] = p.Int_U[i];
            for (int i = 0; i < 3; i++) p.Int_Omega_old[i] = p.Int_Omega[i];
        }
    } else if (mode == PS_ADVANCE) {
        int nm = m, nf = f, who[2] = {-1, -1};
        const int rc = ps_advance(S.mob, nm, S.fix, nf, S.tmp, S.cap_ent, S.cap_own, g, stage, dt, who);
        S.nmob = nm;
        S.nfix = nf;
        if (rc) {
            S.err = rc;
            S.err_a = who[0];
            S.err_b = who[1];
        }
    }
}

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
                             const double *__restrict__ YL, const int *nm, int axis, double *__restrict__ out)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= *nm) return;
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
    if (e >= *D.ne) return;   // launched for the capacity; the block's exit is uniform
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

__global__ void k_ibm_spread(Dom d, IbmDev D, int comp, const double *__restrict__ xs,
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
    const int ne = *D.ne;
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
                              const double *__restrict__ geo, const int *ngeo_p, double shift, double denom,
                              double extra, double *__restrict__ CS)
{
    const int ngeo = *ngeo_p;
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
    if ((int)blockIdx.x >= *A.ne) return;   // launched for the capacity; the block's exit is uniform
    const IbmEntryDev &E = A.ent[blockIdx.x];
    const int np = *A.np;
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
            if (!owns_support(A.plist, np, E.id, A.xc[i], A.yc[j], A.support_width)) continue;
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

// Interpolate_paint_rigid_body_velocity_twod (Interpolate.c:734-800) of every
// mobile entry in list order: vel = vf (U + Omega_z x r) + (1 - vf) vel on the
// face cells of its box
__global__ void k_ps_paint(Dom d, const PSet *ps, int comp, const double *__restrict__ xu,
                           const double *__restrict__ xc, const double *__restrict__ yv,
                           const double *__restrict__ yc, double *__restrict__ vel)
{
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y);
    if (i >= d.NX || j >= d.NY) return;
    const int P = d.P;
    const PSet &S = *ps;
    for (int q = 0; q < S.ne; q++) {
        const PEnt &e = S.ent[q];
        if (!e.mobile) continue;
        const int *b = e.mbox[comp];
        if (i < b[0] || i >= b[1] || j < b[2] || j >= b[3]) continue;
        const double X0 = e.X[0], X1 = e.X[1];
        const double vf = face_solid_fraction(comp, i, j, X0, X1, e.R, xu, xc, yv, yc);
        if (vf <= 0.0) continue;
        const double om = e.Omega[2];
        const double u_rigid = comp == 0 ? e.U[0] - om * (yc[j] - X1) : e.U[1] + om * (xc[i] - X0);
        AT_(vel, i, j) = vf * u_rigid + (1.0 - vf) * AT_(vel, i, j);
    }
}

// ---------------------------------------------------------------------------
// device
// ---------------------------------------------------------------------------

}  // namespace pvof
