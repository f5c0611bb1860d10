// Moving contact line on resolved solids: the characteristic projection of
// Liu & Ding (2015, section 2.4) as PARTIES implements it for the 2D modes in
// Eulerian/VOF_IBM_wetting.c:
//
//   k_mcl_normals        VOF_DIFFUSE_compute_solid_normals_MCL (:1021-1104):
//                        n_s = -grad C_S / |grad C_S| on the whole ghosted
//                        plane, one-sided at its edges, the nearest-particle
//                        direction where the gradient vanishes inside the
//                        diffuse shell (:118-182); the boundary parity of
//                        mcl_apply_normal_parity (:914-1016) is a ghost map
//   k_mcl_apply          mcl_iter_apply_C_L (:1824-1944): every "ghost
//                        contact cell" (Eq. 18: a solid cell, C_S >= 0.05, in
//                        the liquid-gas band or next to a fluid cell that is)
//                        takes C_L from the Eq. 20 quadratic sample where one
//                        of the two characteristics at +-(pi/2 - theta) about
//                        the normal first crosses a usable fluid-side mesh
//                        line (Eq. 19: the larger sample for theta <= 90 deg,
//                        else the smaller)
//   k_mcl_extend_psi     VOF_DIFFUSE_extend_psi_LG_contact_angle
//                        (:2014-2131): the branch re-selected from C_L, then
//                        psi_LG sampled along it
//
// The reference reads every scalar of a pass from a snapshot of the G range
// taken before the pass (mcl_global_refresh, :670-705), with out-of-range
// indices folded back by the boundary maps of :534-648; the kernels read the
// same G-range values through the same maps (mcl_map_x/y), so the cells of a
// pass are independent and run one thread each.  The tracer is the
// reference's grid DDA over scalar mesh lines, at most 32 crossings
// (:1390-1499); the bracketing searches of :1168-1210 are binary searches
// that return the first bracket the reference's linear scan finds.
#include <cfloat>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

namespace {

constexpr double MCL_CS_SOLID = 0.05;
constexpr double MCL_GRAD_EPS = 1.0e-12;
constexpr double MCL_NORM_EPS = 1.0e-12;
constexpr double MCL_TINY = 1.0e-30;
constexpr int MCL_MAX_DDA_STEPS = 32;

// mcl_global_map_x / _y (:534-625): fold an index of the ghosted range onto
// the G range
__host__ __device__ inline bool map_axis(int i, int N, int periodic, int free_lo, int free_hi, int &ii)
{
    if (periodic) {
        ii = i % N;
        if (ii < 0) ii += N;
        return true;
    }
    if (i >= 0 && i < N) { ii = i; return true; }
    if (i < 0) {
        if (free_lo) {
            ii = -i - 1;
            return ii >= 0 && ii < N;
        }
        ii = 0;
        return true;
    }
    if (free_hi) {
        ii = 2 * N - i - 1;
        return ii >= 0 && ii < N;
    }
    ii = N - 1;
    return true;
}

struct Mcl {
    const Dom &d;
    const MclView &v;

    __host__ __device__ bool in_x(int i) const { return i >= -NG && i < v.NX + NG; }
    __host__ __device__ bool in_y(int j) const { return j >= -NG && j < v.NY + NG; }

    // mcl_global_value (:650-668)
    __host__ __device__ bool read(const double *buf, int i, int j, double &out) const
    {
        if (!in_x(i) || !in_y(j)) return false;
        int ii, jj;
        if (!map_axis(i, v.NX, v.perx, v.free_lo_x, v.free_hi_x, ii)) return false;
        if (!map_axis(j, v.NY, v.pery, v.free_lo_y, v.free_hi_y, jj)) return false;
        const int P = d.P;
        out = AT_(buf, ii, jj);
        return true;
    }

    __host__ __device__ bool solid(int i, int j) const
    {
        double cs = 0.0;
        return read(v.CS, i, j, cs) && cs >= MCL_CS_SOLID;
    }

    __host__ __device__ bool band(double cl, double cg) const
    {
        return (cl > v.cmin) && (cl < v.cmax) && (cg > v.cmin) && (cg < v.cmax);
    }

    // mcl_is_ghost_contact_cell (:1517-1551)
    __host__ __device__ bool contact(int i, int j) const
    {
        if (!solid(i, j)) return false;
        double cl = 0.0, cg = 0.0;
        if (read(v.CL, i, j, cl) && read(v.CG, i, j, cg) && band(cl, cg)) return true;
        const int di[4] = {1, -1, 0, 0}, dj[4] = {0, 0, 1, -1};
        for (int s = 0; s < 4; ++s) {
            const int ni = i + di[s], nj = j + dj[s];
            if (!in_x(ni) || !in_y(nj)) continue;
            if (solid(ni, nj)) continue;
            if (read(v.CL, ni, nj, cl) && read(v.CG, ni, nj, cg) && band(cl, cg)) return true;
        }
        return false;
    }

    // mcl_bracket_y / _x (:1168-1210): the first j of [-NG, N+NG-1) with
    // c[j] - eps <= p <= c[j+1] + eps on the increasing coordinates c.  The
    // upper condition holds from some j on and the lower one up to some j,
    // so the first j meeting both is the first j meeting the upper one, if
    // the lower one holds there.
    __host__ __device__ static bool bracket(const double *c, int N, double p, int &lo)
    {
        const double eps = 1.0e-12;
        int a = -NG, b = N + NG - 1;
        while (a < b) {
            const int m = a + ((b - a) >> 1);
            if (p <= c[m + 1] + eps) b = m;
            else a = m + 1;
        }
        if (a >= N + NG - 1) return false;
        if (!(p >= c[a] - eps)) return false;
        lo = a;
        return true;
    }

    __host__ __device__ bool valid_for_quad(int i, int j) const { return in_x(i) && in_y(j) && !solid(i, j); }

    // mcl_try_quad_stencil (:1226-1273) with mcl_quad_interp_eq20 (:1144-1153)
    __host__ __device__ bool quad(const double *field, int iA, int jA, int iB, int jB, int iC, int jC, double xD, double yD,
                         int axis, double &value, double &score) const
    {
        if (!valid_for_quad(iA, jA) || !valid_for_quad(iB, jB) || !valid_for_quad(iC, jC)) return false;
        double h, lAD;
        if (axis == 0) {
            h = fabs(v.yc[jB] - v.yc[jA]);
            lAD = fabs(yD - v.yc[jA]);
        } else {
            h = fabs(v.xc[iB] - v.xc[iA]);
            lAD = fabs(xD - v.xc[iA]);
        }
        if (h <= MCL_TINY) return false;
        if (lAD < -1e-12 || lAD > h + 1e-12) return false;
        double fA, fB, fC;
        if (!read(field, iA, jA, fA) || !read(field, iB, jB, fB) || !read(field, iC, jC, fC)) return false;
        const double r = lAD / h;
        value = r * r * (0.5 * fA - fB + 0.5 * fC) + r * (-1.5 * fA + 2.0 * fB - 0.5 * fC) + fA;
        return read(v.CS, iC, jC, score);
    }

    // mcl_sample_at_hit (:1275-1383): D on a vertical (axis 0) or horizontal
    // scalar mesh line; C beyond either end of AB, the one nearer C_S = 0.05
    __host__ __device__ bool sample(const double *field, int ci, int cj, int axis, double xD, double yD, double &out) const
    {
        double v1 = 0.0, v2 = 0.0, s1 = -DBL_MAX, s2 = -DBL_MAX;
        bool ok1, ok2;
        if (axis == 0) {
            if (!in_x(ci)) return false;
            int jlo;
            if (!bracket(v.yc, v.NY, yD, jlo)) return false;
            const int jhi = jlo + 1;
            ok1 = quad(field, ci, jlo, ci, jhi, ci, jhi + 1, xD, yD, axis, v1, s1);
            ok2 = quad(field, ci, jhi, ci, jlo, ci, jlo - 1, xD, yD, axis, v2, s2);
        } else {
            if (!in_y(cj)) return false;
            int ilo;
            if (!bracket(v.xc, v.NX, xD, ilo)) return false;
            const int ihi = ilo + 1;
            ok1 = quad(field, ilo, cj, ihi, cj, ihi + 1, cj, xD, yD, axis, v1, s1);
            ok2 = quad(field, ihi, cj, ilo, cj, ilo - 1, cj, xD, yD, axis, v2, s2);
        }
        if (!ok1 && !ok2) return false;
        if (ok1 && ok2) out = (s1 >= s2) ? v1 : v2;
        else out = ok1 ? v1 : v2;
        return true;
    }

    // mcl_trace_branch_by_scalar_lines (:1390-1499)
    __host__ __device__ bool trace(const double *field, int i0, int j0, const double dir[2], double &out) const
    {
        double x = v.xc[i0], y = v.yc[j0];
        int il = i0, jl = j0;
        for (int step = 0; step < MCL_MAX_DDA_STEPS; ++step) {
            double tx = 1.0e300, ty = 1.0e300;
            int next_i = il, next_j = jl;
            if (dir[0] > MCL_TINY) {
                next_i = il + 1;
                if (!in_x(next_i)) return false;
                tx = (v.xc[next_i] - x) / dir[0];
            } else if (dir[0] < -MCL_TINY) {
                next_i = il - 1;
                if (!in_x(next_i)) return false;
                tx = (v.xc[next_i] - x) / dir[0];
            }
            if (dir[1] > MCL_TINY) {
                next_j = jl + 1;
                if (!in_y(next_j)) return false;
                ty = (v.yc[next_j] - y) / dir[1];
            } else if (dir[1] < -MCL_TINY) {
                next_j = jl - 1;
                if (!in_y(next_j)) return false;
                ty = (v.yc[next_j] - y) / dir[1];
            }
            if (tx <= MCL_TINY) tx = 1.0e300;
            if (ty <= MCL_TINY) ty = 1.0e300;
            if (tx >= 1.0e299 && ty >= 1.0e299) return false;
            double tmin;
            int ci, cj, axis;
            if (tx <= ty) {
                tmin = tx;
                ci = next_i;
                cj = jl;
                axis = 0;
                il = next_i;
            } else {
                tmin = ty;
                ci = il;
                cj = next_j;
                axis = 1;
                jl = next_j;
            }
            x = x + tmin * dir[0];
            y = y + tmin * dir[1];
            if (sample(field, ci, cj, axis, x, y, out)) return true;
        }
        return false;
    }
};

// mcl_characteristic_dirs (:1110-1138); ct, st = cos, sin of theta
__host__ __device__ bool characteristic_dirs(double nx, double ny, double ct, double st, double d1[2], double d2[2])
{
    const double mag = sqrt(nx * nx + ny * ny);
    if (mag < MCL_NORM_EPS) return false;
    const double n0 = nx / mag, n1 = ny / mag;
    const double t0 = -n1, t1 = n0;
    d1[0] = ct * t0 + st * n0;
    d1[1] = ct * t1 + st * n1;
    d2[0] = -ct * t0 + st * n0;
    d2[1] = -ct * t1 + st * n1;
    const double l1 = sqrt(d1[0] * d1[0] + d1[1] * d1[1]);
    const double l2 = sqrt(d2[0] * d2[0] + d2[1] * d2[1]);
    if (l1 < MCL_NORM_EPS || l2 < MCL_NORM_EPS) return false;
    d1[0] /= l1;
    d1[1] /= l1;
    d2[0] /= l2;
    d2[1] /= l2;
    return true;
}

}  // namespace

// VOF_DIFFUSE_compute_solid_normals_MCL (:1021-1104) at one cell of the
// ghosted plane; plist: x, y, R, ID of every entry of the current particle
// lists (mobile, then fixed), as mcl_nearest_particle_normal (:118-182)
// walks them
__host__ __device__ void mcl_normal_cell(const Dom &d, const double *xc, const double *yc, const double *CS,
                                         const double *plist, int np, double support_width, double *nxo,
                                         double *nyo, int i, int j)
{
    const int P = d.P;
    const int iL = -NG, iE = d.NX + NG, jL = -NG, jE = d.NY + NG;
    double gx, gy;
    if (i > iL && i < iE - 1) gx = (AT_(CS, i + 1, j) - AT_(CS, i - 1, j)) * (1.0 / (xc[i + 1] - xc[i - 1]));
    else if (i == iL) gx = (AT_(CS, i + 1, j) - AT_(CS, i, j)) * d.m.idx_c[i];
    else gx = (AT_(CS, i, j) - AT_(CS, i - 1, j)) * d.m.idx_c[i - 1];
    if (j > jL && j < jE - 1) gy = (AT_(CS, i, j + 1) - AT_(CS, i, j - 1)) * (1.0 / (yc[j + 1] - yc[j - 1]));
    else if (j == jL) gy = (AT_(CS, i, j + 1) - AT_(CS, i, j)) * d.m.idy_c[j];
    else gy = (AT_(CS, i, j) - AT_(CS, i, j - 1)) * d.m.idy_c[j - 1];
    const double mag = sqrt(gx * gx + gy * gy);
    double nx = 0.0, ny = 0.0;
    if (mag < MCL_GRAD_EPS) {
        const double cs = AT_(CS, i, j);
        if (cs > 1.0e-12 && cs < 1.0 - 1.0e-12) {
            const double x = xc[i], y = yc[j];
            double best_gap = DBL_MAX, bx = 0.0, by = 0.0, bz = 0.0, best_id = 0.0;
            bool found = false;
            for (int q = 0; q < np; q++) {
                const double *pq = plist + 4 * q;
                const double support = pq[2] + support_width;
                const double dx = x - pq[0], dy = y - pq[1], dz = 0.0;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 > support * support || d2 <= 1.0e-30) continue;
                const double gap = sqrt(d2) - pq[2];
                if (!found || gap < best_gap - 1.0e-12 || (fabs(gap - best_gap) <= 1.0e-12 && pq[3] < best_id)) {
                    best_gap = gap;
                    bx = dx;
                    by = dy;
                    bz = dz;
                    best_id = pq[3];
                    found = true;
                }
            }
            if (found) {
                const double len = sqrt(bx * bx + by * by + bz * bz);
                if (len > 1.0e-30) {
                    nx = bx / len;
                    ny = by / len;
                }
            }
        }
    } else {
        nx = -gx / mag;
        ny = -gy / mag;
    }
    AT_(nxo, i, j) = nx;
    AT_(nyo, i, j) = ny;
}

// mcl_iter_apply_C_L (:1824-1944) at one G-range cell: reads v.CL (the
// snapshot), writes the projected value of a ghost contact cell into CLout
__host__ __device__ void mcl_apply_cell(const Dom &d, const MclView &v, const double *nxa, const double *nya,
                                        double *CLout, int i, int j)
{
    Mcl m{d, v};
    if (!m.contact(i, j)) return;
    const int P = d.P;
    double d1[2], d2[2];
    if (!characteristic_dirs(AT_(nxa, i, j), AT_(nya, i, j), v.ct, v.st, d1, d2)) return;
    double r1 = 0.0, r2 = 0.0;
    const bool ok1 = m.trace(v.CL, i, j, d1, r1);
    const bool ok2 = m.trace(v.CL, i, j, d2, r2);
    if (!ok1 && !ok2) return;
    double cl;
    if (ok1 && ok2) {
        if (v.hydrophilic) cl = (r1 >= r2) ? r1 : r2;
        else cl = (r1 <= r2) ? r1 : r2;
    } else {
        cl = ok1 ? r1 : r2;
    }
    if (cl < 0.0) cl = 0.0;
    if (cl > 1.0) cl = 1.0;
    AT_(CLout, i, j) = cl;
}

// VOF_DIFFUSE_extend_psi_LG_contact_angle (:2014-2131) at one G-range cell:
// the branch from v.CL, the sample from v.field (the psi_LG snapshot)
__host__ __device__ void mcl_extend_cell(const Dom &d, const MclView &v, const double *nxa, const double *nya,
                                         double *PSIout, int i, int j)
{
    Mcl m{d, v};
    if (!m.contact(i, j)) return;
    const int P = d.P;
    double d1[2], d2[2];
    if (!characteristic_dirs(AT_(nxa, i, j), AT_(nya, i, j), v.ct, v.st, d1, d2)) return;
    double c1 = 0.0, c2 = 0.0;
    const bool ok1 = m.trace(v.CL, i, j, d1, c1);
    const bool ok2 = m.trace(v.CL, i, j, d2, c2);
    if (!ok1 && !ok2) return;
    int branch;
    if (ok1 && ok2) {
        if (v.hydrophilic) branch = (c1 >= c2) ? +1 : -1;
        else branch = (c1 <= c2) ? +1 : -1;
    } else {
        branch = ok1 ? +1 : -1;
    }
    double p = 0.0;
    if (m.trace(v.field, i, j, branch == +1 ? d1 : d2, p)) AT_(PSIout, i, j) = p;
}

__global__ void k_mcl_normals(Dom d, const double *__restrict__ xc, const double *__restrict__ yc,
                              const double *__restrict__ CS, const double *__restrict__ plist,
                              const int *np, double support_width, double *__restrict__ nxo,
                              double *__restrict__ nyo)
{
    const int i = -NG + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = -NG + (int)blockIdx.y;
    if (i >= d.NX + NG) return;
    mcl_normal_cell(d, xc, yc, CS, plist, *np, support_width, nxo, nyo, i, j);
}

// VOF_DIFFUSE_compute_solid_normals_MCL and mcl_apply_normal_parity on the
// symmetry axis (VOF_IBM_wetting.c:938-953, :1092-1099): the radial component
// is zero in the first cell column, and the ghost columns mirror it, the
// radial component with its sign flipped; one thread per row of the ghosted
// plane
__global__ void k_mcl_axis_normals(Dom d, double *__restrict__ nx, double *__restrict__ ny)
{
    const int j = -NG + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (j >= d.NY + NG) return;
    const int P = d.P;
    AT_(nx, 0, j) = 0.0;
    for (int g = 1; g <= NG; ++g) {
        AT_(nx, -g, j) = -AT_(nx, g - 1, j);
        AT_(ny, -g, j) = AT_(ny, g - 1, j);
    }
}

__global__ void k_mcl_apply(Dom d, MclView v, const double *__restrict__ nxa, const double *__restrict__ nya,
                            double *__restrict__ CLout)
{
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y;
    if (i >= v.NX || j >= v.NY) return;
    mcl_apply_cell(d, v, nxa, nya, CLout, i, j);
}

__global__ void k_mcl_extend_psi(Dom d, MclView v, const double *__restrict__ nxa, const double *__restrict__ nya,
                                 double *__restrict__ PSIout)
{
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y;
    if (i >= v.NX || j >= v.NY) return;
    mcl_extend_cell(d, v, nxa, nya, PSIout, i, j);
}

}  // namespace pvof
