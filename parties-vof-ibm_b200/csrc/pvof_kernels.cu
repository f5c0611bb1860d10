// Routine kernels of the two-phase substep (everything except the iterative
// solvers, which live in pvof_cg.cu).  One kernel per reference loop nest,
// each running on the reference's index range; file:line citations are
// relative to PARTIES/src.
#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

#define KERNEL_2D_INDEX                                   \
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; \
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y; \
    const int P = d.P;                                    \
    (void)P;                                              \
    if (i >= i1 || j >= j1) return;

// ---------------------------------------------------------------------------
// ghost updates: one pass over the frame, reading interior sources only
// ---------------------------------------------------------------------------
__device__ __forceinline__ int frame_col(int c, int NX) { return c < 4 ? c - 3 : NX - 1 + (c - 4); }

__global__ void k_fill(Dom d, BcMap m, double *__restrict__ f)
{
    const int P = d.P;
    const int SXall = d.NX + 2 * NG, SYall = d.NY + 2 * NG;
    const int ncol = 8 * SYall;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int i, j;
    if (t < ncol) {
        i = frame_col(t / SYall, d.NX);
        j = t % SYall - NG;
    } else {
        t -= ncol;
        if (t >= 8 * SXall) return;
        j = frame_col(t / SXall, d.NY);
        i = t % SXall - NG;
        if (i <= 0 || i >= d.NX - 1) return;  // columns handled by the first pass
    }
    int si = m.x.src[i + NG], sj = m.y.src[j + NG];
    double mx = m.x.mul[i + NG], my = m.y.mul[j + NG];
    if (si == i && sj == j && mx == 1.0 && my == 1.0) return;
    double v = 0.0;
    if (mx != 0.0 && my != 0.0) v = mx * my * AT_(f, si, sj);
    AT_(f, i, j) = v;
}

// ---------------------------------------------------------------------------
// Cahn-Hilliard substep (Eulerian/VOF_DIFFUSE.c)
// ---------------------------------------------------------------------------

// VOF_DIFFUSE_compute_bulk_S (VOF_DIFFUSE.c:865-885)
__global__ void k_bulk_S(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                         const double *__restrict__ CS, double *__restrict__ bS)
{
    KERNEL_2D_INDEX
    double c = AT_(CL, i, j), cs = AT_(CS, i, j);
    AT_(bS, i, j) = 0.5 * c - 1.5 * c * c + c * c * c - c * cs * (1.0 - c - cs);
}

// bulk S in single precision (the FP32 stencil form)
__global__ void k_bulk_S_f(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                           const double *__restrict__ CS, double *__restrict__ bS)
{
    KERNEL_2D_INDEX
    const float c = (float)AT_(CL, i, j), cs = (float)AT_(CS, i, j);
    AT_(bS, i, j) = (double)(0.5f * c - 1.5f * c * c + c * c * c - c * cs * (1.0f - c - cs));
}

// the Laplacian in single precision (the FP32 stencil form)
__global__ void k_laplacian_f(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ in,
                              double *__restrict__ out)
{
    KERNEL_2D_INDEX
    AT_(out, i, j) = (double)lap_at_f(d, i, j, [&](int a, int b) { return AT_(in, a, b); });
}

// TwodOps_scalar_laplacian over the G range (VOF_DIFFUSE.c:834-861)
__global__ void k_laplacian(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ in,
                            double *__restrict__ out)
{
    KERNEL_2D_INDEX
    AT_(out, i, j) = lap_at(d, i, j, [&](int a, int b) { return AT_(in, a, b); });
}

// a = a / s (VOF_DIFFUSE.c:1007-1013)
__global__ void k_div_by(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ a, double s)
{
    KERNEL_2D_INDEX
    AT_(a, i, j) = AT_(a, i, j) / s;
}

// a += b (VOF_DIFFUSE.c:1290-1295)
__global__ void k_add(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ a, const double *__restrict__ b)
{
    KERNEL_2D_INDEX
    AT_(a, i, j) += AT_(b, i, j);
}

// a -= s * b (VOF_DIFFUSE.c:1049-1055)
__global__ void k_sub_scaled(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ a, const double *__restrict__ b, double s)
{
    KERNEL_2D_INDEX
    AT_(a, i, j) -= s * AT_(b, i, j);
}

// RK assembly rhs_vec (VOF_DIFFUSE.c:1299-1315)
__global__ void k_rhs_vec(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ vec, const double *__restrict__ CL,
                          const double *__restrict__ cur, const double *__restrict__ rn, double a_dt, int s)
{
    KERNEL_2D_INDEX
    if (s == 0) AT_(vec, i, j) = a_dt * AT_(CL, i, j) + gamb(0) * AT_(cur, i, j);
    else AT_(vec, i, j) = a_dt * AT_(CL, i, j) + gamb(s) * AT_(cur, i, j) + zetb(s) * AT_(rn, i, j);
}

// deterministic block partial sum of one value per thread (2D blocks)
__device__ __forceinline__ void block_partial(double v, double *partials)
{
    __shared__ double sh[32];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = (lane < nwarps) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) partials[blockIdx.y * gridDim.x + blockIdx.x] = w;
    }
}

// diffuse_bound_liquid_fraction (VOF_DIFFUSE.c:1093-1127) over the G range;
// the returned mass change counts the physical cells only (the half cells are
// copies that the ghost update overwrites).  Every thread of the launch must
// reach block_partial, so out-of-range threads add zero.
__global__ void k_bound(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ CL, const double *__restrict__ CS,
                        double *__restrict__ CG, double *partials)
{
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    const int P = d.P;
    double contrib = 0.0;
    if (i < i1 && j < j1) {
        double old_cl = AT_(CL, i, j);
        double cs = AT_(CS, i, j);
        double max_cl = 1.0 - cs;
        if (max_cl < 0.0) max_cl = 0.0;
        if (max_cl > 1.0) max_cl = 1.0;
        double new_cl = old_cl;
        if (new_cl < 0.0) new_cl = 0.0;
        if (new_cl > max_cl) new_cl = max_cl;
        AT_(CL, i, j) = new_cl;
        double cg = 1.0 - new_cl - cs;
        AT_(CG, i, j) = cg < 0.0 ? 0.0 : (cg > 1.0 ? 1.0 : cg);
        if (cs < 0.05 && i < d.NX - 1 && j < d.NY - 1)
            contrib = (new_cl - old_cl) * cell_measure(d, i, j);
    }
    block_partial(contrib, partials);
}

// sum of per-block partials in a fixed order, one block
__global__ void k_finalize_sum(const double *partials, int n, double *out)
{
    __shared__ double sh[32];
    double v = 0.0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) v += partials[q];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) *out = w;
    }
}

// VOF_DIFFUSE_update_phase_cache (VOF_DIFFUSE.c:108-126) over the whole
// allocated plane (L ranges), then F <- C_L
__global__ void k_phase_cache(size_t n, const double *__restrict__ CL, const double *__restrict__ CS,
                              double *__restrict__ CG, double *__restrict__ F)
{
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    double cg = 1.0 - CL[q] - CS[q];
    CG[q] = cg < 0.0 ? 0.0 : (cg > 1.0 ? 1.0 : cg);
    F[q] = CL[q];
}

// a W x H block between a contiguous buffer (row stride W) and a pitched
// plane (row stride P): the host copies move one contiguous block, these
// kernels do the strides on the device
__global__ void k_unpack_rows(double *__restrict__ dst, int P, const double *__restrict__ src, int W, int H)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)W * H) return;
    const int j = (int)(q / W), i = (int)(q - (size_t)j * W);
    dst[(size_t)j * P + i] = src[q];
}

__global__ void k_pack_rows(double *__restrict__ dst, const double *__restrict__ src, int P, int W, int H)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)W * H) return;
    const int j = (int)(q / W), i = (int)(q - (size_t)j * W);
    dst[q] = src[(size_t)j * P + i];
}

// C_L = clamp01(F) over the L ranges (VOF_DIFFUSE.c:532-538)
__global__ void k_clamp_from(size_t n, const double *__restrict__ F, double *__restrict__ CL)
{
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    double v = F[q];
    CL[q] = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

// VOF_DIFFUSE_update_density_viscosity (VOF_DIFFUSE.c:1453-1488)
__global__ void k_density(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                          const double *__restrict__ CS, const double *__restrict__ CG, double *__restrict__ rho,
                          double *__restrict__ mu, double rho_g, double mu_g)
{
    KERNEL_2D_INDEX
    const double rho_s = 1.0, mu_s = 1.0;
    AT_(rho, i, j) = AT_(CL, i, j) + rho_s * AT_(CS, i, j) + rho_g * AT_(CG, i, j);
    AT_(mu, i, j) = AT_(CL, i, j) + mu_s * AT_(CS, i, j) + mu_g * AT_(CG, i, j);
}

// VOF_DIFFUSE_compute_psi_LG (VOF_DIFFUSE.c:907-929)
__global__ void k_psi_LG(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                         const double *__restrict__ lap, double *__restrict__ psi, double cn2)
{
    KERNEL_2D_INDEX
    double c = AT_(CL, i, j);
    AT_(psi, i, j) = c * c * c - 1.5 * c * c + 0.5 * c - cn2 * AT_(lap, i, j);
}

// psi_LG in single precision (the FP32 stencil form)
__global__ void k_psi_LG_f(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                           const double *__restrict__ lap, double *__restrict__ psi, double cn2)
{
    KERNEL_2D_INDEX
    const float c = (float)AT_(CL, i, j);
    AT_(psi, i, j) = (double)(c * c * c - 1.5f * c * c + 0.5f * c - (float)cn2 * (float)AT_(lap, i, j));
}

// f_sigma in single precision (the FP32 stencil form); the band test on the
// averaged fractions stays as the reference's
__global__ void k_f_sigma_f(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                            const double *__restrict__ CG, const double *__restrict__ CS,
                            const double *__restrict__ psi, double *__restrict__ fx, double *__restrict__ fy,
                            double scale, int ui0, int ui1, int uj1, int vj0, int vi1, int vj1)
{
    KERNEL_2D_INDEX
    float vx = 0.0f, vy = 0.0f;
    const float sc = (float)scale;
    if (i >= ui0 && i < ui1 && j < uj1) {
        const float cl = 0.5f * ((float)AT_(CL, i, j) + (float)AT_(CL, i - 1, j));
        const float cg = 0.5f * ((float)AT_(CG, i, j) + (float)AT_(CG, i - 1, j));
        const float cs = 0.5f * ((float)AT_(CS, i, j) + (float)AT_(CS, i - 1, j));
        if (!(cl < 0.005f || cl > 0.995f || cg < 0.005f || cg > 0.995f || cs > 0.05f)) {
            const float pf = 0.5f * ((float)AT_(psi, i, j) + (float)AT_(psi, i - 1, j));
            const float gc = ((float)AT_(CL, i, j) - (float)AT_(CL, i - 1, j)) * (float)d.m.idx_c[i - 1];
            vx = sc * pf * gc;
        }
    }
    if (j >= vj0 && j < vj1 && i < vi1) {
        const float cl = 0.5f * ((float)AT_(CL, i, j) + (float)AT_(CL, i, j - 1));
        const float cg = 0.5f * ((float)AT_(CG, i, j) + (float)AT_(CG, i, j - 1));
        const float cs = 0.5f * ((float)AT_(CS, i, j) + (float)AT_(CS, i, j - 1));
        if (!(cl < 0.005f || cl > 0.995f || cg < 0.005f || cg > 0.995f || cs > 0.05f)) {
            const float pf = 0.5f * ((float)AT_(psi, i, j) + (float)AT_(psi, i, j - 1));
            const float gc = ((float)AT_(CL, i, j) - (float)AT_(CL, i, j - 1)) * (float)d.m.idy_c[j - 1];
            vy = sc * pf * gc;
        }
    }
    AT_(fx, i, j) = (double)vx;
    AT_(fy, i, j) = (double)vy;
}

// VOF_DIFFUSE_compute_f_sigma (VOF_DIFFUSE.c:1364-1445): zero the G range,
// then the band-limited face forces on the u and v ranges
__global__ void k_f_sigma(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL,
                          const double *__restrict__ CG, const double *__restrict__ CS, const double *__restrict__ psi,
                          double *__restrict__ fx, double *__restrict__ fy, double scale, int ui0, int ui1, int uj1,
                          int vj0, int vi1, int vj1)
{
    KERNEL_2D_INDEX
    double vx = 0.0, vy = 0.0;
    if (i >= ui0 && i < ui1 && j < uj1) {
        double cl = 0.5 * (AT_(CL, i, j) + AT_(CL, i - 1, j));
        double cg = 0.5 * (AT_(CG, i, j) + AT_(CG, i - 1, j));
        double cs = 0.5 * (AT_(CS, i, j) + AT_(CS, i - 1, j));
        if (!(cl < 0.005 || cl > 0.995 || cg < 0.005 || cg > 0.995 || cs > 0.05)) {
            double pf = 0.5 * (AT_(psi, i, j) + AT_(psi, i - 1, j));
            double gc = (AT_(CL, i, j) - AT_(CL, i - 1, j)) * d.m.idx_c[i - 1];
            vx = scale * pf * gc;
        }
    }
    if (j >= vj0 && j < vj1 && i < vi1) {
        double cl = 0.5 * (AT_(CL, i, j) + AT_(CL, i, j - 1));
        double cg = 0.5 * (AT_(CG, i, j) + AT_(CG, i, j - 1));
        double cs = 0.5 * (AT_(CS, i, j) + AT_(CS, i, j - 1));
        if (!(cl < 0.005 || cl > 0.995 || cg < 0.005 || cg > 0.995 || cs > 0.05)) {
            double pf = 0.5 * (AT_(psi, i, j) + AT_(psi, i, j - 1));
            double gc = (AT_(CL, i, j) - AT_(CL, i, j - 1)) * d.m.idy_c[j - 1];
            vy = scale * pf * gc;
        }
    }
    AT_(fx, i, j) = vx;
    AT_(fy, i, j) = vy;
}

// VOF_apply_f_sigma_old (VOF_SurfaceTension.c:1983-2041), one component
__global__ void k_add_to(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ rhs, const double *__restrict__ f)
{
    KERNEL_2D_INDEX
    AT_(rhs, i, j) += AT_(f, i, j);
}

// Velocity_add_gravity_2_RHS (VOF_SurfaceTension.c:2075-2154), one component
__global__ void k_gravity(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ rho,
                          double *__restrict__ rhs, int di, int dj, double Ri, double g)
{
    KERNEL_2D_INDEX
    double rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i - di, j - dj));
    AT_(rhs, i, j) += 2.0 * rf * Ri * g;
}

// Velocity_cell_center averages (Velocity.c:322-352) over the L ranges minus one
__global__ void k_cell_center(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ u,
                              const double *__restrict__ v, double *__restrict__ ub, double *__restrict__ vb)
{
    KERNEL_2D_INDEX
    AT_(ub, i, j) = 0.5 * (AT_(u, i, j) + AT_(u, i + 1, j));
    AT_(vb, i, j) = 0.5 * (AT_(v, i, j) + AT_(v, i, j + 1));
}

// Velocity_u_set_implicit_explicit (Velocity.c:366-762), diffuse VOF
__global__ void k_u_impexp(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ u,
                           const double *__restrict__ v, const double *__restrict__ ub, const double *__restrict__ mu,
                           double *__restrict__ ex, double *__restrict__ im, double *__restrict__ vx, double iRe)
{
    KERNEL_2D_INDEX
    const Metrics &m = d.m;
    double muE = AT_(mu, i, j), muW = AT_(mu, i - 1, j);
    double a = 0.5 * (AT_(mu, i - 1, j + 1) + AT_(mu, i, j + 1));
    double b = 0.5 * (AT_(mu, i - 1, j) + AT_(mu, i, j));
    double c = 0.5 * (AT_(mu, i - 1, j - 1) + AT_(mu, i, j - 1));
    double mu_yp = 2.0 * a * b / (a + b + 1e-12);
    double mu_ym = 2.0 * b * c / (b + c + 1e-12);
    double dudxE = (AT_(u, i + 1, j) - AT_(u, i, j)) * m.idx_u[i];
    double dudxW = (AT_(u, i, j) - AT_(u, i - 1, j)) * m.idx_u[i - 1];
    double dudyN = (AT_(u, i, j + 1) - AT_(u, i, j)) * m.idy_c[j];
    double dudyS = (AT_(u, i, j) - AT_(u, i, j - 1)) * m.idy_c[j - 1];
    double d2udy2 = iRe * (mu_yp * dudyN - mu_ym * dudyS) * m.idy_v[j];
    double dvdxN = (AT_(v, i, j + 1) - AT_(v, i - 1, j + 1)) * m.idx_c[i - 1];
    double dvdxS = (AT_(v, i, j) - AT_(v, i - 1, j)) * m.idx_c[i - 1];
    double d2udx2 = iRe * u_cv_x_div(d, i, muE * dudxE, muW * dudxW);
    double ddydvdx = iRe * (mu_yp * dvdxN - mu_ym * dvdxS) * m.idy_v[j];
    double axc = axisym_ur_term(d, i, iRe * 0.5 * (muE + muW), AT_(u, i, j));
    double vCN = 0.5 * (AT_(v, i, j + 1) + AT_(v, i - 1, j + 1));
    double vCS = 0.5 * (AT_(v, i, j) + AT_(v, i - 1, j));
    double uuE = AT_(ub, i, j) * AT_(ub, i, j);
    double uuW = AT_(ub, i - 1, j) * AT_(ub, i - 1, j);
    double uvN = 0.5 * (AT_(u, i, j) + AT_(u, i, j + 1)) * vCN;
    double uvS = 0.5 * (AT_(u, i, j) + AT_(u, i, j - 1)) * vCS;
    double duudx = u_cv_x_div(d, i, uuE, uuW);
    double duvdy = (uvN - uvS) * m.idy_v[j];
    AT_(ex, i, j) = -(duudx + duvdy);
    AT_(vx, i, j) = d2udx2 + ddydvdx;
    AT_(im, i, j) = d2udx2 + d2udy2 + axc;
}

// Velocity_v_set_implicit_explicit (Velocity.c:771-1148), diffuse VOF
__global__ void k_v_impexp(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ u,
                           const double *__restrict__ v, const double *__restrict__ vb, const double *__restrict__ mu,
                           double *__restrict__ ex, double *__restrict__ im, double *__restrict__ vx, double iRe)
{
    KERNEL_2D_INDEX
    const Metrics &m = d.m;
    double a = 0.5 * (AT_(mu, i + 1, j - 1) + AT_(mu, i + 1, j));
    double b = 0.5 * (AT_(mu, i, j - 1) + AT_(mu, i, j));
    double c = 0.5 * (AT_(mu, i - 1, j - 1) + AT_(mu, i - 1, j));
    double mu_xp = 2.0 * a * b / (a + b + 1e-12);
    double mu_xm = 2.0 * b * c / (b + c + 1e-12);
    double mu_yp = AT_(mu, i, j), mu_ym = AT_(mu, i, j - 1);
    double dvdxE = (AT_(v, i + 1, j) - AT_(v, i, j)) * m.idx_c[i];
    double dvdxW = (AT_(v, i, j) - AT_(v, i - 1, j)) * m.idx_c[i - 1];
    double dvdyN = (AT_(v, i, j + 1) - AT_(v, i, j)) * m.idy_v[j];
    double dvdyS = (AT_(v, i, j) - AT_(v, i, j - 1)) * m.idy_v[j - 1];
    double d2vdx2 = iRe * v_cv_x_div(d, i, mu_xp * dvdxE, mu_xm * dvdxW);
    double d2vdy2 = iRe * (mu_yp * dvdyN - mu_ym * dvdyS) * m.idy_c[j - 1];
    double dudyE = (AT_(u, i + 1, j) - AT_(u, i + 1, j - 1)) * m.idy_c[j - 1];
    double dudyW = (AT_(u, i, j) - AT_(u, i, j - 1)) * m.idy_c[j - 1];
    double ddxdudy = iRe * v_cv_x_div(d, i, mu_xp * dudyE, mu_xm * dudyW);
    double uCE = 0.5 * (AT_(u, i + 1, j) + AT_(u, i + 1, j - 1));
    double uCW = 0.5 * (AT_(u, i, j) + AT_(u, i, j - 1));
    double vuE = 0.5 * (AT_(v, i, j) + AT_(v, i + 1, j)) * uCE;
    double vuW = 0.5 * (AT_(v, i, j) + AT_(v, i - 1, j)) * uCW;
    double vvN = AT_(vb, i, j) * AT_(vb, i, j);
    double vvS = AT_(vb, i, j - 1) * AT_(vb, i, j - 1);
    double dvudx = v_cv_x_div(d, i, vuE, vuW);
    double dvvdy = (vvN - vvS) * m.idy_c[j - 1];
    AT_(ex, i, j) = -(dvudx + dvvdy);
    AT_(vx, i, j) = ddxdudy + d2vdy2;
    AT_(im, i, j) = d2vdx2 + d2vdy2;
}

// Velocity_{u,v}_set_RHS (Velocity.c:1494-1728, :1739-1940), diffuse VOF
__global__ void k_set_rhs(Dom d, int i0, int i1, int j0, int j1, int comp, const double *__restrict__ data,
                          const double *__restrict__ pd, const double *__restrict__ rho, double *__restrict__ rhs,
                          const double *__restrict__ ex, double *__restrict__ exo, const double *__restrict__ vx,
                          double *__restrict__ vxo, const double *__restrict__ im, double a_dt, int s, double dp_src,
                          int resolved)
{
    KERNEL_2D_INDEX
    double dp, rf;
    if (comp == 0) {
        dp = (AT_(pd, i, j) - AT_(pd, i - 1, j)) * d.m.idx_c[i - 1];
        rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i - 1, j));
    } else {
        dp = (AT_(pd, i, j) - AT_(pd, i, j - 1)) * d.m.idy_c[j - 1];
        rf = 0.5 * (AT_(rho, i, j) + AT_(rho, i, j - 1));
    }
    double e = AT_(ex, i, j), eo = AT_(exo, i, j), v = AT_(vx, i, j), vo = AT_(vxo, i, j);
    double conv = gamb(s) * e + zetb(s) * eo;
    conv *= rf;
    double r = rf * a_dt * AT_(data, i, j) + conv + AT_(im, i, j) + (gamb(s) * v + zetb(s) * vo) - 2.0 * dp;
    // with resolved particles the implicit part goes in twice; Lagrangian_force(-1)
    // takes the second copy out again (Velocity.c:1665-1667, Lagrangian.c:1855-1867)
    if (resolved) r += AT_(im, i, j);
    if (comp == 0 && d.perx) r += 2.0 * dp_src;
    AT_(rhs, i, j) = r;
    AT_(exo, i, j) = e;
    AT_(vxo, i, j) = v;
}

// Pressure_set_RHS (Pressure.c:100-196), GRID_UNIFORM
__global__ void k_p_rhs(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ u,
                        const double *__restrict__ v, double *__restrict__ rhs, double ihdt)
{
    KERNEL_2D_INDEX
    AT_(rhs, i, j) = cell_div(d, u, v, i, j, ihdt, ihdt);
}

// Pressure_compute_preconditioner (psolve_cg.c:63-101)
__global__ void k_p_precond(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ rho, double *__restrict__ M)
{
    KERNEL_2D_INDEX
    double r0 = AT_(rho, i, j);
    double bxp = 2.0 / (r0 + AT_(rho, i + 1, j));
    double bxm = 2.0 / (r0 + AT_(rho, i - 1, j));
    double byp = 2.0 / (r0 + AT_(rho, i, j + 1));
    double bym = 2.0 / (r0 + AT_(rho, i, j - 1));
    double cxm, cxp, cym, cyp;
    face_coeffs(d, i, bxm, bxp, bym, byp, cxm, cxp, cym, cyp);
    double aii = cxm + cxp + cym + cyp + 0.0 + 0.0;
    AT_(M, i, j) = 1.0 / (row_weight(d, i) * aii + 1e-12);
}

// p += deltap (Pressure.c:296-309)
__global__ void k_p_update(Dom d, int i0, int i1, int j0, int j1, double *__restrict__ pd, const double *__restrict__ dp)
{
    KERNEL_2D_INDEX
    AT_(pd, i, j) += AT_(dp, i, j);
}

// velocity projection (Pressure.c:340-410), one component
__global__ void k_project(Dom d, int i0, int i1, int j0, int j1, int comp, double *__restrict__ vel,
                          const double *__restrict__ dp, const double *__restrict__ rho, double mdt)
{
    KERNEL_2D_INDEX
    if (comp == 0) {
        double inv = 2.0 / (AT_(rho, i, j) + AT_(rho, i - 1, j));
        AT_(vel, i, j) -= (AT_(dp, i, j) - AT_(dp, i - 1, j)) * (d.m.idx_c[i - 1] * mdt * inv);
    } else {
        double inv = 2.0 / (AT_(rho, i, j) + AT_(rho, i, j - 1));
        AT_(vel, i, j) -= (AT_(dp, i, j) - AT_(dp, i, j - 1)) * (d.m.idy_c[j - 1] * mdt * inv);
    }
}

// Pressure_compute_velocity_divergence (Pressure.c:475-597): max |div|;
// non-negative doubles order like their bit patterns
__global__ void k_div_max(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ u,
                          const double *__restrict__ v, unsigned long long *out)
{
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    double dc = 0.0;
    if (i < i1 && j < j1) dc = fabs(cell_div(d, u, v, i, j, d.m.idx_u[i], d.m.idy_v[j]));
    __shared__ double sh[32];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int o = 16; o > 0; o >>= 1) dc = fmax(dc, __shfl_down_sync(0xffffffffu, dc, o));
    if (lane == 0) sh[warp] = dc;
    __syncthreads();
    if (tid == 0) {
        double m = sh[0];
        for (int w = 1; w < (int)((blockDim.x * blockDim.y + 31) >> 5); w++) m = fmax(m, sh[w]);
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// liquid mass diagnostic over the physical cells
__global__ void k_mass(Dom d, int i0, int i1, int j0, int j1, const double *__restrict__ CL, double *partials)
{
    const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = j0 + blockIdx.y * blockDim.y + threadIdx.y;
    const int P = d.P;
    double v = 0.0;
    if (i < i1 && j < j1) v = AT_(CL, i, j) * cell_measure(d, i, j);
    block_partial(v, partials);
}

}  // namespace pvof
