// Cluster-resident Jacobi-PCG solvers in a column-strip layout, for solve
// ranges that fit one thread-block cluster (16 CTAs of NT threads, at most CPT
// cells per thread):
//
//   Pressure_solve_cg  (Eulerian/lsolver/psolve_cg.c:130-293)
//   Velocity_solve_cg  (Eulerian/lsolver/msolve_cg.c:525-722), u and v in one
//                      launch as two independent clusters (the reference
//                      solves them back to back from inputs neither solve
//                      changes, Temporal_int.c:996-997).
//
// Layout and schedule:
//   * the cluster's CTAs split the rows of the solve range into slabs; in a
//     CTA, thread t owns column t % W and a strip of up to CPT consecutive
//     rows of the slab (band t / W), so the north and south neighbours of a
//     cell are in the thread's own registers except at the strip ends;
//   * the residual and the search direction of the thread's cells (and the
//     preconditioner or the solution) are kept in registers; the operator's
//     coefficients are computed once per solve (rho and mu do not change
//     during it) into shared memory;
//   * per iteration each thread writes the new direction of its cells to
//     shared memory once, in rows with one ghost column on each side that the
//     owners of the ghosts' source columns fill, so east/west and strip-end
//     neighbours are plain shared-memory reads after one CTA barrier;
//   * the rows just outside the slab are evaluated from the neighbouring CTA's
//     boundary z row and previous direction through distributed shared memory,
//     both visible since the last cluster barrier, so the direction update and
//     the operator need no cluster barrier of their own;
//   * the inner products are reduced through distributed shared memory behind
//     hardware cluster barriers, every CTA summing the per-CTA partials in the
//     same order, so every CTA takes the same convergence decisions; the
//     iteration's scalar arithmetic (alpha, beta, the stopping test) runs once
//     per CTA and is broadcast with the sums.
// Two cluster barriers per iteration.  The per-cell arithmetic is the
// reference's: the same operands in the same order.
#include <cooperative_groups.h>
#include <cstdlib>
#include <mutex>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace cg = cooperative_groups;

namespace pvof {

// ---------------------------------------------------------------------------
// slab partition of H rows over nb CTAs
// ---------------------------------------------------------------------------
__host__ __device__ inline int slab_row0(int c, int H, int nb) { return (int)(((long long)c * H) / nb); }

__host__ __device__ inline int slab_owner(int j, int H, int nb)
{
    int c = (int)(((long long)j * nb) / H);
    while (c > 0 && slab_row0(c, H, nb) > j) c--;
    while (c < nb - 1 && slab_row0(c + 1, H, nb) <= j) c++;
    return c;
}

// Source of the row just outside a slab (side < 0: below, > 0: above) under
// the ghost map `ym` of the solve range [rj0, rj0 + H): the range row it
// reads (or -1 when the value is zero) and the multiplier.
__host__ __device__ inline int edge_source(const int *ysrc, const double *ymul, int rj0, int H, int b, double &mul)
{
    if (b >= rj0 && b < rj0 + H) { mul = 1.0; return b - rj0; }
    const int s = ysrc[b + NG];
    mul = ymul[b + NG];
    if (mul == 0.0 || s < rj0 || s >= rj0 + H) { mul = 0.0; return -1; }
    return s - rj0;
}

// One neighbour row of the slab, outside it.
struct SlabEdge {
    double mul;          // 0: the neighbour value is zero
    int local;           // 1: the source row is in this CTA's slab
    int lrow;            // its local row (local) or its row in the owner's slab
    int zsel;            // 0: the owner's first row, 1: its last row
    int owner;
};

__device__ inline SlabEdge slab_edge(const int *ysrc, const double *ymul, int rj0, int H, int nb, int rank, int b,
                                     int *error)
{
    SlabEdge e;
    int s = edge_source(ysrc, ymul, rj0, H, b, e.mul);
    e.local = 1; e.lrow = 0; e.zsel = 0; e.owner = rank;
    if (s < 0) return e;
    e.owner = slab_owner(s, H, nb);
    e.lrow = s - slab_row0(e.owner, H, nb);
    e.local = e.owner == rank;
    if (!e.local) {
        const int nro = slab_row0(e.owner + 1, H, nb) - slab_row0(e.owner, H, nb);
        if (e.lrow == 0) e.zsel = 0;
        else if (e.lrow == nro - 1) e.zsel = 1;
        else { e.mul = 0.0; e.local = 1; e.lrow = 0; atomicCAS(error, 0, 3); }   // excluded by the host check
    }
    return e;
}

// The CTA's two slab edges, kept in shared memory (read by the edge threads
// only, so they hold no registers in the others).
struct EdgePair {
    const double *zrow[2];   // owner's boundary z row (remote edges)
    const double *prow[2];   // owner's direction row in buffer 0 (remote edges)
    double mul[2];           // 0: the neighbour value is zero
    int local[2];            // 1: the source row is in this slab
    int lrow[2];             // local source row (local edges)
};

// Fills `ep` (thread 0) for the rows below (b0) and above (b1) the slab.
__device__ inline void edge_pair(cg::cluster_group &cl, EdgePair &ep, double *zb, double *pb, const AxisMap &ym, int rj0,
                                 int H, int nb, int rank, int b0, int b1, int W, int Wp, int *error)
{
    const int bs[2] = {b0, b1};
    for (int q = 0; q < 2; q++) {
        const SlabEdge e = slab_edge(ym.src, ym.mul, rj0, H, nb, rank, bs[q], error);
        ep.mul[q] = e.mul;
        ep.local[q] = e.local;
        ep.lrow[q] = e.lrow;
        ep.zrow[q] = cl.map_shared_rank(zb, e.owner) + e.zsel * W;
        ep.prow[q] = cl.map_shared_rank(pb, e.owner) + e.lrow * Wp + 1;
    }
}

// Column source of the east/west neighbour a (range coordinates) of a thread.
__device__ inline int col_source(const int *xsrc, const double *xmul, int ri0, int W, int a, double &mul)
{
    if (a >= 0 && a < W) { mul = 1.0; return a; }
    const int g = ri0 + a;
    const int s = xsrc[g + NG];
    mul = xmul[g + NG];
    if (mul == 0.0 || s < ri0 || s >= ri0 + W) { mul = 0.0; return 0; }
    return s - ri0;
}

// Sum of NV values over the cluster.  Lane 0 of warp 0 then runs `post` on
// the totals (the iteration's uniform scalar arithmetic: one thread per CTA
// instead of all of them) and every thread of every CTA receives the same
// four results in `out`.
template <int NT, int NV, class Post>
__device__ __forceinline__ void cluster_reduce(cg::cluster_group &cl, const double (&v)[NV], double (*slots)[2], int slot,
                                               double (&out)[4], Post post)
{
    constexpr int NW = NT / 32;
    __shared__ double sh[NW][2];
    __shared__ double res[4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double w[NV];
#pragma unroll
    for (int n = 0; n < NV; n++) {
        w[n] = v[n];
        for (int o = 16; o > 0; o >>= 1) w[n] += __shfl_down_sync(0xffffffffu, w[n], o);
    }
    if (lane == 0)
#pragma unroll
        for (int n = 0; n < NV; n++) sh[warp][n] = w[n];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int n = 0; n < NV; n++) {
            double x = (lane < NW) ? sh[lane][n] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) slots[slot][n] = x;
        }
    }
    cl.sync();
    if (warp == 0) {
        const unsigned nb = cl.num_blocks();
        double t[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int n = 0; n < NV; n++) {
            double x = 0.0;
            if ((unsigned)lane < nb) x = cl.map_shared_rank(&slots[slot][n], lane)[0];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            t[n] = x;
        }
        if (lane == 0) {
            post(t);
            res[0] = t[0]; res[1] = t[1]; res[2] = t[2]; res[3] = t[3];
        }
    }
    __syncthreads();
    out[0] = res[0]; out[1] = res[1]; out[2] = res[2]; out[3] = res[3];
}

// Thread's place in the column-strip layout of a W x H range.
struct Strip {
    int nb, rank;        // cluster size, CTA rank
    int j0, NR, NRmax;   // slab: first range row, rows, max rows over CTAs
    int col;             // thread's column (range coordinates)
    int r0, nr;          // thread's strip: local rows [r0, r0 + nr)
};

template <int NT>
__device__ inline Strip strip_of(int W, int H, int nb, int rank)
{
    Strip s;
    s.nb = nb;
    s.rank = rank;
    s.j0 = slab_row0(rank, H, nb);
    s.NR = slab_row0(rank + 1, H, nb) - s.j0;
    s.NRmax = (H + nb - 1) / nb;
    const int nband = NT / W;
    const int used = min(nband, s.NR);
    const int band = threadIdx.x / W;
    s.col = threadIdx.x - band * W;
    if (band < used) {
        s.r0 = (band * s.NR) / used;
        s.nr = ((band + 1) * s.NR) / used - s.r0;
    } else {
        s.r0 = 0;
        s.nr = 0;
    }
    return s;
}

// The direction buffers keep one ghost column on each side of a row
// (pitch W + 2, column c at c + 1): the thread owning the source column of a
// ghost writes it, times the ghost map's multiplier, with its own cells, so
// east and west neighbours are plain shared-memory reads.
struct GhostCols {
    double mL, mR;       // multipliers (0: the ghost stays zero)
    int sL, sR;          // source columns
};

__device__ inline GhostCols ghost_cols(const AxisMap &xm, int ri0, int W)
{
    GhostCols g;
    g.sL = col_source(xm.src, xm.mul, ri0, W, -1, g.mL);
    g.sR = col_source(xm.src, xm.mul, ri0, W, W, g.mR);
    return g;
}

// ===========================================================================
// Pressure
// ===========================================================================
template <int NT, int CPT, bool AXI>
__global__ void __launch_bounds__(NT, 1) k_cgs_pressure(PresArgs A)
{
    cg::cluster_group cl = cg::this_cluster();
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY;
    const int W = NX - 1, H = NY - 1, Wp = W + 2;
    const Strip s = strip_of<NT>(W, H, (int)cl.num_blocks(), (int)cl.block_rank());
    const int NRmax = s.NRmax, ci = s.col, nr = s.nr, r0 = s.r0, NR = s.NR;

    extern __shared__ double smem[];
    double *pb = smem;                        // direction, two buffers [2][NRmax][Wp]
    double *cxm = pb + 2 * NRmax * Wp;        // per-cell x coefficients [NRmax][W]
    double *cxp = cxm + NRmax * W;
    double *cy = cxp + NRmax * W;             // y faces 0..NR of the slab [(NRmax+1)][W]
    double *zb = cy + (NRmax + 1) * W;        // z of the slab's first and last rows [2][W]
    double *phs = zb + 2 * W;                 // solution [NRmax][W]
    __shared__ double slots[4][2];

    for (int q = threadIdx.x; q < 2 * NRmax * Wp; q += NT) pb[q] = 0.0;   // first previous direction, zero ghosts
    double rr[CPT], mr[CPT], pd[CPT], ad[CPT];
    double sg = 0.0;
    const double rw = AXI ? d.m.r_c[ci] : 1.0;  // row_weight
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        rr[k] = mr[k] = pd[k] = ad[k] = 0.0;
        if (k >= nr) continue;
        const int lr = r0 + k, i = ci, j = s.j0 + lr;
        // face coefficients (TwodOps_build_scalar_face_coeffs, psolve_cg.c:330-337)
        double r0v = AT_(A.rho, i, j);
        double bxp = 2.0 / (r0v + AT_(A.rho, i + 1, j));
        double bxm = 2.0 / (r0v + AT_(A.rho, i - 1, j));
        double byp = 2.0 / (r0v + AT_(A.rho, i, j + 1));
        double bym = 2.0 / (r0v + AT_(A.rho, i, j - 1));
        double a, b, c2, e;
        face_coeffs(d, i, bxm, bxp, bym, byp, a, b, c2, e);
        cxm[lr * W + ci] = a;
        cxp[lr * W + ci] = b;
        if (lr == 0) cy[ci] = c2;               // cym of a row = cyp of the row below
        cy[(lr + 1) * W + ci] = e;
        // initial residual r = rhs - A phi (phi with its ghost update); the
        // axisymmetric right-hand side carries the operator's row weight r_c
        // (as psolve_hypre.c:184-200 forms it; the reference's in-tree CG
        // leaves it out and its projection then diverges)
        double ad0 = pressure_op(d, A.rho, i, j, [&](int x, int y) { return remap(A.mp, A.phi, P, NX, NY, x, y); });
        double rv = (AXI ? AT_(A.rhs, i, j) * rw : AT_(A.rhs, i, j)) - ad0;
        double m = AT_(A.M, i, j);
        double z = rv * m;
        rr[k] = rv;
        phs[lr * W + ci] = AT_(A.phi, i, j);
        mr[k] = m;
        if (lr == 0) zb[ci] = z;
        if (lr == NR - 1) zb[W + ci] = z;
        sg += rv * z;
    }
    double out[4];
    double gamma = 0.0, gamma_new = 0.0;
    {
        const double v1[1] = {sg};
        cluster_reduce<NT>(cl, v1, slots, 0, out, [](double *t) {});
        gamma = out[0];
    }
    if (sqrt(gamma) < A.tol) {
        cl.sync();
        if (s.rank == 0 && threadIdx.x == 0) { A.scal->p_iters = 0; A.scal->p_res = sqrt(gamma); }
        return;
    }
    __shared__ EdgePair ep;
    __shared__ GhostCols gcs;
    if (threadIdx.x == 0) {
        edge_pair(cl, ep, zb, pb, A.mp.y, 0, H, s.nb, s.rank, s.j0 - 1, s.j0 + NR, W, Wp, &A.scal->error);
        gcs = ghost_cols(A.mp.x, 0, W);
    }
    __syncthreads();
    // bit 0/1: writes the left/right ghost column; bit 2/3: first/last band of the slab
    const int role = (nr > 0 && gcs.mL != 0.0 && ci == gcs.sL ? 1 : 0) | (nr > 0 && gcs.mR != 0.0 && ci == gcs.sR ? 2 : 0) |
                     (nr > 0 && r0 == 0 ? 4 : 0) | (nr > 0 && r0 + nr == NR ? 8 : 0);

    int cur = 0, iters, slot = 1;
    double beta = 0.0, res_final = 0.0;
    for (iters = 1; iters <= A.maxit; iters++) {
        double *pnew = pb + (1 - cur) * NRmax * Wp;
        const int off = cur * NRmax * Wp;
        // d = z + beta d (z = M r; the first direction is z: beta = 0, d = 0)
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            double *row = pnew + (r0 + k) * Wp;
            pd[k] = rr[k] * mr[k] + beta * pd[k];
            row[ci + 1] = pd[k];
            if (role & 1) row[0] = gcs.mL * pd[k];
            if (role & 2) row[W + 1] = gcs.mR * pd[k];
        }
        // rows outside the slab owned by other CTAs: z + beta d from their memory
        double dS0 = 0.0, dN0 = 0.0;   // south of the strip's first row, north of its last
        if ((role & 4) && !ep.local[0] && ep.mul[0] != 0.0) dS0 = ep.mul[0] * (ep.zrow[0][ci] + beta * ep.prow[0][off + ci]);
        if ((role & 8) && !ep.local[1] && ep.mul[1] != 0.0) dN0 = ep.mul[1] * (ep.zrow[1][ci] + beta * ep.prow[1][off + ci]);
        __syncthreads();
        if (nr > 0) {
            if (r0 > 0) dS0 = pnew[(r0 - 1) * Wp + ci + 1];
            else if (ep.local[0] && ep.mul[0] != 0.0) dS0 = ep.mul[0] * pnew[ep.lrow[0] * Wp + ci + 1];
            if (r0 + nr < NR) dN0 = pnew[(r0 + nr) * Wp + ci + 1];
            else if (ep.local[1] && ep.mul[1] != 0.0) dN0 = ep.mul[1] * pnew[ep.lrow[1] * Wp + ci + 1];
        }
        double sdad = 0.0;
        double cyS = nr > 0 ? cy[r0 * W + ci] : 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            const int lr = r0 + k;
            const double *row = pnew + lr * Wp + ci + 1;
            const double c = pd[k];
            const double dE = row[1], dW = row[-1];
            const double dN = (k + 1 < CPT && k + 1 < nr) ? pd[k + 1 < CPT ? k + 1 : k] : dN0;
            const double dS = k > 0 ? pd[k > 0 ? k - 1 : 0] : dS0;
            const double cyN = cy[(lr + 1) * W + ci];
            // Pressure_operator_variableCoeff (psolve_cg.c:302-344)
            double val = cxp[lr * W + ci] * (dE - c) - cxm[lr * W + ci] * (c - dW) + cyN * (dN - c) - cyS * (c - dS);
            const double a = AXI ? rw * val : val;
            ad[k] = a;
            sdad += c * a;
            cyS = cyN;
        }
        {
            const double v1[1] = {sdad};
            const double g = gamma;
            cluster_reduce<NT>(cl, v1, slots, slot, out, [g](double *t) { t[0] = g / (t[0] + 1e-30); });
        }
        slot = (slot + 1) & 3;
        const double alpha = out[0];
        double sgn = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            const int lr = r0 + k;
            phs[lr * W + ci] += alpha * pd[k];
            rr[k] -= alpha * ad[k];
            const double z = rr[k] * mr[k];
            if (lr == 0) zb[ci] = z;
            if (lr == NR - 1) zb[W + ci] = z;
            sgn += rr[k] * z;
        }
        {
            const double v1[1] = {sgn};
            const double g = gamma, tol = A.tol;
            cluster_reduce<NT>(cl, v1, slots, slot, out, [g, tol](double *t) {
                const double gn = t[0], rs = sqrt(gn);
                t[1] = gn / (g + 1e-30);
                t[2] = rs < tol ? 1.0 : 0.0;
                t[3] = rs;
            });
        }
        slot = (slot + 1) & 3;
        gamma_new = out[0];
        res_final = out[3];
        cur = 1 - cur;
        if (out[2] != 0.0) break;
        beta = out[1];
        gamma = gamma_new;
    }
    // remove the mean (every face Neumann or periodic), psolve_cg.c:255-279
    double ssum = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; k++)
        if (k < nr) ssum += phs[(r0 + k) * W + ci];
    {
        const double v1[1] = {ssum};
        cluster_reduce<NT>(cl, v1, slots, slot, out, [](double *t) {});
    }
    const double avg = out[0] / (double)(W * H);
#pragma unroll
    for (int k = 0; k < CPT; k++)
        if (k < nr) AT_(A.phi, ci, s.j0 + r0 + k) = phs[(r0 + k) * W + ci] - avg;
    if (iters > A.maxit) iters = A.maxit;
    cl.sync();  // no CTA leaves while another may still read its shared memory
    if (s.rank == 0 && threadIdx.x == 0) { A.scal->p_iters = iters; A.scal->p_res = res_final; }
}

// ===========================================================================
// Velocity (u and v as two clusters of one launch)
// ===========================================================================

// Face viscosities of the momentum operator at (i,j): matVec and
// vel_jacobi_diag (msolve_cg.c:98-493) for the diffuse VOF.  The east face of
// a cell is the west face of its east neighbour and the north face the south
// face of its north neighbour: the expressions are identical.
__device__ __forceinline__ double vel_mu_xm(const Dom &d, int comp, const double *__restrict__ mu, int i, int j)
{
    const int P = d.P;
    if (comp == 0) return AT_(mu, i - 1, j);
    return harm(avg2(AT_(mu, i, j - 1), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i - 1, j)));
}
__device__ __forceinline__ double vel_mu_xp(const Dom &d, int comp, const double *__restrict__ mu, int i, int j)
{
    const int P = d.P;
    if (comp == 0) return AT_(mu, i, j);
    return harm(avg2(AT_(mu, i + 1, j - 1), AT_(mu, i + 1, j)), avg2(AT_(mu, i, j - 1), AT_(mu, i, j)));
}
__device__ __forceinline__ double vel_mu_ym(const Dom &d, int comp, const double *__restrict__ mu, int i, int j)
{
    const int P = d.P;
    if (comp == 0) return harm(avg2(AT_(mu, i - 1, j), AT_(mu, i, j)), avg2(AT_(mu, i - 1, j - 1), AT_(mu, i, j - 1)));
    return AT_(mu, i, j - 1);
}
__device__ __forceinline__ double vel_mu_yp(const Dom &d, int comp, const double *__restrict__ mu, int i, int j)
{
    const int P = d.P;
    if (comp == 0) return harm(avg2(AT_(mu, i - 1, j + 1), AT_(mu, i, j + 1)), avg2(AT_(mu, i - 1, j), AT_(mu, i, j)));
    return AT_(mu, i, j);
}

template <int NT, int CPT, bool AXI>
__global__ void __launch_bounds__(NT, 1) k_cgs_velocity(const __grid_constant__ VelPair V)
{
    cg::cluster_group cl = cg::this_cluster();
    const int nb = (int)cl.num_blocks();
    const VelArgs &A = V.c[blockIdx.x / nb];
    const Dom &d = A.d;
    const int P = d.P;
    const int comp = A.comp;
    const int W = A.i1 - A.i0, H = A.j1 - A.j0, Wp = W + 2;
    const Strip s = strip_of<NT>(W, H, nb, (int)cl.block_rank());
    const int NRmax = s.NRmax, ci = s.col, nr = s.nr, r0 = s.r0, NR = s.NR, i = A.i0 + ci;
    const double EPS = 1e-14;
    const double iRe = A.iRe;

    extern __shared__ double smem[];
    double *pb = smem;                        // direction, two buffers [2][NRmax][Wp]
    double *ftm = pb + 2 * NRmax * Wp;        // rho_face / (beta dt) per cell [NRmax][W]
    double *dgm = ftm + NRmax * W;            // Jacobi diagonal + EPS per cell
    double *fx = dgm + NRmax * W;             // x-face viscosities [NRmax][W+1]
    double *fy = fx + NRmax * (W + 1);        // y-face viscosities [NRmax+1][W]
    double *zb = fy + (NRmax + 1) * W;        // z of the slab's first and last rows [2][W]
    double *rowc = zb + 2 * W;                // per-row metrics [NRmax][3]
    __shared__ double slots[4][2];

    // column metrics (TwodOps_u_cv_x_flux_divergence and friends, TwodOps.c:231-309)
    double ixe, ixw, icx, rce = 0.0, rcw = 0.0, iru = 0.0;
    if (comp == 0) {
        ixe = d.m.idx_u[i]; ixw = d.m.idx_u[i - 1]; icx = d.m.idx_c[i - 1];
        if (AXI) { rce = d.m.r_c[i]; rcw = d.m.r_c[i - 1]; iru = d.m.inv_r_u[i]; }
    } else {
        ixe = d.m.idx_c[i]; ixw = d.m.idx_c[i - 1]; icx = d.m.idx_u[i];
        if (AXI) { rce = d.m.r_u[i + 1]; rcw = d.m.r_u[i]; iru = d.m.inv_r_c[i]; }
    }

    for (int q = threadIdx.x; q < 2 * NRmax * Wp; q += NT) pb[q] = 0.0;   // first previous direction, zero ghosts
    double xv[CPT], rr[CPT], pd[CPT], ad[CPT];
    double srz = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        xv[k] = rr[k] = pd[k] = ad[k] = 0.0;
        if (k >= nr) continue;
        const int lr = r0 + k, j = A.j0 + s.j0 + lr;
        if (ci == 0) {
            if (comp == 0) { rowc[3 * lr] = d.m.idy_c[j]; rowc[3 * lr + 1] = d.m.idy_c[j - 1]; rowc[3 * lr + 2] = d.m.idy_v[j]; }
            else { rowc[3 * lr] = d.m.idy_v[j]; rowc[3 * lr + 1] = d.m.idy_v[j - 1]; rowc[3 * lr + 2] = d.m.idy_c[j - 1]; }
        }
        const double rf = comp == 0 ? 0.5 * (AT_(A.rho, i, j) + AT_(A.rho, i - 1, j))
                                    : 0.5 * (AT_(A.rho, i, j) + AT_(A.rho, i, j - 1));
        ftm[lr * W + ci] = rf / A.alpha_dt;
        const double dg = vel_diag(d, comp, A.rho, A.mu, i, j, iRe, A.alpha_dt) + EPS;
        dgm[lr * W + ci] = dg;
        fx[lr * (W + 1) + ci] = vel_mu_xm(d, comp, A.mu, i, j);
        if (ci == W - 1) fx[lr * (W + 1) + W] = vel_mu_xp(d, comp, A.mu, i, j);
        fy[lr * W + ci] = vel_mu_ym(d, comp, A.mu, i, j);
        if (lr == NR - 1) fy[(lr + 1) * W + ci] = vel_mu_yp(d, comp, A.mu, i, j);
        // r = rhs - A x, z = r / diag (msolve_cg.c:628-643)
        const double ad0 = vel_op(d, comp, A.rho, A.mu, i, j, iRe, A.alpha_dt, [&](int a, int b) { return AT_(A.x, a, b); });
        const double rv = AT_(A.rhs, i, j) - ad0;
        const double dv = rv / dg;
        rr[k] = rv;
        xv[k] = AT_(A.x, i, j);
        if (lr == 0) zb[ci] = dv;
        if (lr == NR - 1) zb[W + ci] = dv;
        srz += rv * dv;
    }
    double out[4];
    double rz;
    {
        const double v1[1] = {srz};
        cluster_reduce<NT>(cl, v1, slots, 0, out, [](double *t) {});
        rz = out[0];
    }

    __shared__ EdgePair ep;
    __shared__ GhostCols gcs;
    if (threadIdx.x == 0) {
        edge_pair(cl, ep, zb, pb, A.mcg.y, A.j0, H, nb, s.rank, A.j0 + s.j0 - 1, A.j0 + s.j0 + NR, W, Wp, &A.scal->error);
        gcs = ghost_cols(A.mcg.x, A.i0, W);
    }
    __syncthreads();
    const int role = (nr > 0 && gcs.mL != 0.0 && ci == gcs.sL ? 1 : 0) | (nr > 0 && gcs.mR != 0.0 && ci == gcs.sR ? 2 : 0) |
                     (nr > 0 && r0 == 0 ? 4 : 0) | (nr > 0 && r0 + nr == NR ? 8 : 0);

    double RMS = 0.0, beta = 0.0;
    int iters = 0, cur = 0, slot = 1;
    while (iters < A.maxit) {
        iters++;
        double *pnew = pb + (1 - cur) * NRmax * Wp;
        const int off = cur * NRmax * Wp;
        // d = M^-1 r + beta d (the first direction is M^-1 r: beta = 0, d = 0)
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            const int lr = r0 + k;
            double *row = pnew + lr * Wp;
            pd[k] = rr[k] / dgm[lr * W + ci] + beta * pd[k];
            row[ci + 1] = pd[k];
            if (role & 1) row[0] = gcs.mL * pd[k];
            if (role & 2) row[W + 1] = gcs.mR * pd[k];
        }
        double xS0 = 0.0, xN0 = 0.0;
        if ((role & 4) && !ep.local[0] && ep.mul[0] != 0.0) xS0 = ep.mul[0] * (ep.zrow[0][ci] + beta * ep.prow[0][off + ci]);
        if ((role & 8) && !ep.local[1] && ep.mul[1] != 0.0) xN0 = ep.mul[1] * (ep.zrow[1][ci] + beta * ep.prow[1][off + ci]);
        __syncthreads();
        if (nr > 0) {
            if (r0 > 0) xS0 = pnew[(r0 - 1) * Wp + ci + 1];
            else if (ep.local[0] && ep.mul[0] != 0.0) xS0 = ep.mul[0] * pnew[ep.lrow[0] * Wp + ci + 1];
            if (r0 + nr < NR) xN0 = pnew[(r0 + nr) * Wp + ci + 1];
            else if (ep.local[1] && ep.mul[1] != 0.0) xN0 = ep.mul[1] * pnew[ep.lrow[1] * Wp + ci + 1];
        }
        double sdad = 0.0;
        double mym = nr > 0 ? fy[r0 * W + ci] : 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            const int lr = r0 + k;
            const double *row = pnew + lr * Wp + ci + 1;
            const double c = pd[k];
            const double xE = row[1], xW = row[-1];
            const double xN = (k + 1 < CPT && k + 1 < nr) ? pd[k + 1 < CPT ? k + 1 : k] : xN0;
            const double xS = k > 0 ? pd[k > 0 ? k - 1 : 0] : xS0;
            const double mxm = fx[lr * (W + 1) + ci], mxp = fx[lr * (W + 1) + ci + 1];
            const double myp = fy[(lr + 1) * W + ci];
            const double iyn = rowc[3 * lr], iys = rowc[3 * lr + 1], iyv = rowc[3 * lr + 2];
            // matVec (msolve_cg.c:255-493), diffuse VOF
            const double Ax = ftm[lr * W + ci] * c;
            const double fxp = mxp * (xE - c) * ixe;
            const double fxm = mxm * (c - xW) * ixw;
            const double fyp = myp * (xN - c) * iyn;
            const double fym = mym * (c - xS) * iys;
            double op = 0.0;
            const double xd = AXI ? (rce * fxp - rcw * fxm) * icx * iru : (fxp - fxm) * icx;
            op += iRe * xd;
            op += iRe * (fyp - fym) * iyv;
            if (comp == 0) op += AXI ? -2.0 * (iRe * 0.5 * (mxp + mxm)) * c * iru * iru : 0.0;
            const double a = Ax - op;
            ad[k] = a;
            sdad += c * a;
            mym = myp;
        }
        {
            const double v1[1] = {sdad};
            const double g = rz;
            const double se = A.step_eps;
            cluster_reduce<NT>(cl, v1, slots, slot, out, [g, se](double *t) { t[0] = g / (t[0] + se); });
        }
        slot = (slot + 1) & 3;
        const double alpha = out[0];
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            if (k >= nr) continue;
            const int lr = r0 + k;
            xv[k] += alpha * pd[k];
            rr[k] -= alpha * ad[k];
            const double ri = rr[k], dg = dgm[lr * W + ci];
            if (lr == 0) zb[ci] = ri / dg;
            if (lr == NR - 1) zb[W + ci] = ri / dg;
            s0 += ri * ri / dg;
            s1 += ri * ri;
        }
        {
            const double v2[2] = {s0, s1};
            const double g = rz, in_tot = A.in_tot, tol = A.tol;
            const double se = A.step_eps;
            cluster_reduce<NT>(cl, v2, slots, slot, out, [g, in_tot, tol, se](double *t) {
                const double rms = sqrt(in_tot * t[1]);
                t[1] = t[0] / (g + se);
                t[2] = rms < tol ? 1.0 : 0.0;
                t[3] = rms;
            });
        }
        slot = (slot + 1) & 3;
        cur = 1 - cur;
        RMS = out[3];
        if (out[2] != 0.0) break;
        beta = out[1];
        rz = out[0];
    }
#pragma unroll
    for (int k = 0; k < CPT; k++)
        if (k < nr) AT_(A.x, i, A.j0 + s.j0 + r0 + k) = xv[k];
    cl.sync();  // no CTA leaves while another may still read its shared memory
    if (s.rank == 0 && threadIdx.x == 0) { A.scal->vel_iters[comp] = iters; A.scal->vel_rms[comp] = RMS; }
}

// ===========================================================================
// host side
// ===========================================================================

// Shared memory of a strip kernel of NT threads and CPT cells per thread for a
// W x H range, 0 if the range does not fit one cluster that way.
static size_t strip_smem(int W, int H, int velocity, int NT, int CPT)
{
    if (W < 1 || W > NT || H < 2 * CGC_CTAS) return 0;
    const int nb = CGC_CTAS;
    const int NRmax = (H + nb - 1) / nb;
    const int nband = NT / W;
    if ((NRmax + nband - 1) / nband > CPT) return 0;
    const size_t Wp = (size_t)W + 2, Wn = (size_t)W, R = (size_t)NRmax;
    size_t n;
    if (velocity) n = 2 * R * Wp + 2 * R * Wn + R * (Wn + 1) + (R + 1) * Wn + 2 * Wn + 3 * R;
    else n = 2 * R * Wp + 3 * R * Wn + (R + 1) * Wn + 2 * Wn;
    const size_t bytes = n * sizeof(double);
    return bytes > 220 * 1024 ? 0 : bytes;
}

// Every row just outside a slab must be read either from the slab itself or
// from the first or last row of the slab that owns it.
static bool strip_edges_ok(const std::vector<int> &ysrc, const std::vector<double> &ymul, int rj0, int H)
{
    const int nb = CGC_CTAS;
    for (int c = 0; c < nb; c++) {
        const int a = slab_row0(c, H, nb), b = slab_row0(c + 1, H, nb);
        for (int side = 0; side < 2; side++) {
            double mul;
            const int s = edge_source(ysrc.data(), ymul.data(), rj0, H, side ? rj0 + b : rj0 + a - 1, mul);
            if (s < 0) continue;
            const int o = slab_owner(s, H, nb);
            if (o == c) continue;
            const int lr = s - slab_row0(o, H, nb), nro = slab_row0(o + 1, H, nb) - slab_row0(o, H, nb);
            if (lr != 0 && lr != nro - 1) return false;
        }
    }
    return true;
}

static cudaLaunchConfig_t strip_config(int nclusters, int nt, size_t smem, cudaStream_t stream, cudaLaunchAttribute *at)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CGC_CTAS * nclusters);
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CGC_CTAS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

// The dynamic shared memory limit is an attribute of the kernel, shared by
// every context of the process: contexts of different grid sizes need
// different amounts, so the limit only ever grows (to the largest any
// context launches with; a launch with less is unaffected), under a lock, as
// contexts may be created from several threads.
bool raise_dynamic_smem(const void *fn, size_t bytes)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return false;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return true;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}

template <class K>
static bool strip_kernel_fits(K fn, int nt, size_t smem)
{
    if (!raise_dynamic_smem((const void *)fn, smem) ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = strip_config(1, nt, smem, 0, at);
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return false;
    }
    return true;
}

static bool identity_on(const std::vector<int> &src, const std::vector<double> &mul, int a, int b)
{
    for (int q = a; q < b; q++)
        if (src[q + NG] != q || mul[q + NG] != 1.0) return false;
    return true;
}

StripPlan cgs_pressure_setup(int NX, int NY, int axisym, const HostMap &mp)
{
    StripPlan plan = {0, 0};
    const int W = NX - 1, H = NY - 1;
    if (!identity_on(mp.xsrc, mp.xmul, 0, W) || !identity_on(mp.ysrc, mp.ymul, 0, H)) return plan;
    if (!strip_edges_ok(mp.ysrc, mp.ymul, 0, H)) return plan;
    size_t smem;
    // 512 threads first: the 1024-thread form spills at 64 registers per thread
    if ((smem = strip_smem(W, H, 0, 512, 8)) &&
        (axisym ? strip_kernel_fits(k_cgs_pressure<512, 8, true>, 512, smem)
                : strip_kernel_fits(k_cgs_pressure<512, 8, false>, 512, smem)))
        return StripPlan{smem, 512};
    if ((smem = strip_smem(W, H, 0, 1024, 4)) &&
        (axisym ? strip_kernel_fits(k_cgs_pressure<1024, 4, true>, 1024, smem)
                : strip_kernel_fits(k_cgs_pressure<1024, 4, false>, 1024, smem)))
        return StripPlan{smem, 1024};
    return plan;
}

cudaError_t cgs_pressure_launch(const PresArgs &A, const StripPlan &plan, cudaStream_t stream)
{
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = strip_config(1, plan.threads, plan.smem, stream, at);
    const bool axi = A.d.axisym != 0;
    if (plan.threads == 1024)
        return axi ? cudaLaunchKernelEx(&cfg, k_cgs_pressure<1024, 4, true>, A)
                   : cudaLaunchKernelEx(&cfg, k_cgs_pressure<1024, 4, false>, A);
    return axi ? cudaLaunchKernelEx(&cfg, k_cgs_pressure<512, 8, true>, A)
               : cudaLaunchKernelEx(&cfg, k_cgs_pressure<512, 8, false>, A);
}

static bool velocity_range_ok(const int r[4], const HostMap &mcg)
{
    if (!identity_on(mcg.xsrc, mcg.xmul, r[0], r[1]) || !identity_on(mcg.ysrc, mcg.ymul, r[2], r[3])) return false;
    return strip_edges_ok(mcg.ysrc, mcg.ymul, r[2], r[3] - r[2]);
}

StripPlan cgs_velocity_setup(const int ru[4], const HostMap &mu, const int rv[4], const HostMap &mv, int axisym)
{
    StripPlan plan = {0, 0};
    if (!velocity_range_ok(ru, mu) || !velocity_range_ok(rv, mv)) return plan;
    const int Wu = ru[1] - ru[0], Hu = ru[3] - ru[2], Wv = rv[1] - rv[0], Hv = rv[3] - rv[2];
    for (int nt : {1024, 512}) {
        const int cpt = nt == 1024 ? 4 : 8;
        const size_t su = strip_smem(Wu, Hu, 1, nt, cpt), sv = strip_smem(Wv, Hv, 1, nt, cpt);
        if (!su || !sv) continue;
        const size_t smem = su > sv ? su : sv;
        bool ok;
        if (nt == 1024) ok = axisym ? strip_kernel_fits(k_cgs_velocity<1024, 4, true>, nt, smem)
                                    : strip_kernel_fits(k_cgs_velocity<1024, 4, false>, nt, smem);
        else ok = axisym ? strip_kernel_fits(k_cgs_velocity<512, 8, true>, nt, smem)
                         : strip_kernel_fits(k_cgs_velocity<512, 8, false>, nt, smem);
        if (ok) return StripPlan{smem, nt};
    }
    return plan;
}

cudaError_t cgs_velocity_launch(const VelPair &V, int ncomp, const StripPlan &plan, cudaStream_t stream)
{
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = strip_config(ncomp, plan.threads, plan.smem, stream, at);
    const bool axi = V.c[0].d.axisym != 0;
    if (plan.threads == 1024)
        return axi ? cudaLaunchKernelEx(&cfg, k_cgs_velocity<1024, 4, true>, V)
                   : cudaLaunchKernelEx(&cfg, k_cgs_velocity<1024, 4, false>, V);
    return axi ? cudaLaunchKernelEx(&cfg, k_cgs_velocity<512, 8, true>, V)
               : cudaLaunchKernelEx(&cfg, k_cgs_velocity<512, 8, false>, V);
}

}  // namespace pvof
