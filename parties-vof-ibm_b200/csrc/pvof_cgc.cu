// Cluster-resident pressure solver for grids that fit one thread-block
// cluster (at most 16 CTAs x 512 threads x CPT cells).
//
// Pressure_solve_cg (Eulerian/lsolver/psolve_cg.c:130-293), the same Jacobi
// PCG as k_cg_pressure, restructured for the latency of a small problem:
//   * the cluster's CTAs split the physical rows into slabs; each CTA keeps
//     z = M r, the two search-direction buffers and the operator's face
//     coefficients of its slab in shared memory, and each thread keeps the
//     residual, the solution and the diagonal of its CPT cells in registers;
//   * the direction rows just outside a slab are computed from the
//     neighbouring CTA's z and previous direction through distributed shared
//     memory, so a CTA only waits for its own threads before the stencil;
//   * the two inner products of an iteration are reduced through
//     distributed shared memory behind hardware cluster barriers
//     (barrier.cluster arrive.release / wait.acquire), every CTA summing the
//     16 partials in the same order.
// Per cell and per iteration the arithmetic is the reference's: the face
// coefficients are the per-cell beta * idx^2 products of
// TwodOps_build_scalar_face_coeffs, computed once per solve because rho does
// not change during it.
#include <cooperative_groups.h>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace cg = cooperative_groups;

namespace pvof {

constexpr int CL_THREADS = 512;

// sum over the cluster of one value per thread; identical in every CTA
__device__ double cluster_sum(cg::cluster_group &cl, double v, double *slots, int slot)
{
    __shared__ double sh[CL_THREADS / 32];
    __shared__ double res;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = (lane < CL_THREADS / 32) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) slots[slot] = w;
    }
    cl.sync();
    if (warp == 0) {
        double t = 0.0;
        const unsigned nb = cl.num_blocks();
        if ((unsigned)lane < nb) t = cl.map_shared_rank(slots, lane)[slot];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) res = t;
    }
    __syncthreads();
    return res;
}

template <int CPT>
__global__ void __launch_bounds__(CL_THREADS, 1) k_cgc_pressure(PresArgs A)
{
    cg::cluster_group cl = cg::this_cluster();
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY;
    const int W = NX - 1, NYp = NY - 1;
    const int nb = (int)cl.num_blocks(), rank = (int)cl.block_rank();
    auto row0 = [&](int c) { return (int)(((long long)c * NYp) / nb); };
    const int j0 = row0(rank), j1 = row0(rank + 1), NR = j1 - j0;
    const int NRmax = (NYp + nb - 1) / nb;
    const int ncell = NR * W;

    extern __shared__ double smem[];
    double *zs = smem;                       // z = M r, own rows   [NRmax*W]
    double *dsb = zs + NRmax * W;            // direction buffers   [2][NRmax*W]
    double *cxm = dsb + 2 * NRmax * W;       // per-cell x coefficients
    double *cxp = cxm + NRmax * W;
    double *by = cxp + NRmax * W;            // y faces j0..j1      [(NRmax+1)*W]
    double *halo = by + (NRmax + 1) * W;     // direction rows j0-1 and j1 [2*W]
    __shared__ double slots[4];

    // owner CTA and local row of a physical row
    auto owner = [&](int j) {
        int c = (int)(((long long)j * nb) / NYp);
        while (c > 0 && row0(c) > j) c--;
        while (c < nb - 1 && row0(c + 1) <= j) c++;
        return c;
    };
    // pressure ghost update (Pressure_apply_BCs + exchange) along each axis
    auto sx = [&](int i) { return (i >= 0 && i < W) ? i : A.mp.x.src[i + NG]; };
    auto sy = [&](int j) { return (j >= 0 && j < NYp) ? j : A.mp.y.src[j + NG]; };

    // registers: residual, solution, diagonal, Ad of the thread's cells
    double rr[CPT], ph[CPT], mm[CPT], ad[CPT];
    double sg = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int q = threadIdx.x + k * CL_THREADS;
        rr[k] = ph[k] = mm[k] = ad[k] = 0.0;
        if (q >= ncell) continue;
        const int i = q % W, j = j0 + q / W;
        // face coefficients (TwodOps_build_scalar_face_coeffs, psolve_cg.c:330-337)
        double r0 = AT_(A.rho, i, j);
        double bxp = 2.0 / (r0 + AT_(A.rho, i + 1, j));
        double bxm = 2.0 / (r0 + AT_(A.rho, i - 1, j));
        double byp = 2.0 / (r0 + AT_(A.rho, i, j + 1));
        double bym = 2.0 / (r0 + AT_(A.rho, i, j - 1));
        double a, b, c2, e;
        face_coeffs(d, i, bxm, bxp, bym, byp, a, b, c2, e);
        cxm[q] = a;
        cxp[q] = b;
        if (q / W == 0) by[i] = c2;
        by[q + W] = e;
        // initial residual r = rhs - A phi (phi with its ghost update)
        double ad0 = pressure_op(d, A.rho, i, j, [&](int x, int y) { return remap(A.mp, A.phi, P, NX, NY, x, y); });
        double rv = AT_(A.rhs, i, j) - ad0;
        double m = AT_(A.M, i, j);
        double z = rv * m;
        rr[k] = rv;
        ph[k] = AT_(A.phi, i, j);
        mm[k] = m;
        zs[q] = z;
        dsb[q] = 0.0;
        dsb[NRmax * W + q] = 0.0;
        sg += rv * z;
    }
    double gamma = cluster_sum(cl, sg, slots, 0), gamma_new = 0.0;
    if (sqrt(gamma) < A.tol) {
        cl.sync();
        if (rank == 0 && threadIdx.x == 0) { A.scal->p_iters = 0; A.scal->p_res = sqrt(gamma); }
        return;
    }
    // rows just outside the slab: their source rows and owners
    const int jb = sy(j0 - 1), ja = sy(j1);
    const int ob = owner(jb), oa = owner(ja);
    const bool rem_b = (ob != rank), rem_a = (oa != rank);
    double *zs_b = cl.map_shared_rank(zs, ob), *zs_a = cl.map_shared_rank(zs, oa);
    double *ds_b = cl.map_shared_rank(dsb, ob), *ds_a = cl.map_shared_rank(dsb, oa);
    const int lb = jb - row0(ob), la = ja - row0(oa);

    int cur = 0, iters, slot = 1;
    double beta = 0.0;
    for (iters = 1; iters <= A.maxit; iters++) {
        double *dold = dsb + cur * NRmax * W, *dnew = dsb + (1 - cur) * NRmax * W;
        const int off = cur * NRmax * W;
        // d = z + beta d (the first direction is z: beta = 0, d_old = 0)
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            const int q = threadIdx.x + k * CL_THREADS;
            if (q < ncell) dnew[q] = zs[q] + beta * dold[q];
        }
        for (int t = threadIdx.x; t < 2 * W; t += CL_THREADS) {
            const int i = t % W;
            if (t < W) {
                if (rem_b) halo[i] = zs_b[lb * W + i] + beta * ds_b[off + lb * W + i];
            } else {
                if (rem_a) halo[W + i] = zs_a[la * W + i] + beta * ds_a[off + la * W + i];
            }
        }
        __syncthreads();
        double sdad = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            const int q = threadIdx.x + k * CL_THREADS;
            if (q >= ncell) continue;
            const int i = q % W, lr = q / W;
            const double c = dnew[q];
            const int ie = sx(i + 1), iw = sx(i - 1);
            const double dE = dnew[lr * W + ie], dW = dnew[lr * W + iw];
            double dN, dS;
            if (lr + 1 < NR) dN = dnew[q + W];
            else if (!rem_a) dN = dnew[la * W + i];
            else dN = halo[W + i];
            if (lr > 0) dS = dnew[q - W];
            else if (!rem_b) dS = dnew[lb * W + i];
            else dS = halo[i];
            // by holds cym of the cell above a face and cyp of the cell below
            double val = cxp[q] * (dE - c) - cxm[q] * (c - dW) + by[(lr + 1) * W + i] * (dN - c) - by[lr * W + i] * (c - dS);
            double a = row_weight(d, i) * val;
            ad[k] = a;
            sdad += c * a;
        }
        const double dAd = cluster_sum(cl, sdad, slots, slot);
        slot = (slot + 1) & 3;
        const double alpha = gamma / (dAd + 1e-30);
        double sgn = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; k++) {
            const int q = threadIdx.x + k * CL_THREADS;
            if (q >= ncell) continue;
            ph[k] += alpha * dnew[q];
            rr[k] -= alpha * ad[k];
            const double z = rr[k] * mm[k];
            zs[q] = z;
            sgn += rr[k] * z;
        }
        gamma_new = cluster_sum(cl, sgn, slots, slot);
        slot = (slot + 1) & 3;
        cur = 1 - cur;
        if (sqrt(gamma_new) < A.tol) break;
        beta = gamma_new / (gamma + 1e-30);
        gamma = gamma_new;
    }
    // remove the mean (every face Neumann or periodic), psolve_cg.c:255-279
    double ssum = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int q = threadIdx.x + k * CL_THREADS;
        if (q < ncell) ssum += ph[k];
    }
    const double avg = cluster_sum(cl, ssum, slots, slot) / (double)(W * NYp);
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        const int q = threadIdx.x + k * CL_THREADS;
        if (q >= ncell) continue;
        const int i = q % W, j = j0 + q / W;
        AT_(A.phi, i, j) = ph[k] - avg;
    }
    if (iters > A.maxit) iters = A.maxit;
    cl.sync();  // no CTA leaves while another may still read its shared memory
    if (rank == 0 && threadIdx.x == 0) { A.scal->p_iters = iters; A.scal->p_res = sqrt(gamma_new); }
}

// Shared memory of k_cgc_pressure for a grid, or 0 if it does not fit one
// cluster of `nb` CTAs with CPT cells per thread.
static size_t cgc_pressure_smem(int NX, int NY, int nb, int cpt)
{
    const int W = NX - 1, NYp = NY - 1;
    const int NRmax = (NYp + nb - 1) / nb;
    if ((long long)NRmax * W > (long long)CL_THREADS * cpt) return 0;
    size_t bytes = sizeof(double) * ((size_t)5 * NRmax * W + (size_t)(NRmax + 1) * W + 2 * (size_t)W);
    if (bytes > 227 * 1024) return 0;
    return bytes;
}

static cudaLaunchConfig_t cgc_config(size_t smem, cudaStream_t stream, cudaLaunchAttribute *at)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CGC_CTAS);
    cfg.blockDim = dim3(CL_THREADS);
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

size_t cgc_pressure_setup(int NX, int NY)
{
    size_t cs = cgc_pressure_smem(NX, NY, CGC_CTAS, CGC_CPT);
    if (!cs) return 0;
    auto fn = k_cgc_pressure<CGC_CPT>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs) != cudaSuccess ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = cgc_config(cs, 0, at);
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return 0;
    }
    return cs;
}

cudaError_t cgc_pressure_launch(const PresArgs &A, size_t smem, cudaStream_t stream)
{
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = cgc_config(smem, stream, at);
    return cudaLaunchKernelEx(&cfg, k_cgc_pressure<CGC_CPT>, A);
}

}  // namespace pvof
