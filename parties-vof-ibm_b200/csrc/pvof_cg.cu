// Persistent iterative solvers of the two-phase substep.
//
// Each solve is ONE cooperative launch that runs the reference's whole CG
// loop on the device: the blocks step through the iterations together,
// separated by a grid barrier, and every block reduces the per-block partial
// sums of each inner product in the same fixed order, so all blocks take the
// same convergence decisions.  Cells are assigned to threads by the same
// grid-stride mapping in every phase, so a thread reads back its own cells'
// private values (diagonal, Ad) without a barrier.
//
// Two grid barriers per iteration: the new search direction d_k = z_k +
// beta d_{k-1} is not written in a phase of its own; the matrix-vector phase
// writes it for its own cells into the second direction buffer and evaluates
// it on the fly at the stencil neighbours (from z and d_{k-1}, with the
// reference's ghost update of d applied through the same source maps).  The
// arithmetic per value is the reference's, so the iterates are those of the
// reference's loop.
//
// The grid barriers are this file's own (not cooperative_groups::grid_group::
// sync) so that their waits are bounded: if the other blocks never arrive
// they record an error in DevScalars::error and every block leaves the
// solver.  The context's solvers count arrivals on a counter that the host
// zeroes before each launch (grid_barrier_counted: a fence, one atomic and
// the poll that sees the total); the no-allocation entry point's pressure
// solve keeps the generation barrier (grid_barrier), which needs no reset.
#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

constexpr unsigned long long BARRIER_SPIN_LIMIT = 1ull << 26;

struct GridSync {
    DevScalars *s;
    unsigned nblocks;
};

// Returns false (in every thread of the block) when the barrier gave up.
__device__ __noinline__ bool grid_barrier(const GridSync &gs)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &gs.s->bar_gen;
        volatile int *verr = &gs.s->error;
        int good = (*verr == 0);
        unsigned g = *vgen;
        __threadfence();
        unsigned arrived = atomicAdd(&gs.s->bar_count, 1u);
        if (arrived == gs.nblocks - 1) {
            gs.s->bar_count = 0u;
            __threadfence();
            atomicAdd(&gs.s->bar_gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (*vgen == g) {
                ++spins;
                if ((spins & 1023ull) == 0 && (*verr != 0 || spins > BARRIER_SPIN_LIMIT)) {
                    atomicCAS(&gs.s->error, 0, 1);   // 1: a grid-wide solver's barrier
                    good = 0;
                    break;
                }
                if (spins > 4096) __nanosleep(64);
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Grid barrier on a counter of arrivals that the host zeroes before the
// launch: the g-th barrier of a launch is passed once the counter reaches
// g * gridDim.x.  Each block's thread 0 publishes the block's writes
// (block barrier, then a device-scope fence), adds its arrival without
// waiting for the result and polls the counter; nothing is reset or bumped
// after the last arrival, so the barrier costs a fence, one atomic and the
// poll that sees the total.  Bounded like grid_barrier: false (in every
// thread of the block) when it gave up, with the error recorded.
__device__ __noinline__ bool grid_barrier_counted(unsigned long long *arrivals, int *error, unsigned long long target)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned long long *va = arrivals;
        volatile int *verr = error;
        int good = 1;
        __threadfence();
        atomicAdd(arrivals, 1ull);
        unsigned long long spins = 0;
        while (*va < target) {
            ++spins;
            if ((spins & 1023ull) == 0 && (*verr != 0 || spins > BARRIER_SPIN_LIMIT)) {
                atomicCAS(error, 0, 1);   // 1: a grid-wide solver's barrier
                good = 0;
                break;
            }
            if (spins > 4096) __nanosleep(64);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// The counting barrier of one launch: the launch's g-th call waits for
// g * gridDim.x arrivals.
struct CountedSync {
    DevScalars *s;
    unsigned long long target;
    __device__ bool sync()
    {
        target += gridDim.x;
        return grid_barrier_counted(&s->bar_arrivals, &s->error, target);
    }
};

// sum of v over the block (1D blocks, multiple of 32 threads)
__device__ double block_sum(double v)
{
    __shared__ double sh[32];
    __shared__ double res;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (lane == 0) res = w;
    }
    __syncthreads();
    return res;
}

// Sum of the per-block partials, identical in every block.  Each reduction
// uses its own slot of the partials buffer; a slot is rewritten only after at
// least one more barrier has passed since every block read it.
__device__ double grid_total(const double *part)
{
    __shared__ double res;
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (unsigned q = threadIdx.x; q < gridDim.x; q += 32) v += part[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) res = v;
    }
    __syncthreads();
    double r = res;
    __syncthreads();
    return r;
}

__device__ __forceinline__ void put_partial(double *part, double v)
{
    double s = block_sum(v);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

struct Range {
    int i0, j0, w, n;
    __device__ __forceinline__ void ij(int q, int &i, int &j) const { i = i0 + q % w; j = j0 + q / w; }
};

// source of (i,j) under a ghost map (identity in the interior)
__device__ __forceinline__ void src_of(const BcMap &m, int NX, int NY, int i, int j, int &si, int &sj, double &mul)
{
    if (i >= 1 && i <= NX - 2 && j >= 1 && j <= NY - 2) {
        si = i; sj = j; mul = 1.0;
        return;
    }
    si = m.x.src[i + NG];
    sj = m.y.src[j + NG];
    mul = m.x.mul[i + NG] * m.y.mul[j + NG];
}

// ---------------------------------------------------------------------------
// diffuse_solve_biharmonic_pcg (Eulerian/VOF_DIFFUSE.c:339-429): CG on
// [a_dt I + bih L.L] x = b.  The reference iterates over the G range, whose
// half cells (i = NX-1, j = NY-1) hold exact copies of their boundary source
// cells at every iteration; here every physical cell carries the summed
// measure W of itself and its copies, and both Laplacians of the operator are
// evaluated on the fly (with the scalar ghost update in between), so one
// iteration needs two grid barriers.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_cg_biharmonic(BihArgs A)
{
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY;
    CountedSync gs{A.scal, 0};
    const Range R{0, 0, NX - 1, (NX - 1) * (NY - 1)};
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const double nk = (double)d.nk;
    double *part0 = A.partials, *part1 = A.partials + gridDim.x;
    double *part2 = A.partials + 2 * gridDim.x, *part3 = A.partials + 3 * gridDim.x;

    // L(L(f)) at (i,j) for a field given at sources: lap of the ghost-updated
    // Laplacian of the ghost-updated f (VOF_DIFFUSE_compute_laplacian twice)
    auto bilap = [&](int i, int j, auto fsrc) {
        auto fv = [&](int a, int b) {
            int si, sj;
            double mul;
            src_of(A.msc, NX, NY, a, b, si, sj, mul);
            return fsrc(si, sj);
        };
        auto lapv = [&](int a, int b) {
            int si, sj;
            double mul;
            src_of(A.msc, NX, NY, a, b, si, sj, mul);
            return lap_at(d, si, sj, fv);
        };
        return lap_at(d, i, j, lapv);
    };

    double sbb = 0.0, srr = 0.0;
    for (int q = tid; q < R.n; q += nth) {
        int i, j;
        R.ij(q, i, j);
        double l2 = bilap(i, j, [&](int a, int b) { return AT_(A.x, a, b); });
        double ap = A.a_dt * AT_(A.x, i, j) + A.bih * l2;
        double bv = AT_(A.b, i, j);
        double rv = bv - ap;
        AT_(A.r, i, j) = rv;
        AT_(A.p1, i, j) = rv;
        double m = d.m.wx[i] * d.m.wy[j] * d.wz;
        sbb += m * bv * bv;
        srr += m * rv * rv;
    }
    put_partial(part0, sbb);
    put_partial(part1, srr);
    if (!gs.sync()) return;
    double rhs_norm = sqrt(nk * grid_total(part0));
    if (rhs_norm < 1e-30) rhs_norm = 1.0;
    double rz = nk * grid_total(part1);
    double rel = sqrt(rz) / rhs_norm;
    int iter = 0;
    if (rel < A.tol) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { A.scal->ch_iters = 0; A.scal->ch_rel = rel; }
        return;
    }
    double *pcur = A.p1, *pnxt = A.p2;
    double beta = 0.0;
    bool first = true;
    while (iter < A.maxit) {
        // p = z + beta p (z = r); Ap = a_dt p + bih L(L(p))
        double spap = 0.0;
        const double bt = beta;
        const double *pold = pcur;
        for (int q = tid; q < R.n; q += nth) {
            int i, j;
            R.ij(q, i, j);
            double pv, l2;
            if (first) {
                pv = AT_(pold, i, j);
                l2 = bilap(i, j, [&](int a, int b) { return AT_(pold, a, b); });
            } else {
                pv = AT_(A.r, i, j) + bt * AT_(pold, i, j);
                AT_(pnxt, i, j) = pv;
                l2 = bilap(i, j, [&](int a, int b) { return AT_(A.r, a, b) + bt * AT_(pold, a, b); });
            }
            double ap = A.a_dt * pv + A.bih * l2;
            AT_(A.Ap, i, j) = ap;
            spap += d.m.wx[i] * d.m.wy[j] * d.wz * pv * ap;
        }
        if (!first) { double *t = pcur; pcur = pnxt; pnxt = t; }
        first = false;
        put_partial(part2, spap);
        if (!gs.sync()) return;
        double pAp = nk * grid_total(part2);
        if (fabs(pAp) < 1e-30) break;
        double alpha = rz / pAp;
        double srr2 = 0.0;
        for (int q = tid; q < R.n; q += nth) {
            int i, j;
            R.ij(q, i, j);
            AT_(A.x, i, j) += alpha * AT_(pcur, i, j);
            double rv = AT_(A.r, i, j) - alpha * AT_(A.Ap, i, j);
            AT_(A.r, i, j) = rv;
            srr2 += d.m.wx[i] * d.m.wy[j] * d.wz * rv * rv;
        }
        put_partial(part3, srr2);
        if (!gs.sync()) return;
        ++iter;
        double rr = nk * grid_total(part3);
        rel = sqrt(rr) / rhs_norm;
        if (rel < A.tol) break;
        double rz_new = rr;  // z == r: the same weighted sum
        beta = rz_new / (rz + 1e-30);
        rz = rz_new;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { A.scal->ch_iters = iter; A.scal->ch_rel = rel; }
}

// ---------------------------------------------------------------------------
// Velocity_solve_cg (Eulerian/lsolver/msolve_cg.c:525-722): Jacobi PCG with
// the RMS residual stop, one velocity component.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_cg_velocity(VelArgs A)
{
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY;
    CountedSync gs{A.scal, 0};
    const Range R{A.i0, A.j0, A.i1 - A.i0, (A.i1 - A.i0) * (A.j1 - A.j0)};
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const double EPS = 1e-14;
    double *part0 = A.partials, *part1 = A.partials + gridDim.x;
    double *part2 = A.partials + 2 * gridDim.x, *part3 = A.partials + 3 * gridDim.x;
    auto active = [&](int a, int b) { return a >= A.i0 && a < A.i1 && b >= A.j0 && b < A.j1; };

    double srz = 0.0;
    for (int q = tid; q < R.n; q += nth) {
        int i, j;
        R.ij(q, i, j);
        double dg = vel_diag(d, A.comp, A.rho, A.mu, i, j, A.iRe, A.alpha_dt) + EPS;
        AT_(A.diag, i, j) = dg;
        vel_weights(d, A.comp, A.rho, A.mu, A.ft, A.mc, i, j, A.i0, A.j0, A.alpha_dt);
        double ad = vel_op(d, A.comp, A.rho, A.mu, i, j, A.iRe, A.alpha_dt, [&](int a, int b) { return AT_(A.x, a, b); });
        double rv = AT_(A.rhs, i, j) - ad;
        AT_(A.r, i, j) = rv;
        double dv = rv / dg;
        AT_(A.dir, i, j) = dv;
        AT_(A.z, i, j) = dv;
        srz += rv * dv;
    }
    put_partial(part0, srz);
    if (!gs.sync()) return;
    double rz = grid_total(part0);
    double RMS = 0.0, beta = 0.0;
    int iters = 0;
    double *dcur = A.dir, *dnxt = A.dir2;
    bool first = true;
    while (iters < A.maxit) {
        iters++;
        // d = M^-1 r + beta d, Ad = A d with the VEL_TYPE_CG ghost update of d
        double sdad = 0.0;
        const double bt = beta;
        const double *dold = dcur;
        for (int q = tid; q < R.n; q += nth) {
            int i, j;
            R.ij(q, i, j);
            double dv, ad;
            if (first) {
                dv = AT_(dold, i, j);
                ad = vel_op_w(d, A.comp, A.ft, A.mc, A.mu, i, j, A.iRe, [&](int a, int b) {
                    int si, sj;
                    double mul;
                    src_of(A.mcg, NX, NY, a, b, si, sj, mul);
                    if (mul == 0.0 || !active(si, sj)) return 0.0;
                    return mul * AT_(dold, si, sj);
                });
            } else {
                dv = AT_(A.z, i, j) + bt * AT_(dold, i, j);
                AT_(dnxt, i, j) = dv;
                ad = vel_op_w(d, A.comp, A.ft, A.mc, A.mu, i, j, A.iRe, [&](int a, int b) {
                    int si, sj;
                    double mul;
                    src_of(A.mcg, NX, NY, a, b, si, sj, mul);
                    if (mul == 0.0 || !active(si, sj)) return 0.0;
                    return mul * (AT_(A.z, si, sj) + bt * AT_(dold, si, sj));
                });
            }
            AT_(A.Ad, i, j) = ad;
            sdad += dv * ad;
        }
        if (!first) { double *t = dcur; dcur = dnxt; dnxt = t; }
        first = false;
        put_partial(part1, sdad);
        if (!gs.sync()) return;
        double dAd = grid_total(part1);
        double alpha = rz / (dAd + A.step_eps);
        double s0 = 0.0, s1 = 0.0;
        for (int q = tid; q < R.n; q += nth) {
            int i, j;
            R.ij(q, i, j);
            AT_(A.x, i, j) += alpha * AT_(dcur, i, j);
            double ri = AT_(A.r, i, j) - alpha * AT_(A.Ad, i, j);
            AT_(A.r, i, j) = ri;
            double dg = AT_(A.diag, i, j);
            AT_(A.z, i, j) = ri / dg;
            s0 += ri * ri / dg;
            s1 += ri * ri;
        }
        put_partial(part2, s0);
        put_partial(part3, s1);
        if (!gs.sync()) return;
        double rz_new = grid_total(part2), rr = grid_total(part3);
        RMS = sqrt(A.in_tot * rr);
        if (RMS < A.tol) break;
        beta = rz_new / (rz + A.step_eps);
        rz = rz_new;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { A.scal->vel_iters[A.comp] = iters; A.scal->vel_rms[A.comp] = RMS; }
}

// ---------------------------------------------------------------------------
// Pressure_solve_cg (Eulerian/lsolver/psolve_cg.c:130-293): Jacobi PCG on the
// variable-density Poisson operator, absolute stop on sqrt(r.M^-1 r), mean
// removed at the end.
//
// FW (the context's solve): the operator's face weights 2 / (rho_P + rho_N)
// are computed once, in the set-up phase, into the planes A.bx / A.by, so an
// iteration multiplies instead of dividing four times per cell; without FW
// (the no-allocation entry point, which has no room for the planes) they are
// computed from rho at every application.  The pressure ghost rules copy
// with weight 1 (psolve_cg.c:374-460: Neumann copies, periodic wrap) and
// leave the solve range [0, NX-2] x [0, NY-2] unmapped, so a neighbour's
// source differs from it only at the four ends of the axes: those sources
// are read once from the maps and the stencil is gathered without branches.
// The FW form also uses counting grid barriers (grid_barrier_counted; the
// host zeroes the counter before the launch).  DEFER: the update
// phi += alpha d of an iteration is applied in the next iteration's direction
// pass, which reads d at the cell anyway (the same operands and operation,
// one pass later; before the mean removal after the last iteration), so the
// update pass reads three planes instead of five.  U1: cells per loop trip
// of the direction pass (the update pass takes two), their loads issued
// before either cell's stores.  Measured per iteration on B200 (the same
// results bit for bit in every form): 1024x1024 31.7 us for the plain form
// (without FW), 20.8 us for FW with DEFER and U1 = 1, which the context
// uses; 2048x2048 154 and 96.6 us; 256x512 10.7 and 8.2 us.  At 64
// registers (two 512-thread blocks per SM) U1 = 2 with DEFER loses loads in
// flight and ran 16% slower at 2048x2048.  PAIR (k_cg_pressure_fwp): both
// passes over pairs of neighbouring cells with 16-byte accesses, for ranges
// of at least two cells per resident thread (the context picks it by size):
// 2048x2048 94.0 -> 86.9 us, 1024x1024 20.7 -> 19.9 us.
// ---------------------------------------------------------------------------
template <bool FW, bool DEFER, int U1, bool PAIR>
__device__ __forceinline__ void cg_pressure(const PresArgs &A)
{
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY;
    const GridSync gs{A.scal, gridDim.x};
    const Range R{0, 0, NX - 1, (NX - 1) * (NY - 1)};
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    double *part0 = A.partials, *part1 = A.partials + gridDim.x, *part2 = A.partials + 2 * gridDim.x;
    // sources of the neighbours beyond the ends of the solve range
    const int xw = A.mp.x.src[NG - 1], xe = A.mp.x.src[NX - 1 + NG];
    const int ys = A.mp.y.src[NG - 1], yn = A.mp.y.src[NY - 1 + NG];
    const double *__restrict__ rho = A.rho;
    const double *__restrict__ bx = A.bx;
    const double *__restrict__ by = A.by;
    CountedSync cs{A.scal, 0};
    auto barrier = [&]() { return FW ? cs.sync() : grid_barrier(gs); };

    double sg = 0.0;
    for (int q = tid; q < R.n; q += nth) {
        int i, j;
        R.ij(q, i, j);
        if (FW) pressure_face_weights(d, rho, A.bx, A.by, i, j);
        double ad = pressure_op(d, rho, i, j, [&](int a, int b) { return remap(A.mp, A.phi, P, NX, NY, a, b); });
        // the axisymmetric right-hand side carries the row weight r_c of the
        // operator (psolve_hypre.c:184-200)
        double rv = (d.axisym ? AT_(A.rhs, i, j) * d.m.r_c[i] : AT_(A.rhs, i, j)) - ad;
        AT_(A.res, i, j) = rv;
        double z = rv * AT_(A.M, i, j);
        AT_(A.dir, i, j) = z;
        AT_(A.z, i, j) = z;
        sg += rv * z;
    }
    put_partial(part0, sg);
    if (!barrier()) return;
    double gamma = grid_total(part0), gamma_new = 0.0, beta = 0.0;
    if (sqrt(gamma) < A.tol) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { A.scal->p_iters = 0; A.scal->p_res = sqrt(gamma); }
        return;
    }

    // d = z + beta d_old at the five points of cell q (d_old alone on the
    // first iteration) and A d at the cell
    auto direction = [&](int q, bool first, const double *__restrict__ zp, const double *__restrict__ dold, double bt,
                         double &dv, double &ad) {
        int i, j;
        R.ij(q, i, j);
        const int iw = i > 0 ? i - 1 : xw, ie = i < NX - 2 ? i + 1 : xe;
        const int js = j > 0 ? j - 1 : ys, jn = j < NY - 2 ? j + 1 : yn;
        const ptrdiff_t row = (ptrdiff_t)j * P;
        const ptrdiff_t cC = row + i, cE = row + ie, cW = row + iw;
        const ptrdiff_t cN = (ptrdiff_t)jn * P + i, cS = (ptrdiff_t)js * P + i;
        double vc, ve, vw, vn, vs;
        if (first) {
            vc = dold[cC]; ve = dold[cE]; vw = dold[cW]; vn = dold[cN]; vs = dold[cS];
        } else {
            vc = zp[cC] + bt * dold[cC];
            ve = zp[cE] + bt * dold[cE];
            vw = zp[cW] + bt * dold[cW];
            vn = zp[cN] + bt * dold[cN];
            vs = zp[cS] + bt * dold[cS];
        }
        double bxm, bxp, bym, byp;
        if (FW) {
            bxm = bx[cC - 1]; bxp = bx[cC]; bym = by[cC - P]; byp = by[cC];
        } else {
            const double r0 = rho[cC];
            bxp = 2.0 / (r0 + rho[cC + 1]);
            bxm = 2.0 / (r0 + rho[cC - 1]);
            byp = 2.0 / (r0 + rho[cC + P]);
            bym = 2.0 / (r0 + rho[cC - P]);
        }
        double cxm, cxp, cym, cyp;
        face_coeffs(d, i, bxm, bxp, bym, byp, cxm, cxp, cym, cyp);
        const double val = cxp * (ve - vc) - cxm * (vc - vw) + cyp * (vn - vc) - cym * (vc - vs);
        dv = vc;
        ad = row_weight(d, i) * val;
    };

    // PAIR: the two passes over pairs of cells (2k, 2k+1) of a row with
    // 16-byte loads and stores (the planes' rows start on 16-byte boundaries
    // and i = 0 sits at an even column); a row of odd length ends in a single
    // cell, whose stores are 8 bytes wide.  The values are those of the
    // single-cell passes: the same operands in the same operations.
    const int W = NX - 1, Wp = (W + 1) / 2, Np = Wp * (NY - 1);
    auto ld2 = [](const double *p) { return *reinterpret_cast<const double2 *>(p); };
    auto st2 = [](double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); };
    auto direction_pair = [&](int p, bool first, const double *__restrict__ zp, const double *__restrict__ dold,
                              double *__restrict__ dn, double bt, double al, double &sdad) {
        const int j = p / Wp, i0 = 2 * (p - j * Wp), i1 = i0 + 1;
        const bool has1 = i1 < W;
        const int iw = i0 > 0 ? i0 - 1 : xw, ie = i0 + 2 <= NX - 2 ? i0 + 2 : xe;
        const int js = j > 0 ? j - 1 : ys, jn = j < NY - 2 ? j + 1 : yn;
        const ptrdiff_t r = (ptrdiff_t)j * P + i0, rn = (ptrdiff_t)jn * P + i0, rs = (ptrdiff_t)js * P + i0;
        const ptrdiff_t rw = (ptrdiff_t)j * P + iw, re = (ptrdiff_t)j * P + ie;
        const double2 oc = ld2(dold + r), on = ld2(dold + rn), os = ld2(dold + rs);
        const double ow = dold[rw], oe = dold[re];
        double2 vc = oc, vn = on, vs = os;
        double vw = ow, ve = oe;
        if (!first) {
            const double2 zc = ld2(zp + r), zn = ld2(zp + rn), zs = ld2(zp + rs);
            const double zw = zp[rw], ze = zp[re];
            vc = make_double2(zc.x + bt * oc.x, zc.y + bt * oc.y);
            vn = make_double2(zn.x + bt * on.x, zn.y + bt * on.y);
            vs = make_double2(zs.x + bt * os.x, zs.y + bt * os.y);
            vw = zw + bt * ow;
            ve = ze + bt * oe;
        }
        const double2 bxc = ld2(bx + r), byc = ld2(by + r), bys = ld2(by + r - P);
        const double bxw = bx[r - 1];
        double cxm, cxp, cym, cyp;
        face_coeffs(d, i0, bxw, bxc.x, bys.x, byc.x, cxm, cxp, cym, cyp);
        const double e0 = has1 ? vc.y : ve;
        const double ad0 = row_weight(d, i0) *
                           (cxp * (e0 - vc.x) - cxm * (vc.x - vw) + cyp * (vn.x - vc.x) - cym * (vc.x - vs.x));
        face_coeffs(d, i1, bxc.x, bxc.y, bys.y, byc.y, cxm, cxp, cym, cyp);
        const double ad1 = row_weight(d, i1) *
                           (cxp * (ve - vc.y) - cxm * (vc.y - vc.x) + cyp * (vn.y - vc.y) - cym * (vc.y - vs.y));
        if (has1) {
            if (DEFER && !first) {
                const double2 ph = ld2(A.phi + r);
                st2(A.phi + r, ph.x + al * oc.x, ph.y + al * oc.y);
            }
            if (!first) st2(dn + r, vc.x, vc.y);
            st2(A.Ad + r, ad0, ad1);
            sdad += vc.x * ad0;
            sdad += vc.y * ad1;
        } else {
            if (DEFER && !first) A.phi[r] = A.phi[r] + al * oc.x;
            if (!first) dn[r] = vc.x;
            A.Ad[r] = ad0;
            sdad += vc.x * ad0;
        }
    };
    auto update_pair = [&](int p, double alpha, double &sgn) {
        const int j = p / Wp, i0 = 2 * (p - j * Wp);
        const bool has1 = i0 + 1 < W;
        const ptrdiff_t r = (ptrdiff_t)j * P + i0;
        const double2 rr = ld2(A.res + r), aa = ld2(A.Ad + r), mm = ld2(A.M + r);
        const double rv0 = rr.x - alpha * aa.x, z0 = rv0 * mm.x;
        const double rv1 = rr.y - alpha * aa.y, z1 = rv1 * mm.y;
        if (has1) {
            st2(A.res + r, rv0, rv1);
            st2(A.z + r, z0, z1);
            sgn += rv0 * z0;
            sgn += rv1 * z1;
        } else {
            A.res[r] = rv0;
            A.z[r] = z0;
            sgn += rv0 * z0;
        }
    };

    double *dcur = A.dir, *dnxt = A.dir2;
    bool first = true;
    double alpha = 0.0;   // FW: the step of the update phi += alpha d_cur still to be applied
    int iters;
    for (iters = 1; iters <= A.maxit; iters++) {
        // d = z + beta d (z = M r), Ad with the pressure ghost update of d;
        // FW: phi += alpha d_old from the previous iteration at the cell
        double sdad = 0.0;
        const double bt = beta, al = alpha;
        const double *dold = dcur;
        if (PAIR)
            for (int p = tid; p < Np; p += nth) direction_pair(p, first, A.z, dold, dnxt, bt, al, sdad);
        else
        for (int q = tid; q < R.n; q += U1 * nth) {
            const int q1 = q + nth;
            const bool two = U1 == 2 && q1 < R.n;
            double dv0, ad0, dv1 = 0.0, ad1 = 0.0;
            direction(q, first, A.z, dold, bt, dv0, ad0);
            if (two) direction(q1, first, A.z, dold, bt, dv1, ad1);
            int i, j;
            R.ij(q, i, j);
            double ph0 = 0.0, do0 = 0.0, ph1 = 0.0, do1 = 0.0;
            if (DEFER && !first) {
                ph0 = AT_(A.phi, i, j); do0 = AT_(dold, i, j);
                if (two) {
                    int i1, j1;
                    R.ij(q1, i1, j1);
                    ph1 = AT_(A.phi, i1, j1); do1 = AT_(dold, i1, j1);
                }
            }
            if (!first) AT_(dnxt, i, j) = dv0;
            AT_(A.Ad, i, j) = ad0;
            if (DEFER && !first) AT_(A.phi, i, j) = ph0 + al * do0;
            sdad += dv0 * ad0;
            if (two) {
                R.ij(q1, i, j);
                if (!first) AT_(dnxt, i, j) = dv1;
                AT_(A.Ad, i, j) = ad1;
                if (DEFER && !first) AT_(A.phi, i, j) = ph1 + al * do1;
                sdad += dv1 * ad1;
            }
        }
        if (!first) { double *t = dcur; dcur = dnxt; dnxt = t; }
        first = false;
        put_partial(part1, sdad);
        if (!barrier()) return;
        alpha = gamma / (grid_total(part1) + 1e-30);
        double sgn = 0.0;
        if (PAIR)
            for (int p = tid; p < Np; p += nth) update_pair(p, alpha, sgn);
        else
        for (int q = tid; q < R.n; q += 2 * nth) {
            const int q1 = q + nth;
            const bool two = q1 < R.n;
            int i0, j0, i1 = 0, j1 = 0;
            R.ij(q, i0, j0);
            double ph0 = 0.0, dc0 = 0.0, ph1 = 0.0, dc1 = 0.0;
            if (!DEFER) { ph0 = AT_(A.phi, i0, j0); dc0 = AT_(dcur, i0, j0); }
            double r0 = AT_(A.res, i0, j0), a0 = AT_(A.Ad, i0, j0), m0 = AT_(A.M, i0, j0);
            double r1 = 0.0, a1 = 0.0, m1 = 0.0;
            if (two) {
                R.ij(q1, i1, j1);
                if (!DEFER) { ph1 = AT_(A.phi, i1, j1); dc1 = AT_(dcur, i1, j1); }
                r1 = AT_(A.res, i1, j1); a1 = AT_(A.Ad, i1, j1); m1 = AT_(A.M, i1, j1);
            }
            {
                const double rv = r0 - alpha * a0, z = rv * m0;
                if (!DEFER) AT_(A.phi, i0, j0) = ph0 + alpha * dc0;
                AT_(A.res, i0, j0) = rv;
                AT_(A.z, i0, j0) = z;
                sgn += rv * z;
            }
            if (two) {
                const double rv = r1 - alpha * a1, z = rv * m1;
                if (!DEFER) AT_(A.phi, i1, j1) = ph1 + alpha * dc1;
                AT_(A.res, i1, j1) = rv;
                AT_(A.z, i1, j1) = z;
                sgn += rv * z;
            }
        }
        put_partial(part2, sgn);
        if (!barrier()) return;
        gamma_new = grid_total(part2);
        if (sqrt(gamma_new) < A.tol) break;
        beta = gamma_new / (gamma + 1e-30);
        gamma = gamma_new;
    }
    // remove the mean (every face Neumann or periodic), psolve_cg.c:255-279;
    // FW: after the last iteration's pending update
    double ssum = 0.0;
    const bool pending = DEFER && !first;
    for (int q = tid; q < R.n; q += nth) {
        int i, j;
        R.ij(q, i, j);
        if (pending) AT_(A.phi, i, j) += alpha * AT_(dcur, i, j);
        ssum += AT_(A.phi, i, j);
    }
    put_partial(part0, ssum);
    if (!barrier()) return;
    double avg = grid_total(part0) / (double)R.n;
    for (int q = tid; q < R.n; q += nth) {
        int i, j;
        R.ij(q, i, j);
        AT_(A.phi, i, j) -= avg;
    }
    if (iters > A.maxit) iters = A.maxit;
    if (blockIdx.x == 0 && threadIdx.x == 0) { A.scal->p_iters = iters; A.scal->p_res = sqrt(gamma_new); }
}

__global__ void __launch_bounds__(512) k_cg_pressure(PresArgs A) { cg_pressure<false, false, 2, false>(A); }
__global__ void __launch_bounds__(512, 2) k_cg_pressure_fw(PresArgs A) { cg_pressure<true, true, 1, false>(A); }
__global__ void __launch_bounds__(512, 2) k_cg_pressure_fwp(PresArgs A) { cg_pressure<true, true, 1, true>(A); }

}  // namespace pvof
