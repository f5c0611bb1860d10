// Pressure PCG with a constant-density spectral preconditioner: a form with
// no counterpart in the reference (which preconditions Pressure_solve_cg,
// Eulerian/lsolver/psolve_cg.c:130-293, with the Jacobi diagonal).
//
// The operator is the reference's variable-density one (pressure_op,
// psolve_cg.c:302-344) with its ghost rules (Pressure_apply_BCs: x periodic,
// mirror walls in y).  The preconditioner applies the inverse of the same
// five-point operator with the density set to one, -L, which a Fourier
// transform along the periodic x rows diagonalises into one tridiagonal
// system per wavenumber along y:
//
//   1. every row j: forward complex FFT of the residual row (radix 2 in shared
//      memory, twiddles from a table), stored in FFTW's half-complex order
//      (Re X_0 .. Re X_{N/2}, Im X_{N/2-1} .. Im X_1) times dy^2 / N;
//   2. every half-complex index m: parallel cyclic reduction (one thread per
//      row, log2 M elimination rounds in shared memory) of
//        -z_{j-1} + (b_j + dy^2 lambda_x(m)) z_j - z_{j+1} = rhs_j,
//      b_j = 2 inside, 1 at the two walls; for the mean mode the first row is
//      pinned and the column's mean removed afterwards, so the constant mode,
//      the operator's null space, is projected out;
//   3. every row: inverse transform.
//
// With the density ratio rho_max / rho_min the preconditioned operator's
// condition number is at most that ratio, whatever the grid size; the
// Jacobi-PCG's grows with the square of the grid.  The stopping test is the
// reference's: sqrt(r^T D^-1 r) below P_CG_ETOL with D the Jacobi diagonal,
// so the solve stops at the same residual size; the iterates differ, so the
// result moves within that tolerance of the reference's.
//
// One PCG iteration is four launches (matrix-vector product with the new
// direction formed on the fly, update + forward row transforms, tridiagonal
// solves, inverse row transforms + inner product); each launch's last block
// (arrival counter) forms the iteration's scalars from the per-block sums in
// block order, so the arithmetic does not depend on scheduling.  A device
// flag set at convergence makes the later launches return at once; the host
// looks at it every SPEC_BATCH iterations.
#include <cmath>
#include <vector>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

namespace {

constexpr int ROW_THREADS = 128;

// sum over the block, in a fixed order; the total is valid in thread 0
__device__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < nw; k++) t += sh[k];
    return t;
}

// publish this block's sum; true in the block that arrives last, which then
// adds all the block sums in block order (result valid in its thread 0)
__device__ bool finish_sum(double v, double *part, unsigned *cnt, double *sh, double &total)
{
    __shared__ bool last;
    const double b = block_sum(v, sh);
    const unsigned nb = gridDim.x;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(cnt, 1u) == nb - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0.0;
    for (unsigned k = threadIdx.x; k < nb; k += blockDim.x) s += __ldcg(part + k);
    total = block_sum(s, sh);
    if (threadIdx.x == 0) *cnt = 0u;
    return true;
}

// in-place complex FFT of a[0..N), N = 2^logN, by the block; sign -1 forward
__device__ void fft(double2 *a, int N, int logN, const double2 *__restrict__ tw, double sign)
{
    for (int t = threadIdx.x; t < N; t += blockDim.x) {
        const int r = (int)(__brev((unsigned)t) >> (32 - logN));
        if (r > t) { const double2 x = a[t]; a[t] = a[r]; a[r] = x; }
    }
    __syncthreads();
    for (int s = 0; s < logN; s++) {
        const int half = 1 << s, step = N >> (s + 1);
        for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
            const int pos = t & (half - 1), i0 = ((t >> s) << (s + 1)) + pos, i1 = i0 + half;
            double2 w = tw[pos * step];
            w.y *= -sign;   // the table holds exp(-2 pi i k / N); the inverse takes its conjugate
            const double2 u = a[i0], v = a[i1];
            const double2 x = make_double2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
            a[i0] = make_double2(u.x + x.x, u.y + x.y);
            a[i1] = make_double2(u.x - x.x, u.y - x.y);
        }
        __syncthreads();
    }
}

// sm holds a real row (imaginary parts zero): forward transform into the
// half-complex row j of hat, times scale
__device__ void row_forward(const SpecArgs &A, double2 *sm, int j)
{
    const int P = A.d.P, N = A.N;
    __syncthreads();
    fft(sm, N, A.logN, A.tw, -1.0);
    for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) AT_(A.hat, k, j) = sm[k].x * A.fscale;
    for (int k = 1 + threadIdx.x; k < N / 2; k += blockDim.x) AT_(A.hat, N - k, j) = sm[k].y * A.fscale;
}

__device__ __forceinline__ int src_x(const SpecArgs &A, int i) { return A.mp.x.src[i + NG]; }
__device__ __forceinline__ int src_y(const SpecArgs &A, int j) { return A.mp.y.src[j + NG]; }

}  // namespace

// r = rhs - A phi, the stopping test, forward transforms of r
__global__ void __launch_bounds__(ROW_THREADS) k_spec_init_rows(SpecArgs A)
{
    extern __shared__ double2 sm[];
    __shared__ double sh[32];
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY, j = blockIdx.x;
    double sJ = 0.0;
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) {
        const double ad = pressure_op(d, A.rho, i, j, [&](int a, int b) { return remap(A.mp, A.phi, P, NX, NY, a, b); });
        const double rv = AT_(A.rhs, i, j) - ad;
        AT_(A.res, i, j) = rv;
        sJ += rv * (rv * AT_(A.MJ, i, j));
        sm[i] = make_double2(rv, 0.0);
    }
    row_forward(A, sm, j);
    double tot;
    if (finish_sum(sJ, A.part, &A.s->cnt[0], sh, tot) && threadIdx.x == 0) {
        A.s->iters = 0;
        A.s->res = sqrt(tot);
        A.s->done = sqrt(tot) < A.tol ? 1 : 0;
    }
}

// tridiagonal solves along y by parallel cyclic reduction, one block per
// half-complex index
__global__ void k_spec_tridiag(SpecArgs A)
{
    if (A.s->done) return;
    extern __shared__ double sbuf[];
    __shared__ double sh[32];
    const int P = A.d.P, M = A.M, m = blockIdx.x, j = threadIdx.x;
    double *sa = sbuf, *sb = sa + M, *sc = sb + M, *sd = sc + M;
    const bool row = j < M;
    double a = 0.0, b = 1.0, c = 0.0, r = row ? AT_(A.hat, m, j) : 0.0;
    if (m == 0) {   // the mean mode: a mean-free right-hand side, so the pinned row's equation holds too
        __shared__ double rmean;
        const double t = block_sum(r, sh);
        if (threadIdx.x == 0) rmean = t / (double)M;
        __syncthreads();
        r -= rmean;
    }
    if (row && !(m == 0 && j == 0)) {
        a = j > 0 ? -1.0 : 0.0;
        c = j < M - 1 ? -1.0 : 0.0;
        b = A.lamx[m] + (j > 0 ? 1.0 : 0.0) + (j < M - 1 ? 1.0 : 0.0);
    } else {
        r = 0.0;
    }
    for (int s = 1; s < M; s <<= 1) {
        if (row) { sa[j] = a; sb[j] = b; sc[j] = c; sd[j] = r; }
        __syncthreads();
        if (row) {
            double an = 0.0, cn = 0.0, bn = b, rn = r;
            if (j - s >= 0) {
                const double k1 = a / sb[j - s];
                bn -= sc[j - s] * k1;
                rn -= sd[j - s] * k1;
                an = -sa[j - s] * k1;
            }
            if (j + s < M) {
                const double k2 = c / sb[j + s];
                bn -= sa[j + s] * k2;
                rn -= sd[j + s] * k2;
                cn = -sc[j + s] * k2;
            }
            a = an; b = bn; c = cn; r = rn;
        }
        __syncthreads();
    }
    double x = row ? r / b : 0.0;
    if (m == 0) {   // project out the constant mode
        __shared__ double mean;
        const double t = block_sum(x, sh);
        if (threadIdx.x == 0) mean = t / (double)M;
        __syncthreads();
        x -= mean;
    }
    if (row) AT_(A.hat, m, j) = x;
}

// z = inverse transform of the solved rows; gamma = r.z; first: gamma, beta = 0
__global__ void __launch_bounds__(ROW_THREADS) k_spec_inverse_rows(SpecArgs A, int first)
{
    if (A.s->done) return;
    extern __shared__ double2 sm[];
    __shared__ double sh[32];
    const int P = A.d.P, N = A.N, j = blockIdx.x;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        double2 v;
        if (k == 0 || 2 * k == N) v = make_double2(AT_(A.hat, k, j), 0.0);
        else if (k < N / 2) v = make_double2(AT_(A.hat, k, j), AT_(A.hat, N - k, j));
        else v = make_double2(AT_(A.hat, N - k, j), -AT_(A.hat, k, j));
        sm[k] = v;
    }
    __syncthreads();
    fft(sm, N, A.logN, A.tw, 1.0);
    double g = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double z = sm[i].x;
        AT_(A.z, i, j) = z;
        g += AT_(A.res, i, j) * z;
    }
    double tot;
    if (finish_sum(g, A.part, &A.s->cnt[1], sh, tot) && threadIdx.x == 0) {
        A.s->beta = first ? 0.0 : tot / (A.s->gamma + 1e-30);
        A.s->gamma = tot;
    }
}

// d = z + beta d_old (d = z on the first iteration) at every cell and its
// neighbours, Ad, d.Ad; alpha = gamma / d.Ad
__global__ void __launch_bounds__(ROW_THREADS) k_spec_matvec(SpecArgs A, const double *__restrict__ dold,
                                                             double *__restrict__ dnew, int first)
{
    if (A.s->done) return;
    __shared__ double sh[32];
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY, j = blockIdx.x;
    const double bt = A.s->beta;
    auto dir = [&](int a, int b) {
        int si = a, sj = b;
        if (!(a >= 1 && a <= NX - 2 && b >= 1 && b <= NY - 2)) { si = src_x(A, a); sj = src_y(A, b); }
        return first ? AT_(A.z, si, sj) : AT_(A.z, si, sj) + bt * AT_(dold, si, sj);
    };
    double s = 0.0;
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) {
        const double dv = dir(i, j);
        AT_(dnew, i, j) = dv;
        const double ad = pressure_op(d, A.rho, i, j, dir);
        AT_(A.Ad, i, j) = ad;
        s += dv * ad;
    }
    double tot;
    if (finish_sum(s, A.part, &A.s->cnt[2], sh, tot) && threadIdx.x == 0) A.s->alpha = A.s->gamma / (tot + 1e-30);
}

// phi += alpha d, r -= alpha Ad, the stopping test, forward transforms of r
__global__ void __launch_bounds__(ROW_THREADS) k_spec_update_rows(SpecArgs A, const double *__restrict__ dcur)
{
    if (A.s->done) return;
    extern __shared__ double2 sm[];
    __shared__ double sh[32];
    const int P = A.d.P, j = blockIdx.x;
    const double alpha = A.s->alpha;
    double sJ = 0.0;
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) {
        AT_(A.phi, i, j) += alpha * AT_(dcur, i, j);
        const double rv = AT_(A.res, i, j) - alpha * AT_(A.Ad, i, j);
        AT_(A.res, i, j) = rv;
        sJ += rv * (rv * AT_(A.MJ, i, j));
        sm[i] = make_double2(rv, 0.0);
    }
    row_forward(A, sm, j);
    double tot;
    if (finish_sum(sJ, A.part, &A.s->cnt[3], sh, tot) && threadIdx.x == 0) {
        const int it = A.s->iters + 1;
        A.s->iters = it;
        A.s->res = sqrt(tot);
        if (sqrt(tot) < A.tol || it >= A.maxit) A.s->done = 1;
    }
}

// the mean of phi over the solve range (psolve_cg.c:255-279); a solve that
// stops before its first iteration leaves phi as it is, as the reference does
__global__ void __launch_bounds__(ROW_THREADS) k_spec_mean(SpecArgs A)
{
    __shared__ double sh[32];
    const int P = A.d.P, j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) s += AT_(A.phi, i, j);
    double tot;
    if (finish_sum(s, A.part, &A.s->cnt[4], sh, tot) && threadIdx.x == 0) {
        A.s->avg = A.s->iters == 0 ? 0.0 : tot / ((double)A.N * (double)A.M);
        A.scal->p_iters = A.s->iters;
        A.scal->p_res = A.s->res;
    }
}

__global__ void __launch_bounds__(ROW_THREADS) k_spec_sub_mean(SpecArgs A)
{
    const int P = A.d.P, j = blockIdx.x;
    const double avg = A.s->avg;
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) AT_(A.phi, i, j) -= avg;
}

// ---------------------------------------------------------------------------
// host

bool spec_supported(const Dom &d, const char **why)
{
    const int N = d.NX - 1, M = d.NY - 1;
    if (!d.planar || d.axisym) { *why = "the spectral pressure preconditioner is built for the planar mode only"; return false; }
    if (!d.perx || d.pery) { *why = "the spectral pressure preconditioner needs x periodic and walls in y"; return false; }
    if (N < 2 || (N & (N - 1)) != 0 || N > 2048) { *why = "the spectral pressure preconditioner needs a power-of-two x cell count (2..2048)"; return false; }
    if (M < 1 || M > 1024) { *why = "the spectral pressure preconditioner needs at most 1024 y cells"; return false; }
    return true;
}

int spec_tables(int N, double idx2, double idy2, std::vector<double> &lamx, std::vector<double> &tw)
{
    lamx.assign(N, 0.0);
    for (int m = 0; m < N; m++) {
        const int wave = m <= N / 2 ? m : N - m;
        lamx[m] = (2.0 - 2.0 * std::cos(2.0 * M_PI * wave / N)) * idx2 / idy2;
    }
    tw.assign(N, 0.0);   // N / 2 complex entries exp(-2 pi i k / N)
    for (int k = 0; k < N / 2; k++) {
        tw[2 * k] = std::cos(2.0 * M_PI * k / N);
        tw[2 * k + 1] = -std::sin(2.0 * M_PI * k / N);
    }
    return 0;
}

cudaError_t spec_launch_init(const SpecArgs &A, cudaStream_t st)
{
    const size_t row_smem = (size_t)A.N * sizeof(double2);
    const unsigned tthreads = (unsigned)((A.M + 31) / 32 * 32);
    k_spec_init_rows<<<(unsigned)A.M, ROW_THREADS, row_smem, st>>>(A);
    k_spec_tridiag<<<(unsigned)A.N, tthreads, 4 * (size_t)A.M * sizeof(double), st>>>(A);
    k_spec_inverse_rows<<<(unsigned)A.M, ROW_THREADS, row_smem, st>>>(A, 1);
    return cudaGetLastError();
}

cudaError_t spec_launch_iteration(const SpecArgs &A, const double *dold, double *dnew, int first, cudaStream_t st)
{
    const size_t row_smem = (size_t)A.N * sizeof(double2);
    const unsigned tthreads = (unsigned)((A.M + 31) / 32 * 32);
    k_spec_matvec<<<(unsigned)A.M, ROW_THREADS, 0, st>>>(A, dold, dnew, first);
    k_spec_update_rows<<<(unsigned)A.M, ROW_THREADS, row_smem, st>>>(A, dnew);
    k_spec_tridiag<<<(unsigned)A.N, tthreads, 4 * (size_t)A.M * sizeof(double), st>>>(A);
    k_spec_inverse_rows<<<(unsigned)A.M, ROW_THREADS, row_smem, st>>>(A, 0);
    return cudaGetLastError();
}

cudaError_t spec_launch_mean(const SpecArgs &A, cudaStream_t st)
{
    k_spec_mean<<<(unsigned)A.M, ROW_THREADS, 0, st>>>(A);
    k_spec_sub_mean<<<(unsigned)A.M, ROW_THREADS, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace pvof
