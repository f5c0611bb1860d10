// Pressure PCG with a constant-density spectral preconditioner: a form with
// no counterpart in the reference (which preconditions Pressure_solve_cg,
// Eulerian/lsolver/psolve_cg.c:130-293, with the Jacobi diagonal).
//
// The operator is the reference's variable-density one (pressure_op,
// psolve_cg.c:302-344) with its ghost rules (Pressure_apply_BCs: x periodic,
// mirror walls in y).  The preconditioner is z = s (-L)^-1 (s r): L the same
// five-point operator with the density set to one, s = sqrt(1 / diag A) the
// square root of the Jacobi weights, so the density variation of the
// diagonal is taken out symmetrically.  A Fourier transform along the
// periodic x rows diagonalises L into one tridiagonal system per wavenumber
// along y:
//
//   1. every row j: forward complex FFT of the residual row (radix 2 in shared
//      memory, twiddles from a table), stored in FFTW's half-complex order
//      (Re X_0 .. Re X_{N/2}, Im X_{N/2-1} .. Im X_1) times dy^2 / N;
//   2. every half-complex index m: parallel cyclic reduction (one thread per
//      row, log2 M elimination rounds in shared memory) of
//        -z_{j-1} + (b_j + dy^2 lambda_x(m)) z_j - z_{j+1} = rhs_j,
//      b_j = 2 inside, 1 at the two walls.  The matrices do not change, so
//      the rounds' multipliers and the final reciprocal diagonals are
//      computed once per context on the host (spec_tables, one set per wave
//      number: the half-complex indices m and N - m share it) and a round is
//      two multiply-adds.  The mean mode's system is singular (the constant,
//      the operator's null space): its first row is pinned, the right-hand
//      side and the result are made mean-free, and the right-hand side's mean
//      is added back, i.e. the constant mode is given eigenvalue 1 (the
//      inverse of L + P, P the projector on constants), which keeps the
//      scaled preconditioner positive definite;
//   3. every row: inverse transform.
//
// Without the scaling the preconditioned operator's condition number is at
// most the density ratio rho_max / rho_min, whatever the grid size (the
// Jacobi-PCG's grows with the square of the grid); the scaling cuts the
// iterations further where the ratio is large (about 30 instead of 205 per
// solve at 1e-3 on 1024 x 1024).  The stopping test is the
// reference's: sqrt(r^T D^-1 r) below P_CG_ETOL with D the Jacobi diagonal,
// so the solve stops at the same residual size; the iterates differ, so the
// result moves within that tolerance of the reference's.
//
// The whole solve is ONE cooperative launch: blocks of SPEC_PT threads, eight
// 128-thread row groups in the row phases, SPEC_PT / Mp reduction systems per
// block (Mp = M rounded up to 32), four grid barriers per iteration (after the
// matrix-vector product, the update with its forward transforms, the
// tridiagonal solves, the inverse transforms).  Every block adds the
// per-block sums in block order, so all of them take the same decisions.  The
// grid barrier resets itself (the last arriver zeroes the count and advances
// a generation); its wait is bounded (on timeout the error flag in DevScalars
// is set and every block leaves).
#include <cmath>
#include <vector>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

namespace {

constexpr int ROW_THREADS = 128;
constexpr int ROWG = SPEC_PT / ROW_THREADS;
constexpr unsigned long long SPEC_SPIN_LIMIT = 1ull << 26;

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

// Grid barrier: the last block to arrive resets the arrival count and
// advances the generation that the others wait on, so the barrier needs no
// reset between launches.  The wait is bounded; returns false (in every
// thread of the block) when it gave up or another block did.
__device__ __noinline__ bool spec_barrier(SpecScal *s, int *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &s->bar_gen;
        volatile int *verr = err;
        int good = (*verr == 0);
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&s->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            s->bar_count = 0u;
            __threadfence();
            atomicAdd(&s->bar_gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (*vgen == g) {
                ++spins;
                if ((spins & 1023ull) == 0 && (*verr != 0 || spins > SPEC_SPIN_LIMIT)) {
                    atomicCAS(err, 0, 2);   // 2: the spectral solve's barrier
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

// this block's sum of v into slot[blockIdx.x]
__device__ void put_part(double v, double *slot, double *sh)
{
    const double b = block_sum(v, sh);
    if (threadIdx.x == 0) slot[blockIdx.x] = b;
}

// the sum of a slot over all blocks, in block order, in every thread
__device__ double slot_total(const double *slot, double *sh)
{
    __shared__ double res;
    double s = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) s += __ldcg(slot + k);
    const double t = block_sum(s, sh);
    if (threadIdx.x == 0) res = t;
    __syncthreads();
    const double r = res;
    __syncthreads();
    return r;
}

// complex FFT of a[0..N), N = 2^logN, by the 128 threads of one row group
// (lt = 0..127); sign -1 forward.  All groups of the block run it in lockstep.
// Radix-2 decimation in time after a bit reversal; two successive stages are
// done per pass through shared memory (each thread keeps the four values of
// both stages' butterflies in registers, the arithmetic is that of the two
// radix-2 stages), a last odd stage on its own.
__device__ __forceinline__ double2 cmul(double2 v, double2 w)
{
    return make_double2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
}

__device__ __forceinline__ double2 twid(const double2 *__restrict__ tw, int k, double sign)
{
    double2 w = tw[k];
    w.y *= -sign;   // the table holds exp(-2 pi i k / N); the inverse takes its conjugate
    return w;
}

__device__ void fft_group(double2 *a, int N, int logN, const double2 *__restrict__ tw, double sign, int lt)
{
    for (int t = lt; t < N; t += ROW_THREADS) {
        const int r = (int)(__brev((unsigned)t) >> (32 - logN));
        if (r > t) { const double2 x = a[t]; a[t] = a[r]; a[r] = x; }
    }
    __syncthreads();
    int s = 0;
    for (; s + 1 < logN; s += 2) {   // stages s and s + 1
        const int h = 1 << s;
        for (int t = lt; t < N / 4; t += ROW_THREADS) {
            const int pos = t & (h - 1), i0 = ((t >> s) << (s + 2)) + pos, i1 = i0 + h, i2 = i1 + h, i3 = i2 + h;
            const double2 w1 = twid(tw, pos * (N >> (s + 1)), sign);
            const double2 w2 = twid(tw, pos * (N >> (s + 2)), sign), w3 = twid(tw, (pos + h) * (N >> (s + 2)), sign);
            const double2 x0 = a[i0], x1 = a[i1], x2 = a[i2], x3 = a[i3];
            double2 x = cmul(x1, w1);
            const double2 y0 = make_double2(x0.x + x.x, x0.y + x.y), y1 = make_double2(x0.x - x.x, x0.y - x.y);
            x = cmul(x3, w1);
            const double2 y2 = make_double2(x2.x + x.x, x2.y + x.y), y3 = make_double2(x2.x - x.x, x2.y - x.y);
            x = cmul(y2, w2);
            a[i0] = make_double2(y0.x + x.x, y0.y + x.y);
            a[i2] = make_double2(y0.x - x.x, y0.y - x.y);
            x = cmul(y3, w3);
            a[i1] = make_double2(y1.x + x.x, y1.y + x.y);
            a[i3] = make_double2(y1.x - x.x, y1.y - x.y);
        }
        __syncthreads();
    }
    if (s < logN) {   // the last stage when log2 N is odd
        const int half = 1 << s, step = N >> (s + 1);
        for (int t = lt; t < N / 2; t += ROW_THREADS) {
            const int pos = t & (half - 1), i0 = ((t >> s) << (s + 1)) + pos, i1 = i0 + half;
            const double2 u = a[i0], x = cmul(a[i1], twid(tw, pos * step, sign));
            a[i0] = make_double2(u.x + x.x, u.y + x.y);
            a[i1] = make_double2(u.x - x.x, u.y - x.y);
        }
        __syncthreads();
    }
}

// forward transform of the group's row (already in a) into hat row j
__device__ void group_forward(const SpecArgs &A, double2 *a, int j, bool active, int lt)
{
    const int P = A.d.P, N = A.N;
    __syncthreads();
    fft_group(a, N, A.logN, A.tw, -1.0, lt);
    if (active) {
        for (int k = lt; k <= N / 2; k += ROW_THREADS) AT_(A.hat, k, j) = a[k].x * A.fscale;
        for (int k = 1 + lt; k < N / 2; k += ROW_THREADS) AT_(A.hat, N - k, j) = a[k].y * A.fscale;
    }
    __syncthreads();   // the next row step overwrites a
}

__device__ __forceinline__ int src_x(const SpecArgs &A, int i) { return A.mp.x.src[i + NG]; }
__device__ __forceinline__ int src_y(const SpecArgs &A, int j) { return A.mp.y.src[j + NG]; }

// mean over the block's system 0 (threads sys == 0), broadcast to the block
__device__ double system0_mean(double v, bool sys0, int M, double *sh)
{
    __shared__ double mean;
    const double t = block_sum(sys0 ? v : 0.0, sh);
    if (threadIdx.x == 0) mean = t / (double)M;
    __syncthreads();
    const double r = mean;
    __syncthreads();
    return r;
}

// half-complex index of the q-th system: 0, N/2, then 1, N-1, 2, N-2, ...,
// so the two indices of one wave number (same matrix, same table rows) are
// solved side by side
__device__ __forceinline__ int system_index(int q, int N)
{
    if (q < 2) return q == 0 ? 0 : N / 2;
    return (q & 1) ? N - (q >> 1) : (q >> 1);
}

// the tridiagonal solves of every half-complex index, hat in place
__device__ void tridiag_phase(const SpecArgs &A, double *smem, double *sh)
{
    const int P = A.d.P, N = A.N, M = A.M, Mp = (M + 31) / 32 * 32, S = SPEC_PT / Mp;
    const int sys = threadIdx.x / Mp, j = threadIdx.x - sys * Mp;
    const size_t NM = (size_t)(N / 2 + 1) * M;   // table rows per round: one per wave number
    double *sd = smem + (size_t)sys * Mp;
    for (int m0 = blockIdx.x * S; m0 < N; m0 += gridDim.x * S) {
        const int q = m0 + sys;
        const int m = q < N ? system_index(q, N) : 0;
        const int wave = m <= N / 2 ? m : N - m;
        const bool row = sys < S && q < N && j < M;
        double r = row ? AT_(A.hat, m, j) : 0.0;
        double rmean = 0.0;
        if (m0 == 0) {   // this block holds the mean mode as its system 0
            rmean = system0_mean(r, sys == 0, M, sh);
            if (q == 0) r = j == 0 ? 0.0 : r - rmean;   // mean-free, first row pinned
        }
        // this thread's multipliers, all loads in flight at once: round st
        // k1 at [2 st NM], k2 at [(2 st + 1) NM], then 1 / b at [2 rounds NM]
        const double *k = A.pcr + (size_t)wave * M + j;
        double kr[2 * SPEC_MAXROUNDS + 1];
#pragma unroll
        for (int q = 0; q < 2 * SPEC_MAXROUNDS + 1; q++) kr[q] = (row && q <= 2 * A.rounds) ? k[(size_t)q * NM] : 0.0;
#pragma unroll
        for (int st = 0; st < SPEC_MAXROUNDS; st++) {
            if (st >= A.rounds) break;
            const int s = 1 << st;
            if (row) sd[j] = r;
            __syncthreads();
            if (row) {
                double rn = r;
                if (j - s >= 0) rn -= sd[j - s] * kr[2 * st];
                if (j + s < M) rn -= sd[j + s] * kr[2 * st + 1];
                r = rn;
            }
            __syncthreads();
        }
        double ib = 0.0;
#pragma unroll
        for (int q = 0; q < 2 * SPEC_MAXROUNDS + 1; q++)
            if (q == 2 * A.rounds) ib = kr[q];
        double x = row ? r * ib : 0.0;   // times the final 1 / b
        if (m0 == 0) {
            // the constant mode, the operator's null space, gets eigenvalue 1
            // (in units of 1 / dy^2) instead of 0: the mean-free solution plus
            // the right-hand side's mean, so the scaled preconditioner stays
            // positive definite
            const double mean = system0_mean(x, sys == 0, M, sh);
            if (q == 0) x = x - mean + rmean;
        }
        if (row) AT_(A.hat, m, j) = x;
    }
}

}  // namespace

__global__ void __launch_bounds__(SPEC_PT) k_spec_pcg(SpecArgs A, double *d0, double *d1)
{
    extern __shared__ double smem[];   // the twiddles, then the row / reduction work area
    __shared__ double sh[32];
    const Dom &d = A.d;
    const int P = d.P, NX = d.NX, NY = d.NY, N = A.N, M = A.M;
    const int grp = threadIdx.x / ROW_THREADS, lt = threadIdx.x - grp * ROW_THREADS;
    double2 *tw = reinterpret_cast<double2 *>(smem);
    double *work = smem + N;   // N / 2 complex twiddles before it
    double2 *row = reinterpret_cast<double2 *>(work) + (size_t)grp * N;
    double *slotA = A.part, *slotB = A.part + gridDim.x, *slotC = A.part + 2 * gridDim.x;
    SpecScal *S = A.s;
    int *err = &A.scal->error;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    for (int k = threadIdx.x; k < N / 2; k += blockDim.x) tw[k] = A.tw[k];
    __syncthreads();
    SpecArgs B = A;
    B.tw = tw;

    // r = rhs - A phi, the stopping sum, forward transforms
    double sJ = 0.0;
    for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
        const int j = j0 + grp;
        const bool active = j < M;
        if (active) {
            for (int i = lt; i < N; i += ROW_THREADS) {
                const double ad = pressure_op(d, A.rho, i, j, [&](int a, int b) { return remap(A.mp, A.phi, P, NX, NY, a, b); });
                const double rv = AT_(A.rhs, i, j) - ad;
                AT_(A.res, i, j) = rv;
                sJ += rv * (rv * AT_(A.MJ, i, j));
                row[i] = make_double2(rv * sqrt(AT_(A.MJ, i, j)), 0.0);
            }
        }
        group_forward(B, row, j, active, lt);
    }
    put_part(sJ, slotA, sh);
    if (!spec_barrier(S, err)) return;
    double tot = slot_total(slotA, sh);
    int iters = 0;
    double res = sqrt(tot);
    if (sqrt(tot) < A.tol) {   // converged before the first iteration: phi stays as it is
        if (lead) { A.scal->p_iters = 0; A.scal->p_res = res; }
        return;
    }
    double gamma = 0.0, beta = 0.0;
    double *dold = d0, *dnew = d1;
    for (int it = 0;; it++) {
        // z = (-L)^-1 r
        tridiag_phase(A, work, sh);
        if (!spec_barrier(S, err)) return;
        double g = 0.0;
        for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
            const int j = j0 + grp;
            const bool active = j < M;
            if (active) {
                for (int k = lt; k < N; k += ROW_THREADS) {
                    double2 v;
                    if (k == 0 || 2 * k == N) v = make_double2(AT_(A.hat, k, j), 0.0);
                    else if (k < N / 2) v = make_double2(AT_(A.hat, k, j), AT_(A.hat, N - k, j));
                    else v = make_double2(AT_(A.hat, N - k, j), -AT_(A.hat, k, j));
                    row[k] = v;
                }
            }
            __syncthreads();
            fft_group(row, N, A.logN, tw, 1.0, lt);
            if (active) {
                for (int i = lt; i < N; i += ROW_THREADS) {
                    const double z = row[i].x * sqrt(AT_(A.MJ, i, j));
                    AT_(A.z, i, j) = z;
                    g += AT_(A.res, i, j) * z;
                }
            }
            __syncthreads();
        }
        put_part(g, slotB, sh);
        if (!spec_barrier(S, err)) return;
        const double gnew = slot_total(slotB, sh);
        // guards against 0 / 0 only: with the scaling r.z is about the Jacobi
        // weight times smaller than in the reference's iteration, so a guard
        // of the reference's size (1e-30) would bend the steps near a tight
        // tolerance
        beta = it == 0 ? 0.0 : gnew / (gamma + 1e-300);
        gamma = gnew;
        if (it >= A.maxit) break;
        // d = z + beta d_old at every cell and its neighbours, Ad, d.Ad
        const bool first = it == 0;
        auto dir = [&](int a, int b) {
            int si = a, sj = b;
            if (!(a >= 1 && a <= NX - 2 && b >= 1 && b <= NY - 2)) { si = src_x(A, a); sj = src_y(A, b); }
            return first ? AT_(A.z, si, sj) : AT_(A.z, si, sj) + beta * AT_(dold, si, sj);
        };
        double sdad = 0.0;
        for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
            const int j = j0 + grp;
            if (j >= M) continue;
            for (int i = lt; i < N; i += ROW_THREADS) {
                const double dv = dir(i, j);
                AT_(dnew, i, j) = dv;
                const double ad = pressure_op(d, A.rho, i, j, dir);
                AT_(A.Ad, i, j) = ad;
                sdad += dv * ad;
            }
        }
        put_part(sdad, slotC, sh);
        if (!spec_barrier(S, err)) return;
        const double alpha = gamma / (slot_total(slotC, sh) + 1e-300);
        // phi += alpha d, r -= alpha Ad, the stopping sum, forward transforms
        sJ = 0.0;
        for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
            const int j = j0 + grp;
            const bool active = j < M;
            if (active) {
                for (int i = lt; i < N; i += ROW_THREADS) {
                    AT_(A.phi, i, j) += alpha * AT_(dnew, i, j);
                    const double rv = AT_(A.res, i, j) - alpha * AT_(A.Ad, i, j);
                    AT_(A.res, i, j) = rv;
                    sJ += rv * (rv * AT_(A.MJ, i, j));
                    row[i] = make_double2(rv * sqrt(AT_(A.MJ, i, j)), 0.0);
                }
            }
            group_forward(B, row, j, active, lt);
        }
        put_part(sJ, slotA, sh);
        if (!spec_barrier(S, err)) return;
        tot = slot_total(slotA, sh);
        iters = it + 1;
        res = sqrt(tot);
        if (sqrt(tot) < A.tol || iters >= A.maxit) break;
        double *t = dold; dold = dnew; dnew = t;
    }
    // remove the mean (psolve_cg.c:255-279)
    double ssum = 0.0;
    for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
        const int j = j0 + grp;
        if (j >= M) continue;
        for (int i = lt; i < N; i += ROW_THREADS) ssum += AT_(A.phi, i, j);
    }
    put_part(ssum, slotB, sh);
    if (!spec_barrier(S, err)) return;
    const double avg = slot_total(slotB, sh) / ((double)N * (double)M);
    for (int j0 = blockIdx.x * ROWG; j0 < M; j0 += gridDim.x * ROWG) {
        const int j = j0 + grp;
        if (j >= M) continue;
        for (int i = lt; i < N; i += ROW_THREADS) AT_(A.phi, i, j) -= avg;
    }
    if (lead) { A.scal->p_iters = iters; A.scal->p_res = res; }
}

// ---------------------------------------------------------------------------
// host

bool spec_supported(const Dom &d, const char **why)
{
    const int N = d.NX - 1, M = d.NY - 1;
    if (!d.planar || d.axisym) { *why = "the spectral pressure preconditioner is built for the planar mode only"; return false; }
    if (!d.perx || d.pery) { *why = "the spectral pressure preconditioner needs x periodic and walls in y"; return false; }
    if (N < 2 || (N & (N - 1)) != 0 || N > 1024) { *why = "the spectral pressure preconditioner needs a power-of-two x cell count (2..1024)"; return false; }
    if (M < 1 || M > 1024) { *why = "the spectral pressure preconditioner needs at most 1024 y cells"; return false; }
    return true;
}

int spec_tables(int N, int M, double idx2, double idy2, std::vector<double> &tw, std::vector<double> &pcr)
{
    tw.assign(N, 0.0);   // N / 2 complex entries exp(-2 pi i k / N)
    for (int k = 0; k < N / 2; k++) {
        tw[2 * k] = std::cos(2.0 * M_PI * k / N);
        tw[2 * k + 1] = -std::sin(2.0 * M_PI * k / N);
    }
    int nsteps = 0;
    for (int s = 1; s < M; s <<= 1) nsteps++;
    const size_t NM = (size_t)(N / 2 + 1) * M;   // one matrix per wave number 0 .. N/2
    pcr.assign((size_t)(2 * nsteps + 1) * NM, 0.0);
    std::vector<double> a(M), b(M), c(M), a2(M), b2(M), c2(M);
    for (int m = 0; m <= N / 2; m++) {   // m: the wave number
        const double lam = (2.0 - 2.0 * std::cos(2.0 * M_PI * m / N)) * idx2 / idy2;
        for (int j = 0; j < M; j++) {
            if (m == 0 && j == 0) { a[j] = 0.0; b[j] = 1.0; c[j] = 0.0; continue; }   // the pinned row
            a[j] = j > 0 ? -1.0 : 0.0;
            c[j] = j < M - 1 ? -1.0 : 0.0;
            b[j] = lam + (j > 0 ? 1.0 : 0.0) + (j < M - 1 ? 1.0 : 0.0);
        }
        int st = 0;
        for (int s = 1; s < M; s <<= 1, st++) {   // the elimination rounds of the device's cyclic reduction
            for (int j = 0; j < M; j++) {
                double an = 0.0, cn = 0.0, bn = b[j], k1 = 0.0, k2 = 0.0;
                if (j - s >= 0) { k1 = a[j] / b[j - s]; bn -= c[j - s] * k1; an = -a[j - s] * k1; }
                if (j + s < M) { k2 = c[j] / b[j + s]; bn -= a[j + s] * k2; cn = -c[j + s] * k2; }
                pcr[(size_t)(2 * st) * NM + (size_t)m * M + j] = k1;
                pcr[(size_t)(2 * st + 1) * NM + (size_t)m * M + j] = k2;
                a2[j] = an; b2[j] = bn; c2[j] = cn;
            }
            a.swap(a2); b.swap(b2); c.swap(c2);
        }
        for (int j = 0; j < M; j++) pcr[(size_t)(2 * nsteps) * NM + (size_t)m * M + j] = 1.0 / b[j];
    }
    return nsteps;
}

size_t spec_pcg_smem(int N, int M)
{
    const size_t rows = (size_t)ROWG * N * sizeof(double2);
    const int Mp = (M + 31) / 32 * 32;
    const size_t tri = (size_t)(SPEC_PT / Mp) * Mp * sizeof(double);
    return (size_t)N * sizeof(double) + (rows > tri ? rows : tri);   // twiddles first
}

// blocks for k_spec_pcg: enough for one pass over the rows and the systems,
// at most what is co-resident; 0 if the launch cannot be cooperative
int spec_pcg_blocks(int device, int N, int M)
{
    const size_t smem = spec_pcg_smem(N, M);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_spec_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int per_sm = 0, sms = 0, coop = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spec_pcg, SPEC_PT, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    const int Mp = (M + 31) / 32 * 32, S = SPEC_PT / Mp;
    int want = (M + ROWG - 1) / ROWG;
    const int sys = (N + S - 1) / S;
    if (sys > want) want = sys;
    const int most = per_sm * sms;
    return most < 1 ? 0 : (want < most ? want : most);
}

const void *spec_pcg_kernel() { return (const void *)k_spec_pcg; }

cudaError_t spec_launch_pcg(const SpecArgs &A, int blocks, double *d0, double *d1, cudaStream_t st)
{
    SpecArgs a = A;
    void *args[] = {&a, &d0, &d1};
    return cudaLaunchCooperativeKernel((const void *)k_spec_pcg, dim3((unsigned)blocks), dim3(SPEC_PT), args,
                                       spec_pcg_smem(A.N, A.M), st);
}

}  // namespace pvof
