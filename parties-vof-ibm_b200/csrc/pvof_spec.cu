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
//   2. every half-complex index m: the tridiagonal system
//        -z_{j-1} + (b_j + dy^2 lambda_x(m)) z_j - z_{j+1} = rhs_j,
//      b_j = 2 inside, 1 at the two walls, by a partition method: one warp
//      per system, the column staged in shared memory, each lane owning a
//      chunk of consecutive rows.  A lane eliminates its chunk's sub- and
//      super-diagonals down to two equations in the chunk's first and last
//      unknowns; the 2P equations of the P chunks form a tridiagonal system
//      that one lane solves by the Thomas algorithm; each lane then fills in
//      its chunk's interior by back substitution.  The matrices do not change,
//      so every pivot and coupling coefficient, those of the reduced system
//      included, is computed once per context on the host (spec_tables, one
//      set per wave number: the half-complex indices m and N - m share it);
//      per iteration a row costs an add and a multiply or two.  The mean
//      mode's system is singular (the constant, the operator's null space):
//      its first row is pinned, the right-hand side and the result are made
//      mean-free, and the right-hand side's mean is added back, i.e. the
//      constant mode is given eigenvalue 1 (the inverse of L + P, P the
//      projector on constants), which keeps the scaled preconditioner
//      positive definite;
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
// 128-thread row groups in the row phases, eight warps of one tridiagonal
// system each per block in the solve phase, four grid barriers per iteration (after the
// matrix-vector product, the update with its forward transforms, the
// tridiagonal solves, the inverse transforms), one more per solve after the
// solve's constants (face coefficients, weight roots).  Every block adds the
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

constexpr int ROW_THREADS = 256;
constexpr int ROWG = SPEC_PT / ROW_THREADS;   // row groups per block, one pair of rows each
constexpr unsigned long long SPEC_SPIN_LIMIT = 1ull << 26;
constexpr int SPEC_SYS = 8;          // tridiagonal systems per block and pass, one warp each
constexpr int SPEC_CHUNKS = 32;      // chunks of a system, one per lane

// The rows of a column of M (>= 2) unknowns split into P = min(32, M / 2)
// chunks of base or base + 1 rows (at least two each): chunk l starts at
// l base + min(l, rem) and has base + (l < rem) rows; K = the longest chunk.
struct Chunks {
    int P, base, rem, K;
};

__host__ __device__ inline Chunks spec_chunks(int M)
{
    Chunks c;
    c.P = M / 2 < SPEC_CHUNKS ? M / 2 : SPEC_CHUNKS;
    c.base = M / c.P;
    c.rem = M - c.base * c.P;
    c.K = c.base + (c.rem > 0 ? 1 : 0);
    return c;
}

// shared-memory column index of row j: one pad double per 32 rows, so the
// lanes' chunks (about 32 rows apart) fall in different banks
__device__ __forceinline__ int cidx(int j) { return j + (j >> 5); }

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

// Grid barrier on a counter of arrivals that the host zeroes before the
// launch: the launch's g-th barrier is passed once the counter reaches
// g * gridDim.x (spec_bar_target, kept by the block's thread 0 in shared
// memory so that it takes no register of the solve; at most four barriers
// per iteration, so 32 bits hold the count of any iteration cap below
// about 7 million).  Each block's thread 0 publishes
// the block's writes (block barrier, device-scope fence), adds its arrival
// without waiting for the result and polls the counter.  The wait is
// bounded; returns false (in every thread of the block) when it gave up or
// another block did.
__shared__ unsigned spec_bar_target;

__device__ __noinline__ bool spec_barrier(SpecScal *s, int *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = spec_bar_target += gridDim.x;
        volatile unsigned *va = &s->arrivals;
        volatile int *verr = err;
        int good = 1;
        __threadfence();
        atomicAdd(&s->arrivals, 1u);
        unsigned long long spins = 0;
        while (*va < target) {
            ++spins;
            if ((spins & 1023ull) == 0 && (*verr != 0 || spins > SPEC_SPIN_LIMIT)) {
                atomicCAS(err, 0, 2);   // 2: the spectral solve's barrier
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

// Complex FFTs of rows of N = R n points (R = 1, 3 or 5, n = 2^logn) by the
// ROW_THREADS threads of one row group (lt = their index); sign -1 forward.
// All groups of the block run them in lockstep.  The row is stored
// decimated by R (point i at (i mod R) n + i / R, row_slot): the R
// interleaved subsequences are transformed as R rows of n points (radix-2
// decimation in time after a bit reversal, two stages per pass through
// shared memory with the four values of both stages' butterflies in
// registers, a last odd stage on its own), then one radix-R pass combines
// them in place into the N-point transform in natural order (the R outputs
// k, k + n, .. of one column come from the column's R inputs).  Twiddles
// come from the N-point table exp(-2 pi i k / N), k < N/2 (the other half by
// symmetry); a subsequence's twiddle exp(-2 pi i e / n) is the table's
// entry e R.
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

// exp(sign 2 pi i k / N) for any k >= 0
__device__ __forceinline__ double2 twid_full(const double2 *__restrict__ tw, int k, int N, double sign)
{
    k %= N;
    double2 w = k < N / 2 ? tw[k] : make_double2(-tw[k - N / 2].x, -tw[k - N / 2].y);
    w.y *= -sign;
    return w;
}

// where point i of a row goes before the transform
__device__ __forceinline__ int row_slot(const SpecArgs &A, int i) { return A.R == 1 ? i : (i % A.R) * A.n + i / A.R; }

__device__ void fft_rows(double2 *a, int N, int n, int logn, int R, const double2 *__restrict__ tw, double sign, int lt)
{
    for (int t = lt; t < R * n; t += ROW_THREADS) {
        const int c = t / n, u = t - c * n, r = (int)(__brev((unsigned)u) >> (32 - logn));
        if (r > u) { const double2 x = a[c * n + u]; a[c * n + u] = a[c * n + r]; a[c * n + r] = x; }
    }
    __syncthreads();
    int s = 0;
    for (; s + 1 < logn; s += 2) {   // stages s and s + 1
        const int h = 1 << s;
        for (int t = lt; t < R * (n / 4); t += ROW_THREADS) {
            const int c = t / (n / 4), tt = t - c * (n / 4);
            double2 *b = a + c * n;
            const int pos = tt & (h - 1), i0 = ((tt >> s) << (s + 2)) + pos, i1 = i0 + h, i2 = i1 + h, i3 = i2 + h;
            const double2 w1 = twid(tw, pos * (N >> (s + 1)), sign);
            const double2 w2 = twid(tw, pos * (N >> (s + 2)), sign), w3 = twid(tw, (pos + h) * (N >> (s + 2)), sign);
            const double2 x0 = b[i0], x1 = b[i1], x2 = b[i2], x3 = b[i3];
            double2 x = cmul(x1, w1);
            const double2 y0 = make_double2(x0.x + x.x, x0.y + x.y), y1 = make_double2(x0.x - x.x, x0.y - x.y);
            x = cmul(x3, w1);
            const double2 y2 = make_double2(x2.x + x.x, x2.y + x.y), y3 = make_double2(x2.x - x.x, x2.y - x.y);
            x = cmul(y2, w2);
            b[i0] = make_double2(y0.x + x.x, y0.y + x.y);
            b[i2] = make_double2(y0.x - x.x, y0.y - x.y);
            x = cmul(y3, w3);
            b[i1] = make_double2(y1.x + x.x, y1.y + x.y);
            b[i3] = make_double2(y1.x - x.x, y1.y - x.y);
        }
        __syncthreads();
    }
    if (s < logn) {   // the last stage when log2 n is odd
        const int half = 1 << s, step = N >> (s + 1);
        for (int t = lt; t < R * (n / 2); t += ROW_THREADS) {
            const int c = t / (n / 2), tt = t - c * (n / 2);
            double2 *b = a + c * n;
            const int pos = tt & (half - 1), i0 = ((tt >> s) << (s + 1)) + pos, i1 = i0 + half;
            const double2 u = b[i0], x = cmul(b[i1], twid(tw, pos * step, sign));
            b[i0] = make_double2(u.x + x.x, u.y + x.y);
            b[i1] = make_double2(u.x - x.x, u.y - x.y);
        }
        __syncthreads();
    }
    if (R > 1) {   // X[k + t n] = sum_r exp(sign 2 pi i r (k + t n) / N) F_r[k]
        for (int k = lt; k < n; k += ROW_THREADS) {
            double2 f[5];   // (local memory: only the R > 1 rows pass here)
            for (int r = 0; r < R; r++) f[r] = r == 0 ? a[k] : cmul(a[r * n + k], twid_full(tw, r * k, N, sign));
            for (int t = 0; t < R; t++) {
                double2 x = f[0];
                for (int r = 1; r < R; r++) {
                    const double2 y = cmul(f[r], twid_full(tw, r * t * n, N, sign));
                    x = make_double2(x.x + y.x, x.y + y.y);
                }
                a[t * n + k] = x;
            }
        }
        __syncthreads();
    }
}

// Two real rows in one complex transform: the group's pair of rows ja, jb
// sits in a as a + i b.  Forward: Z = FFT(a + i b) gives both spectra,
// X_a[k] = (Z[k] + conj Z[N-k]) / 2, X_b[k] = (Z[k] - conj Z[N-k]) / 2i,
// stored in half-complex order into hat rows ja and jb (each if active).
// Every group of the block calls it (the transform synchronises the block).
__device__ void pair_forward(const SpecArgs &A, double2 *a, int ja, bool acta, bool actb, int lt)
{
    const int P = A.d.P, N = A.N, jb = ja + 1;
    const double sc = 0.5 * A.fscale;
    __syncthreads();
    fft_rows(a, N, A.n, A.logN, A.R, A.tw, -1.0, lt);
    if (acta)
        for (int k = lt; k <= N / 2; k += ROW_THREADS) {
            const double2 zk = a[k], zn = a[k == 0 ? 0 : N - k];
            AT_(A.hat, k, ja) = (zk.x + zn.x) * sc;
            if (actb) AT_(A.hat, k, jb) = (zk.y + zn.y) * sc;
            if (k > 0 && k < N / 2) {
                AT_(A.hat, N - k, ja) = (zk.y - zn.y) * sc;
                if (actb) AT_(A.hat, N - k, jb) = (zn.x - zk.x) * sc;
            }
        }
    __syncthreads();   // the next pair overwrites a
}

// the spectrum X[k] (k = 0 .. N-1) of a real row from its half-complex row j
__device__ __forceinline__ double2 half_complex(const SpecArgs &A, int k, int j)
{
    const int P = A.d.P, N = A.N;
    if (k == 0 || 2 * k == N) return make_double2(AT_(A.hat, k, j), 0.0);
    if (k < N / 2) return make_double2(AT_(A.hat, k, j), AT_(A.hat, N - k, j));
    return make_double2(AT_(A.hat, N - k, j), -AT_(A.hat, k, j));
}

// pressure_op (Pressure_operator_variableCoeff, psolve_cg.c:302-344) in the
// planar mode from the solve's face coefficients: cx(i, j) is the x face
// between cells i and i+1, (2 / (rho_i + rho_i+1)) idx^2, the same value as
// pressure_op's cxp at i and cxm at i+1 (the sum in the division commutes);
// cy likewise in y.  Bit for bit pressure_op's result.
template <class Get>
__device__ __forceinline__ double spec_op(const SpecArgs &A, int i, int j, Get get)
{
    const int P = A.d.P;
    const double c = get(i, j);
    const double val = AT_(A.cx, i, j) * (get(i + 1, j) - c) - AT_(A.cx, i - 1, j) * (c - get(i - 1, j)) +
                       AT_(A.cy, i, j) * (get(i, j + 1) - c) - AT_(A.cy, i, j - 1) * (c - get(i, j - 1));
    return 1.0 * val;
}

__device__ __forceinline__ int src_x(const SpecArgs &A, int i) { return A.mp.x.src[i + NG]; }
__device__ __forceinline__ int src_y(const SpecArgs &A, int j) { return A.mp.y.src[j + NG]; }

// half-complex index of the q-th system: 0, N/2, then 1, N-1, 2, N-2, ...,
// so the two indices of one wave number (same matrix, same table entries)
// sit in neighbouring lanes
__device__ __forceinline__ int system_index(int q, int N)
{
    if (q < 2) return q == 0 ? 0 : N / 2;
    return (q & 1) ? N - (q >> 1) : (q >> 1);
}

__device__ __forceinline__ double warp_total(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The tridiagonal solves of every half-complex index, hat in place.  A
// block takes SPEC_SYS systems at a time: their columns are loaded into
// shared memory (coalesced: the systems are enumerated so that a group holds
// two runs of neighbouring indices), warp s solves system s, and the columns
// go back.  Per warp, with the table T of the system's wave number
// (spec_tables: for chunk row i >= 1 the elimination pivot r_i in
// T[i][lane] and the first-unknown coupling A_i in T[K + i][lane]; the
// chunk's c_0 in T[0][lane], a_0 in T[K][lane]; the reduced system's Thomas
// pivots in T[2K .. 2K + 3][lane]):
//   lane l, rows s_l .. s_l + L - 1 of its chunk:
//     down   D_1 = r_1 d_1, D_i = r_i (d_i + D_{i-1}): row i now reads
//            x_i + A_i x_first + C_i x_{i+1} = D_i (C_i = -r_i inside)
//     up     E_{L-1} = 0, E_i = D_i + r_i E_{i+1} down to E_1
//     the chunk's two equations: row 0 with x_1 eliminated (right-hand side
//     d_0 - c_0 E_1) and row L - 1 as it stands after the down sweep
//   lane 0: the Thomas algorithm over the 2P equations, pivots from the table
//   lane l: x_first, x_last from it, then x_i = D_i - A_i x_first + r_i x_{i+1}
//           for i = L - 2 .. 1
// The mean mode (m = 0) is made mean-free with its first row pinned on the
// way in, and given the right-hand side's mean back on the way out.
// asynchronous 8-byte global -> shared copies (cp.async): all of a thread's
// copies are in flight together, and no register holds them
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gmem_src)
{
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// shared-memory layout of the solve phase (doubles after the twiddles): the
// row groups' rows overlap the systems' columns and reduction scratch; the
// tables come after both
__host__ __device__ inline size_t spec_tab_offset(int N, int M)
{
    const size_t rows = (size_t)ROWG * N * 2;
    const size_t cols = (size_t)SPEC_SYS * ((size_t)M + (M >> 5) + 1 + 256);
    return rows > cols ? rows : cols;
}

// the table rows of the sweeps (pivots and couplings, 2K x 32 per system) of
// the block's systems q0 .. q0 + SPEC_SYS - 1 into shared memory
__device__ void stage_tables(const SpecArgs &A, double *tabs, int q0)
{
    const int N = A.N;
    const int K = spec_chunks(A.M).K, TW = (2 * K + 4) * 32, TS = 2 * K * 32;
    for (int e = threadIdx.x; e < SPEC_SYS * TS; e += blockDim.x) {
        const int s = e / TS, r = e - s * TS;
        if (q0 + s >= N) continue;
        const int m = system_index(q0 + s, N);
        cp_async8(tabs + e, A.tri + (size_t)(m <= N / 2 ? m : N - m) * TW + r);
    }
}

__device__ void tridiag_phase(const SpecArgs &A, double *area, bool resident)
{
    const int N = A.N, M = A.M, P = A.d.P;
    const Chunks ch = spec_chunks(M);
    const int K = ch.K, TW = (2 * K + 4) * 32, TS = 2 * K * 32;
    const int CP = M + (M >> 5) + 1;
    double *cols = area;                      // SPEC_SYS columns of CP doubles
    double *red = area + SPEC_SYS * CP;       // per warp: rhs, lower coupling, pivot, c' of the 2P equations
    double *tabs = area + spec_tab_offset(N, M);   // per system: the table's pivot and coupling rows (2K x 32)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q0 = blockIdx.x * SPEC_SYS; q0 < N; q0 += gridDim.x * SPEC_SYS) {
        __syncthreads();   // the previous group's columns are stored
        for (int e = threadIdx.x; e < SPEC_SYS * M; e += blockDim.x) {
            const int j = e / SPEC_SYS, s = e - j * SPEC_SYS;
            if (q0 + s < N) cp_async8(cols + s * CP + cidx(j), &AT_(A.hat, system_index(q0 + s, N), j));
        }
        // with one group per block the tables stay in shared memory for the
        // whole solve (staged before the first iteration)
        if (!resident) stage_tables(A, tabs, q0);
        cp_async_wait_all();
        __syncthreads();
        const int q = q0 + warp;
        if (warp < SPEC_SYS && q < N) {
            double *col = cols + warp * CP;
            double *rw = red + warp * 256;
            const int m = system_index(q, N);
            const int wave = m <= N / 2 ? m : N - m;
            const double *__restrict__ T = A.tri + (size_t)wave * TW;   // rows 2K.. (the reduced system)
            const double *St = tabs + warp * TS;                          // rows 0 .. 2K-1, staged
            double rmean = 0.0;
            if (m == 0) {   // mean-free, first row pinned
                double sum = 0.0;
                for (int j = lane; j < M; j += 32) sum += col[cidx(j)];
                rmean = warp_total(sum) / (double)M;
                for (int j = lane; j < M; j += 32) col[cidx(j)] = j == 0 ? 0.0 : col[cidx(j)] - rmean;
                __syncwarp();
            }
            const int len = lane < ch.P ? ch.base + (lane < ch.rem ? 1 : 0) : 0;
            const int st = lane * ch.base + (lane < ch.rem ? lane : ch.rem);
            if (len > 0) {
                double Dp = 0.0;
#pragma unroll 4
                for (int i = 1; i < len; i++) {
                    const int c = cidx(st + i);
                    const double r = St[i * 32 + lane], dv = col[c];
                    Dp = i == 1 ? r * dv : r * (dv + Dp);
                    col[c] = Dp;
                }
                double E = 0.0;
#pragma unroll 4
                for (int i = len - 2; i >= 1; i--) E = col[cidx(st + i)] + St[i * 32 + lane] * E;
                rw[2 * lane] = col[cidx(st)] - St[lane] * E;
                rw[2 * lane + 1] = Dp;
                rw[64 + 2 * lane] = St[K * 32 + lane];
                rw[64 + 2 * lane + 1] = St[(K + len - 1) * 32 + lane];
                rw[128 + 2 * lane] = T[(2 * K) * 32 + lane];
                rw[192 + 2 * lane] = T[(2 * K + 1) * 32 + lane];
                rw[128 + 2 * lane + 1] = T[(2 * K + 2) * 32 + lane];
                rw[192 + 2 * lane + 1] = T[(2 * K + 3) * 32 + lane];
            }
            __syncwarp();
            if (lane == 0) {   // the reduced system: 2P equations, Thomas
                const int n2 = 2 * ch.P;
                double prev = 0.0;
#pragma unroll 8
                for (int k = 0; k < n2; k++) {
                    prev = (rw[k] - rw[64 + k] * prev) * rw[128 + k];
                    rw[k] = prev;
                }
                double nxt = 0.0;
#pragma unroll 8
                for (int k = n2 - 1; k >= 0; k--) {
                    nxt = rw[k] - rw[192 + k] * nxt;
                    rw[k] = nxt;
                }
            }
            __syncwarp();
            if (len > 0) {
                const double x0 = rw[2 * lane], x1 = rw[2 * lane + 1];
                col[cidx(st)] = x0;
                col[cidx(st + len - 1)] = x1;
                double xn = x1;
#pragma unroll 4
                for (int i = len - 2; i >= 1; i--) {
                    const int c = cidx(st + i);
                    xn = col[c] - St[(K + i) * 32 + lane] * x0 + St[i * 32 + lane] * xn;
                    col[c] = xn;
                }
            }
            if (m == 0) {
                // the constant mode, the operator's null space, gets eigenvalue
                // 1 (in units of 1 / dy^2) instead of 0: the mean-free solution
                // plus the right-hand side's mean, so the scaled
                // preconditioner stays positive definite
                __syncwarp();
                double sum = 0.0;
                for (int j = lane; j < M; j += 32) sum += col[cidx(j)];
                const double mean = warp_total(sum) / (double)M;
                for (int j = lane; j < M; j += 32) col[cidx(j)] = col[cidx(j)] - mean + rmean;
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < SPEC_SYS * M; e += blockDim.x) {
            const int j = e / SPEC_SYS, s = e - j * SPEC_SYS;
            if (q0 + s < N) AT_(A.hat, system_index(q0 + s, N), j) = cols[s * CP + cidx(j)];
        }
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
    double *work = smem + N;   // N / 2 complex twiddles before it; the row groups' rows, or the systems' columns
    double2 *row = reinterpret_cast<double2 *>(work) + (size_t)grp * N;
    double *slotA = A.part, *slotB = A.part + gridDim.x, *slotC = A.part + 2 * gridDim.x;
    SpecScal *S = A.s;
    int *err = &A.scal->error;
    if (threadIdx.x == 0) spec_bar_target = 0;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    for (int k = threadIdx.x; k < N / 2; k += blockDim.x) tw[k] = A.tw[k];
    __syncthreads();
    SpecArgs B = A;
    B.tw = tw;

    // the solve's constants: face coefficients (x faces i = -1 .. N-1 of rows
    // 0 .. M-1, y faces j = -1 .. M-1 of columns 0 .. N-1) and the square roots
    // of the Jacobi weights, from the density's ghosted plane
    {
        const double idx2 = d.m.idx_c[1] * d.m.idx_c[1], idy2 = d.m.idy_c[1] * d.m.idy_c[1];
        const int W = N + 1, cells = W * (M + 1);
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cells; e += gridDim.x * blockDim.x) {
            const int j = e / W - 1, i = e - (j + 1) * W - 1;
            if (j >= 0) AT_(A.cx, i, j) = (2.0 / (AT_(A.rho, i, j) + AT_(A.rho, i + 1, j))) * idx2;
            if (i >= 0) AT_(A.cy, i, j) = (2.0 / (AT_(A.rho, i, j) + AT_(A.rho, i, j + 1))) * idy2;
            if (i >= 0 && j >= 0) AT_(A.sm, i, j) = sqrt(AT_(A.MJ, i, j));
        }
    }
    // one group of systems per block: its tables are staged once for the solve
    const bool resident = (int)gridDim.x * SPEC_SYS >= N;
    if (resident) {
        stage_tables(A, work + spec_tab_offset(N, M), blockIdx.x * SPEC_SYS);
        cp_async_wait_all();
    }
    if (!spec_barrier(S, err)) return;

    // r = rhs - A phi, the stopping sum, forward transforms
    auto residual = [&](int i, int j, double &sum) {
        const double ad = spec_op(A, i, j, [&](int a, int b) { return remap(A.mp, A.phi, P, NX, NY, a, b); });
        const double rv = AT_(A.rhs, i, j) - ad;
        AT_(A.res, i, j) = rv;
        sum += rv * (rv * AT_(A.MJ, i, j));
        return rv * AT_(A.sm, i, j);
    };
    double sJ = 0.0;
    for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG) {
        const int ja = 2 * (p0 + grp), jb = ja + 1;
        const bool acta = ja < M, actb = jb < M;
        if (acta)
            for (int i = lt; i < N; i += ROW_THREADS) {
                const double va = residual(i, ja, sJ);
                row[row_slot(A, i)] = make_double2(va, actb ? residual(i, jb, sJ) : 0.0);
            }
        pair_forward(B, row, ja, acta, actb, lt);
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
        tridiag_phase(A, work, resident);
        if (!spec_barrier(S, err)) return;
        double g = 0.0;
        for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG) {
            const int ja = 2 * (p0 + grp), jb = ja + 1;
            const bool acta = ja < M, actb = jb < M;
            if (acta)
                for (int k = lt; k < N; k += ROW_THREADS) {
                    const double2 xa = half_complex(A, k, ja);
                    const double2 xb = actb ? half_complex(A, k, jb) : make_double2(0.0, 0.0);
                    row[row_slot(A, k)] = make_double2(xa.x - xb.y, xa.y + xb.x);   // X_a + i X_b
                }
            __syncthreads();
            fft_rows(row, N, A.n, A.logN, A.R, tw, 1.0, lt);
            if (acta)
                for (int i = lt; i < N; i += ROW_THREADS) {
                    const double2 v = row[i];
                    const double za = v.x * AT_(A.sm, i, ja);
                    AT_(A.z, i, ja) = za;
                    g += AT_(A.res, i, ja) * za;
                    if (actb) {
                        const double zb = v.y * AT_(A.sm, i, jb);
                        AT_(A.z, i, jb) = zb;
                        g += AT_(A.res, i, jb) * zb;
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
        for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG)
            for (int h = 0; h < 2; h++) {
                const int j = 2 * (p0 + grp) + h;
                if (j >= M) continue;
                for (int i = lt; i < N; i += ROW_THREADS) {
                    const double dv = dir(i, j);
                    AT_(dnew, i, j) = dv;
                    const double ad = spec_op(A, i, j, dir);
                    AT_(A.Ad, i, j) = ad;
                    sdad += dv * ad;
                }
            }
        put_part(sdad, slotC, sh);
        if (!spec_barrier(S, err)) return;
        const double alpha = gamma / (slot_total(slotC, sh) + 1e-300);
        // phi += alpha d, r -= alpha Ad, the stopping sum, forward transforms
        auto update = [&](int i, int j, double &sum) {
            AT_(A.phi, i, j) += alpha * AT_(dnew, i, j);
            const double rv = AT_(A.res, i, j) - alpha * AT_(A.Ad, i, j);
            AT_(A.res, i, j) = rv;
            sum += rv * (rv * AT_(A.MJ, i, j));
            return rv * AT_(A.sm, i, j);
        };
        sJ = 0.0;
        for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG) {
            const int ja = 2 * (p0 + grp), jb = ja + 1;
            const bool acta = ja < M, actb = jb < M;
            if (acta)
                for (int i = lt; i < N; i += ROW_THREADS) {
                    const double va = update(i, ja, sJ);
                    row[row_slot(A, i)] = make_double2(va, actb ? update(i, jb, sJ) : 0.0);
                }
            pair_forward(B, row, ja, acta, actb, lt);
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
    for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG)
        for (int h = 0; h < 2; h++) {
            const int j = 2 * (p0 + grp) + h;
            if (j >= M) continue;
            for (int i = lt; i < N; i += ROW_THREADS) ssum += AT_(A.phi, i, j);
        }
    put_part(ssum, slotB, sh);
    if (!spec_barrier(S, err)) return;
    const double avg = slot_total(slotB, sh) / ((double)N * (double)M);
    for (int p0 = blockIdx.x * ROWG; 2 * p0 < M; p0 += gridDim.x * ROWG)
        for (int h = 0; h < 2; h++) {
            const int j = 2 * (p0 + grp) + h;
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
    int n = N;
    while (n % 2 == 0 && n > 1) n /= 2;   // the odd factor
    if (N < 2 || N > 1024 || N % 2 != 0 || (n != 1 && n != 3 && n != 5) || N / n < 2) {
        *why = "the spectral pressure preconditioner needs an x cell count of 2^a, 3 2^a or 5 2^a (2..1024)";
        return false;
    }
    if (M < 2 || M > 1024) { *why = "the spectral pressure preconditioner needs 2 to 1024 y cells"; return false; }
    return true;
}

int spec_tables(int N, int M, double idx2, double idy2, std::vector<double> &tw, std::vector<double> &tri)
{
    tw.assign(N, 0.0);   // N / 2 complex entries exp(-2 pi i k / N)
    for (int k = 0; k < N / 2; k++) {
        tw[2 * k] = std::cos(2.0 * M_PI * k / N);
        tw[2 * k + 1] = -std::sin(2.0 * M_PI * k / N);
    }
    // per wave number, (2K + 4) rows of 32 (one entry per chunk): the
    // coefficients of tridiag_phase for a_j z_{j-1} + b_j z_j + c_j z_{j+1} = r_j
    // (a = c = -1 inside)
    const Chunks ch = spec_chunks(M);
    const int K = ch.K, TW = (2 * K + 4) * 32, NW = N / 2 + 1;
    tri.assign((size_t)NW * TW, 0.0);
    std::vector<double> R(K), Ac(K), Cc(K), lo(2 * ch.P), di(2 * ch.P), up(2 * ch.P);
    for (int w = 0; w < NW; w++) {
        const double lam = (2.0 - 2.0 * std::cos(2.0 * M_PI * w / N)) * idx2 / idy2;
        auto coef = [&](int j, double &a, double &b, double &c) {
            if (w == 0 && j == 0) { a = 0.0; b = 1.0; c = 0.0; return; }   // the pinned row
            a = j > 0 ? -1.0 : 0.0;
            c = j < M - 1 ? -1.0 : 0.0;
            b = lam + (j > 0 ? 1.0 : 0.0) + (j < M - 1 ? 1.0 : 0.0);
        };
        double *T = tri.data() + (size_t)w * TW;
        for (int l = 0; l < ch.P; l++) {
            const int L = ch.base + (l < ch.rem ? 1 : 0), s = l * ch.base + (l < ch.rem ? l : ch.rem);
            // down: row i (>= 1) becomes x_i + A_i x_0 + C_i x_{i+1} = D_i
            for (int i = 1; i < L; i++) {
                double a, b, c;
                coef(s + i, a, b, c);
                R[i] = i == 1 ? 1.0 / b : 1.0 / (b - a * Cc[i - 1]);
                Ac[i] = i == 1 ? a * R[i] : -a * R[i] * Ac[i - 1];
                Cc[i] = c * R[i];
                T[i * 32 + l] = R[i];
                T[(K + i) * 32 + l] = Ac[i];
            }
            // up: x_1 = E_1 - F_1 x_0 - G_1 x_{L-1}
            double F = 0.0, G = -1.0;
            for (int i = L - 2; i >= 1; i--) {
                F = Ac[i] - Cc[i] * F;
                G = -Cc[i] * G;
            }
            double a0, b0, c0;
            coef(s, a0, b0, c0);
            T[l] = c0;
            T[K * 32 + l] = a0;
            lo[2 * l] = a0;  di[2 * l] = b0 - c0 * F;  up[2 * l] = -c0 * G;
            lo[2 * l + 1] = Ac[L - 1];  di[2 * l + 1] = 1.0;  up[2 * l + 1] = Cc[L - 1];
        }
        // the reduced system's Thomas pivots
        double cprev = 0.0;
        for (int k = 0; k < 2 * ch.P; k++) {
            const double inv = 1.0 / (di[k] - lo[k] * cprev);
            cprev = up[k] * inv;
            T[(2 * K + 2 * (k & 1)) * 32 + k / 2] = inv;
            T[(2 * K + 2 * (k & 1) + 1) * 32 + k / 2] = cprev;
        }
    }
    return M;
}

size_t spec_pcg_smem(int N, int M)
{
    // twiddles, the rows / columns area, the tables
    return ((size_t)N + spec_tab_offset(N, M) + (size_t)SPEC_SYS * 64 * spec_chunks(M).K) * sizeof(double);
}

// blocks for k_spec_pcg: enough for one pass over the rows and the systems,
// at most what is co-resident; 0 if the launch cannot be cooperative
int spec_pcg_blocks(int device, int N, int M)
{
    const size_t smem = spec_pcg_smem(N, M);
    if (smem > 48 * 1024 &&
        !raise_dynamic_smem((const void *)k_spec_pcg, smem))
        return 0;
    int per_sm = 0, sms = 0, coop = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spec_pcg, SPEC_PT, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    int want = (M + 2 * ROWG - 1) / (2 * ROWG);   // the tridiagonal phase loops over its systems: any block count works
    const int most = per_sm * sms;
    return most < 1 ? 0 : (want < most ? want : most);
}

const void *spec_pcg_kernel() { return (const void *)k_spec_pcg; }

cudaError_t spec_launch_pcg(const SpecArgs &A, int blocks, double *d0, double *d1, cudaStream_t st)
{
    SpecArgs a = A;
    void *args[] = {&a, &d0, &d1};
    // the grid barriers count arrivals from zero
    const cudaError_t e = cudaMemsetAsync(&A.s->arrivals, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel((const void *)k_spec_pcg, dim3((unsigned)blocks), dim3(SPEC_PT), args,
                                       spec_pcg_smem(A.N, A.M), st);
}

}  // namespace pvof
