// CUDA executor of the 3D mode and its entry points (called from the C ABI
// in pvof_api.cu when a context is created with PVOF_GEOM_3D).
//
// Launch shapes: a box of cells is walked row by row, one warp per (j,k)
// row and 32 consecutive i per step, so every field access of a warp is one
// coalesced run along i; grids are capped at a multiple of the SM count and
// stride over the remaining rows.  Reductions write one partial per block
// (a fixed grid of at most NBR blocks) and a one-block scalar kernel adds
// the partials in a fixed order, so every sum is the same from run to run.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "pvof_3d.cuh"
#include "pvof_3d_api.h"

namespace pvof3 {

constexpr int TPB = 256;
constexpr int WPB = TPB / 32;
constexpr int NBR = 148 * 8;        // most blocks of a reduction
constexpr int NBC = 148 * 16;       // most blocks of a cell-wise pass

thread_local std::string g_err3;
const char *last_error() { return g_err3.c_str(); }
static int fail(int code, const std::string &m)
{
    g_err3 = m;
    return code;
}

template <class F>
__global__ void __launch_bounds__(TPB) k3_cells(Range r, const int *gate, F f)
{
    if (gate && *gate == 0) return;
    const int nj = r.j1 - r.j0;
    const long long nrows = (long long)nj * (r.k1 - r.k0);
    const int lane = threadIdx.x & 31;
    for (long long row = (long long)blockIdx.x * WPB + (threadIdx.x >> 5); row < nrows; row += (long long)gridDim.x * WPB) {
        const int j = r.j0 + (int)(row % nj), k = r.k0 + (int)(row / nj);
        for (int i = r.i0 + lane; i < r.i1; i += 32) f(i, j, k);
    }
}

template <int N, bool MAX, class F>
__global__ void __launch_bounds__(TPB) k3_reduce(Range r, const int *gate, double *part, F f)
{
    __shared__ double sh[WPB][N];
    if (gate && *gate == 0) return;
    double acc[N];
#pragma unroll
    for (int q = 0; q < N; q++) acc[q] = 0.0;
    const int nj = r.j1 - r.j0;
    const long long nrows = (long long)nj * (r.k1 - r.k0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long row = (long long)blockIdx.x * WPB + warp; row < nrows; row += (long long)gridDim.x * WPB) {
        const int j = r.j0 + (int)(row % nj), k = r.k0 + (int)(row / nj);
        for (int i = r.i0 + lane; i < r.i1; i += 32) {
            const Vec<N> t = f(i, j, k);
#pragma unroll
            for (int q = 0; q < N; q++) acc[q] = MAX ? fmax(acc[q], t.v[q]) : acc[q] + t.v[q];
        }
    }
#pragma unroll
    for (int q = 0; q < N; q++) {
        double a = acc[q];
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_down_sync(0xffffffffu, a, o);
            a = MAX ? fmax(a, b) : a + b;
        }
        if (lane == 0) sh[warp][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double a = sh[0][threadIdx.x];
        for (int w = 1; w < WPB; w++) a = MAX ? fmax(a, sh[w][threadIdx.x]) : a + sh[w][threadIdx.x];
        part[(size_t)blockIdx.x * 4 + threadIdx.x] = a;
    }
}

struct Pend {
    int nb[NSLOT], nq[NSLOT], mx[NSLOT];
    unsigned mask;
    int stride;   // partial sums per slot (blocks), times 4 values
};

template <class F>
__global__ void __launch_bounds__(TPB) k3_scalar(const double *part, Pend pd, const int *gate, Sc3 *sc, F f)
{
    __shared__ double sh[TPB];
    if (gate && *gate == 0) return;
    for (int s = 0; s < NSLOT; s++) {
        if (!(pd.mask & (1u << s))) continue;
        for (int q = 0; q < pd.nq[s]; q++) {
            double a = 0.0;
            for (int b = threadIdx.x; b < pd.nb[s]; b += TPB) {
                const double v = part[(size_t)s * pd.stride + (size_t)b * 4 + q];
                a = pd.mx[s] ? fmax(a, v) : a + v;
            }
            sh[threadIdx.x] = a;
            __syncthreads();
            for (int w = TPB / 2; w > 0; w >>= 1) {
                if (threadIdx.x < w) sh[threadIdx.x] = pd.mx[s] ? fmax(sh[threadIdx.x], sh[threadIdx.x + w]) : sh[threadIdx.x] + sh[threadIdx.x + w];
                __syncthreads();
            }
            if (threadIdx.x == 0) sc->sum[s][q] = sh[0];
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) f(sc);
}

// ---------------------------------------------------------------------------
// the pressure PCG iteration (psolve_cg.c:209-253) as three streaming kernels
// over the physical cells: a thread takes two neighbouring cells of a row
// (16-byte loads; i = 0 is 16-byte aligned and every row and plane pitch is
// even) in PKB consecutive planes, a block a 64 x 8 tile of (i, j); PKB
// planes per block keep the end-of-block reduction barrier and the number of
// partial sums small.  Reads at
// ghost and half cells go through the pressure ghost map; the arithmetic is
// that of p_apply_st and of the reference's loops, operand for operand.
// ---------------------------------------------------------------------------
constexpr int PKB = 4;

__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ void st2(double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); }

// the cells (i, i+1) of a pressure field at (j, k), after the ghost update
__device__ __forceinline__ void p_pair(const Dom3 &d, const double *__restrict__ X, int i, int j, int k, double &a,
                                       double &b)
{
    if (j >= 0 && j <= d.NY - 2 && k >= 0 && k <= d.NZ - 2) {
        const double2 v = ld2(X + at(d, i, j, k));
        a = v.x;
        b = v.y;
    } else {
        a = rd<K_PRESSURE>(d, X, i, j, k);
        b = rd<K_PRESSURE>(d, X, i + 1, j, k);
    }
}

// The block's sum into part[block]; the last block to finish adds all the
// partials in block order (the same order whichever block is last) and runs
// the scalar step then(sc, sum) on one thread, so no separate launch is
// needed between the passes.
template <class F>
__device__ __forceinline__ void block_sum_then(double acc, double *part, Sc3 *sc, F then)
{
    __shared__ double sh[256];
    __shared__ bool last;
    const int t = threadIdx.x + 32 * threadIdx.y;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) sh[threadIdx.y] = acc;
    __syncthreads();
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    if (t == 0) {
        double a = sh[0];
        for (int q = 1; q < 8; q++) a += sh[q];
        part[(size_t)(blockIdx.x + gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z)) * 4] = a;
        __threadfence();
        last = (atomicAdd(&sc->p_count, 1u) == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // eight loads in flight per thread; the order of the additions is fixed
    double a = 0.0;
    unsigned b = t;
    for (; b + 7 * 256 < nb; b += 8 * 256) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = __ldcg(part + (size_t)(b + u * 256) * 4);
#pragma unroll
        for (int u = 0; u < 8; u++) a += v[u];
    }
    for (; b < nb; b += 256) a += __ldcg(part + (size_t)b * 4);
    sh[t] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    if (t == 0) {
        sc->p_count = 0;
        then(sc, sh[0]);
    }
}

template <class F>
__global__ void __launch_bounds__(256, 4) k3p_apply(Dom3 d, const double *__restrict__ CX, const double *__restrict__ CY,
                                                    const double *__restrict__ CZ, const double *__restrict__ X,
                                                    double *__restrict__ AD, const int *gate, double *part, Sc3 *sc,
                                                    F then)
{
    if (gate && *gate == 0) return;
    const int ni = d.NX - 1, nj = d.NY - 1, nk = d.NZ - 1;
    const int i = 2 * (blockIdx.x * 32 + threadIdx.x), j = blockIdx.y * 8 + threadIdx.y;
    double acc = 0.0;
    if (i < ni && j < nj) {
        const bool two = i + 1 < ni;
#pragma unroll 1
        for (int kk = 0; kk < PKB; kk++) {
            const int k = blockIdx.z * PKB + kk;
            if (k >= nk) break;
            const long long q = at(d, i, j, k);
            if (!two) {
                const double ad = p_apply_st(d, CX, CY, CZ, X, i, j, k);
                AD[q] = ad;
                acc += X[q] * ad;
                continue;
            }
            const double2 c = ld2(X + q);
            const double w0 = (i >= 1) ? X[q - 1] : rd<K_PRESSURE>(d, X, i - 1, j, k);
            const double e1 = (i + 2 <= ni - 1) ? X[q + 2] : rd<K_PRESSURE>(d, X, i + 2, j, k);
            double s0, s1, n0, n1, b0, b1, f0, f1;
            p_pair(d, X, i, j - 1, k, s0, s1);
            p_pair(d, X, i, j + 1, k, n0, n1);
            p_pair(d, X, i, j, k - 1, b0, b1);
            p_pair(d, X, i, j, k + 1, f0, f1);
            const double2 cx = ld2(CX + q), cy = ld2(CY + q), cz = ld2(CZ + q);
            const double2 cym = ld2(CY + q - d.P), czm = ld2(CZ + q - d.S);
            const double cxm = CX[q - 1];
            const double v0 = cx.x * (c.y - c.x) - cxm * (c.x - w0) + cy.x * (n0 - c.x) - cym.x * (c.x - s0) +
                              cz.x * (f0 - c.x) - czm.x * (c.x - b0);
            const double v1 = cx.y * (e1 - c.y) - cx.x * (c.y - c.x) + cy.y * (n1 - c.y) - cym.y * (c.y - s1) +
                              cz.y * (f1 - c.y) - czm.y * (c.y - b1);
            const double ad0 = 1.0 * v0, ad1 = 1.0 * v1;
            st2(AD + q, ad0, ad1);
            acc += c.x * ad0;
            acc += c.y * ad1;
        }
    }
    block_sum_then(acc, part, sc, then);
}

template <class F>
__global__ void __launch_bounds__(256) k3p_update(Dom3 d, double *__restrict__ PHI, double *__restrict__ R,
                                                  const double *__restrict__ DD, const double *__restrict__ AD,
                                                  const double *__restrict__ M, const int *gate, Sc3 *sc,
                                                  double *part, F then)
{
    if (gate && *gate == 0) return;
    const int ni = d.NX - 1, nj = d.NY - 1, nk = d.NZ - 1;
    const int i = 2 * (blockIdx.x * 32 + threadIdx.x), j = blockIdx.y * 8 + threadIdx.y;
    const double alpha = sc->p_alpha;
    double acc = 0.0;
    if (i < ni && j < nj) {
        const bool two = i + 1 < ni;
#pragma unroll
        for (int kk = 0; kk < PKB; kk++) {
            const int k = blockIdx.z * PKB + kk;
            if (k >= nk) break;
            const long long q = at(d, i, j, k);
            if (!two) {
                PHI[q] += alpha * DD[q];
                const double r = R[q] - alpha * AD[q];
                R[q] = r;
                acc += r * (r * M[q]);
                continue;
            }
            const double2 x = ld2(PHI + q), dd = ld2(DD + q), r = ld2(R + q), ad = ld2(AD + q), m = ld2(M + q);
            st2(PHI + q, x.x + alpha * dd.x, x.y + alpha * dd.y);
            const double r0 = r.x - alpha * ad.x, r1 = r.y - alpha * ad.y;
            st2(R + q, r0, r1);
            acc += r0 * (r0 * m.x);
            acc += r1 * (r1 * m.y);
        }
    }
    block_sum_then(acc, part, sc, then);
}

__global__ void __launch_bounds__(256) k3p_dir(Dom3 d, const double *__restrict__ R, const double *__restrict__ M,
                                               double *__restrict__ DD, const int *gate, const Sc3 *sc)
{
    if (gate && *gate == 0) return;
    const int ni = d.NX - 1, nj = d.NY - 1, nk = d.NZ - 1;
    const int i = 2 * (blockIdx.x * 32 + threadIdx.x), j = blockIdx.y * 8 + threadIdx.y;
    if (i >= ni || j >= nj) return;
    const double beta = sc->p_beta;
    const bool two = i + 1 < ni;
#pragma unroll
    for (int kk = 0; kk < PKB; kk++) {
        const int k = blockIdx.z * PKB + kk;
        if (k >= nk) break;
        const long long q = at(d, i, j, k);
        if (!two) {
            DD[q] = R[q] * M[q] + beta * DD[q];
            continue;
        }
        const double2 r = ld2(R + q), m = ld2(M + q), dd = ld2(DD + q);
        st2(DD + q, r.x * m.x + beta * dd.x, r.y * m.y + beta * dd.y);
    }
}

// ---------------------------------------------------------------------------
// spectral preconditioner of the 3D pressure PCG (pressure_preconditioner = 1):
// z = s (-L)^-1 (s r), s = sqrt of the Jacobi weights, L the 7-point operator at
// density one with the reference's ghost rules (x, z periodic, mirror walls in
// y).  A real transform along x (N cells) and a complex one along z (K cells)
// diagonalise L into one tridiagonal system in y per (kx, kz), solved by the
// Thomas algorithm from host tables; the constant mode (the operator's null
// space) gets eigenvalue 1 in units of 1/dy^2.  Spectrum layout: element
// (kx, j, kz) at ((kz * ny + j) * H + kx), H = N/2 + 1.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// twiddles w[q] = exp(sign 2 pi i q / n), q < n/2, into shared memory from
// the table of exp(-2 pi i q / n) made once on the host
__device__ __forceinline__ void fft_twiddles(double2 *w, const double2 *__restrict__ tab, int n, double sign)
{
    for (int q = threadIdx.x; q < n / 2; q += blockDim.x) {
        const double2 v = tab[q];
        w[q] = make_double2(v.x, sign < 0.0 ? v.y : -v.y);
    }
}

// in-place radix-2 transform of a[0..n) (n = 2^logn) by the nt threads of
// one group (t = the thread's index in it); every thread of the block runs
// the same stages, so the block barriers line up
__device__ __forceinline__ void fft_group(double2 *a, const double2 *w, int n, int logn, int t, int nt)
{
    for (int q = t; q < n; q += nt) {
        const int r = (int)(__brev((unsigned)q) >> (32 - logn));
        if (r > q) {
            const double2 x = a[q];
            a[q] = a[r];
            a[r] = x;
        }
    }
    __syncthreads();
    // two radix-2 stages per pass over shared memory: a thread takes the four
    // elements the two stages combine (the same butterflies and twiddles as
    // one stage at a time, so the same numbers), half the shared-memory round
    // trips and barriers
    int s = 1;
    for (; s + 1 <= logn; s += 2) {
        const int h = 1 << (s - 1), st0 = n >> s, st1 = n >> (s + 1);
        for (int b = t; b < n / 4; b += nt) {
            const int pos = b & (h - 1), p = ((b >> (s - 1)) << (s + 1)) + pos;
            const double2 x0 = a[p], x1 = a[p + h], x2 = a[p + 2 * h], x3 = a[p + 3 * h];
            const double2 w0 = w[pos * st0];
            const double2 v1 = cmul(w0, x1), v3 = cmul(w0, x3);
            const double2 y0 = make_double2(x0.x + v1.x, x0.y + v1.y), y1 = make_double2(x0.x - v1.x, x0.y - v1.y);
            const double2 y2 = make_double2(x2.x + v3.x, x2.y + v3.y), y3 = make_double2(x2.x - v3.x, x2.y - v3.y);
            const double2 u2 = cmul(w[pos * st1], y2), u3 = cmul(w[(pos + h) * st1], y3);
            a[p] = make_double2(y0.x + u2.x, y0.y + u2.y);
            a[p + 2 * h] = make_double2(y0.x - u2.x, y0.y - u2.y);
            a[p + h] = make_double2(y1.x + u3.x, y1.y + u3.y);
            a[p + 3 * h] = make_double2(y1.x - u3.x, y1.y - u3.y);
        }
        __syncthreads();
    }
    if (s == logn) {   // an odd number of stages: the last one alone
        const int half = 1 << (s - 1), stride = n >> s;
        for (int b = t; b < n / 2; b += nt) {
            const int pos = b & (half - 1), i0 = ((b >> (s - 1)) << s) + pos, i1 = i0 + half;
            const double2 u = a[i0], v = cmul(w[pos * stride], a[i1]);
            a[i0] = make_double2(u.x + v.x, u.y + v.y);
            a[i1] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

struct SpecDims {
    int N, logN, K, logK, ny, H;
    int nt_x, g_x;   // x transforms: threads per pair of rows, pairs per block
    int ch_z, nt_z;  // z transforms: columns per block, threads per column
};

// t = s r along two x rows at once (one as the real part, the other as the
// imaginary part of a complex row), forward transform, then the two half
// spectra separated, X_a = (Z_k + conj Z_(N-k)) / 2 and
// X_b = (Z_k - conj Z_(N-k)) / 2i, and stored
__global__ void __launch_bounds__(256) k3s_fwd_x(Dom3 d, SpecDims sd, const double *__restrict__ R,
                                                 const double *__restrict__ M, double2 *__restrict__ SP,
                                                 const double2 *__restrict__ TW, const int *gate)
{
    extern __shared__ double2 sm[];
    if (gate && *gate == 0) return;
    double2 *w = sm, *a = sm + sd.N / 2 + (threadIdx.x / sd.nt_x) * sd.N;
    fft_twiddles(w, TW, sd.N, -1.0);
    const int g = threadIdx.x / sd.nt_x, t = threadIdx.x % sd.nt_x;
    const long long rows = (long long)sd.K * sd.ny;
    const long long ra = 2 * ((long long)blockIdx.x * sd.g_x + g), rb = ra + 1;   // row = k * ny + j
    const bool la = ra < rows, lb = rb < rows;
    const int ja = la ? (int)(ra % sd.ny) : 0, ka = la ? (int)(ra / sd.ny) : 0;
    const int jb = lb ? (int)(rb % sd.ny) : 0, kb = lb ? (int)(rb / sd.ny) : 0;
    for (int i = t; i < sd.N; i += sd.nt_x) {
        double va = 0.0, vb = 0.0;
        if (la) {
            const long long q = at(d, i, ja, ka);
            va = sqrt(M[q]) * R[q];
        }
        if (lb) {
            const long long q = at(d, i, jb, kb);
            vb = sqrt(M[q]) * R[q];
        }
        a[i] = make_double2(va, vb);
    }
    __syncthreads();
    fft_group(a, w, sd.N, sd.logN, t, sd.nt_x);
    for (int kx = t; kx < sd.H; kx += sd.nt_x) {
        const double2 zk = a[kx], zn = a[(sd.N - kx) & (sd.N - 1)];
        if (la) SP[ra * sd.H + kx] = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y - zn.y));
        if (lb) SP[rb * sd.H + kx] = make_double2(0.5 * (zk.y + zn.y), -0.5 * (zk.x - zn.x));
    }
}

// complex transform along z of ch_z neighbouring kx columns at one j
__global__ void __launch_bounds__(256) k3s_z(SpecDims sd, double2 *__restrict__ SP, const double2 *__restrict__ TW,
                                             double sign, const int *gate)
{
    extern __shared__ double2 sm[];
    if (gate && *gate == 0) return;
    double2 *w = sm, *a = sm + sd.K / 2;
    fft_twiddles(w, TW, sd.K, sign);
    const int nchunk = (sd.H + sd.ch_z - 1) / sd.ch_z;
    const int j = blockIdx.x / nchunk, kx0 = (blockIdx.x % nchunk) * sd.ch_z;
    const int c = threadIdx.x / sd.nt_z, t = threadIdx.x % sd.nt_z;
    // load: element (kz, col) of the tile at a[col * K + kz]
    for (int e = threadIdx.x; e < sd.K * sd.ch_z; e += blockDim.x) {
        const int kz = e / sd.ch_z, col = e % sd.ch_z, kx = kx0 + col;
        a[col * sd.K + kz] = (kx < sd.H) ? SP[((long long)kz * sd.ny + j) * sd.H + kx] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_group(a + c * sd.K, w, sd.K, sd.logK, t, sd.nt_z);
    for (int e = threadIdx.x; e < sd.K * sd.ch_z; e += blockDim.x) {
        const int kz = e / sd.ch_z, col = e % sd.ch_z, kx = kx0 + col;
        if (kx < sd.H) SP[((long long)kz * sd.ny + j) * sd.H + kx] = a[col * sd.K + kz];
    }
}

// one tridiagonal system in y per (kx, kz): (m_j)^-1 and c'_j from the host
// tables; the right-hand side scaled by dy^2 / (N K) (the transforms' norm)
__global__ void __launch_bounds__(32) k3s_tri(SpecDims sd, double2 *__restrict__ SP, const double *__restrict__ CP,
                                               const double *__restrict__ IM, double scale, const int *gate)
{
    if (gate && *gate == 0) return;
    const long long sys = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sys >= (long long)sd.K * sd.H) return;
    const int kz = (int)(sys / sd.H), kx = (int)(sys % sd.H);
    const int ny = sd.ny;
    auto idx = [&](int j) { return ((long long)kz * ny + j) * sd.H + kx; };
    if (kx == 0 && kz == 0) {
        // the constant mode: the mean-free part by the recurrence of rows
        // 0..ny-2 from u_0 = 0, its mean removed, plus the mean itself
        double2 mean = make_double2(0.0, 0.0);
        for (int j = 0; j < ny; j++) {
            const double2 v = SP[idx(j)];
            mean.x += v.x;
            mean.y += v.y;
        }
        mean.x *= scale / ny;
        mean.y *= scale / ny;
        double2 um = make_double2(0.0, 0.0), uc = make_double2(0.0, 0.0), su = make_double2(0.0, 0.0);
        for (int j = 0; j < ny; j++) {
            double2 un;
            const double2 dj = SP[idx(j)];
            const double2 dd = make_double2(dj.x * scale - mean.x, dj.y * scale - mean.y);
            SP[idx(j)] = uc;
            su.x += uc.x;
            su.y += uc.y;
            if (j == 0) un = make_double2(uc.x - dd.x, uc.y - dd.y);
            else un = make_double2(2.0 * uc.x - um.x - dd.x, 2.0 * uc.y - um.y - dd.y);
            um = uc;
            uc = un;
        }
        su.x /= ny;
        su.y /= ny;
        for (int j = 0; j < ny; j++) {
            const double2 v = SP[idx(j)];
            SP[idx(j)] = make_double2(v.x - su.x + mean.x, v.y - su.y + mean.y);
        }
        return;
    }
    // both sweeps in runs of TU rows: a run's loads are all issued before its
    // dependent chain of updates (a thread's loads would otherwise wait one
    // memory latency per row)
    constexpr int TU = 8;
    double2 dp = make_double2(0.0, 0.0);
    for (int j0 = 0; j0 < ny; j0 += TU) {
        double2 v[TU];
        double m[TU];
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j0 + u < ny) {
                v[u] = SP[idx(j0 + u)];
                m[u] = IM[idx(j0 + u)];
            }
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j0 + u < ny) {
                dp = make_double2((v[u].x * scale + dp.x) * m[u], (v[u].y * scale + dp.y) * m[u]);
                v[u] = dp;
            }
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j0 + u < ny) SP[idx(j0 + u)] = v[u];
    }
    double2 x = dp;   // u_{ny-1}
    for (int j1 = ny - 2; j1 >= 0; j1 -= TU) {
        double2 v[TU];
        double c[TU];
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j1 - u >= 0) {
                v[u] = SP[idx(j1 - u)];
                c[u] = CP[idx(j1 - u)];
            }
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j1 - u >= 0) {
                x = make_double2(v[u].x - c[u] * x.x, v[u].y - c[u] * x.y);
                v[u] = x;
            }
#pragma unroll
        for (int u = 0; u < TU; u++)
            if (j1 - u >= 0) SP[idx(j1 - u)] = v[u];
    }
}

// the block's sum of a 1D block into part[block]; the last block adds them
// all in block order and runs then(sc, sum) (block_sum_then for 1D blocks)
template <class F>
__device__ __forceinline__ void block_sum_then_1d(double acc, double *part, Sc3 *sc, F then)
{
    __shared__ double sh[256];
    __shared__ bool last;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    const unsigned nb = gridDim.x;
    if (t == 0) {
        double a = sh[0];
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) a += sh[q];
        part[(size_t)blockIdx.x * 4] = a;
        __threadfence();
        last = (atomicAdd(&sc->p_count, 1u) == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0.0;
    unsigned b = t;
    for (; b + 7 * 256 < nb; b += 8 * 256) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = __ldcg(part + (size_t)(b + u * 256) * 4);
#pragma unroll
        for (int u = 0; u < 8; u++) a += v[u];
    }
    for (; b < nb; b += 256) a += __ldcg(part + (size_t)b * 4);
    sh[t] = a;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) sh[t] += sh[t + w];
        __syncthreads();
    }
    if (t == 0) {
        sc->p_count = 0;
        then(sc, sh[0]);
    }
}

// inverse transform along x of two rows at once (the complex row X_a + i X_b,
// each spectrum extended by its Hermitian symmetry; row a comes back as the
// real part, row b as the imaginary part), z = s u, and r.z
template <class F>
__global__ void __launch_bounds__(256) k3s_inv_x(Dom3 d, SpecDims sd, const double2 *__restrict__ SP,
                                                 const double *__restrict__ M, const double *__restrict__ R,
                                                 double *__restrict__ Z, const double2 *__restrict__ TW,
                                                 const int *gate, double *part, Sc3 *sc, F then)
{
    extern __shared__ double2 sm[];
    if (gate && *gate == 0) return;
    double2 *w = sm, *a = sm + sd.N / 2 + (threadIdx.x / sd.nt_x) * sd.N;
    fft_twiddles(w, TW, sd.N, 1.0);
    const int g = threadIdx.x / sd.nt_x, t = threadIdx.x % sd.nt_x;
    const long long rows = (long long)sd.K * sd.ny;
    const long long ra = 2 * ((long long)blockIdx.x * sd.g_x + g), rb = ra + 1;
    const bool la = ra < rows, lb = rb < rows;
    const int ja = la ? (int)(ra % sd.ny) : 0, ka = la ? (int)(ra / sd.ny) : 0;
    const int jb = lb ? (int)(rb % sd.ny) : 0, kb = lb ? (int)(rb / sd.ny) : 0;
    for (int kx = t; kx < sd.N; kx += sd.nt_x) {
        const bool lo = kx < sd.H;
        const int c = lo ? kx : sd.N - kx;
        const double sg = lo ? 1.0 : -1.0;
        double2 xa = make_double2(0.0, 0.0), xb = make_double2(0.0, 0.0);
        if (la) {
            const double2 v = SP[ra * sd.H + c];
            xa = make_double2(v.x, sg * v.y);
        }
        if (lb) {
            const double2 v = SP[rb * sd.H + c];
            xb = make_double2(v.x, sg * v.y);
        }
        a[kx] = make_double2(xa.x - xb.y, xa.y + xb.x);
    }
    __syncthreads();
    fft_group(a, w, sd.N, sd.logN, t, sd.nt_x);
    double acc = 0.0;
    for (int i = t; i < sd.N; i += sd.nt_x) {
        if (la) {
            const long long q = at(d, i, ja, ka);
            const double z = sqrt(M[q]) * a[i].x;
            Z[q] = z;
            acc += R[q] * z;
        }
        if (lb) {
            const long long q = at(d, i, jb, kb);
            const double z = sqrt(M[q]) * a[i].y;
            Z[q] = z;
            acc += R[q] * z;
        }
    }
    block_sum_then_1d(acc, part, sc, then);
}

// d = z + beta d (the spectral form's direction)
__global__ void __launch_bounds__(256) k3p_dir_z(Dom3 d, const double *__restrict__ Z, double *__restrict__ DD,
                                                 const int *gate, const Sc3 *sc)
{
    if (gate && *gate == 0) return;
    const int ni = d.NX - 1, nj = d.NY - 1, nk = d.NZ - 1;
    const int i = 2 * (blockIdx.x * 32 + threadIdx.x), j = blockIdx.y * 8 + threadIdx.y;
    if (i >= ni || j >= nj) return;
    const double beta = sc->p_beta;
    const bool two = i + 1 < ni;
    for (int kk = 0; kk < PKB; kk++) {
        const int k = blockIdx.z * PKB + kk;
        if (k >= nk) break;
        const long long q = at(d, i, j, k);
        if (!two) {
            DD[q] = Z[q] + beta * DD[q];
            continue;
        }
        const double2 z = ld2(Z + q), dd = ld2(DD + q);
        st2(DD + q, z.x + beta * dd.x, z.y + beta * dd.y);
    }
}

// host block (reference layout) <-> padded field
__global__ void k3_unpack(Dom3 d, double *fld, const double *blk, int ng)
{
    const int nx = ng ? d.NX : d.NX + 2 * NG, ny = ng ? d.NY : d.NY + 2 * NG, nz = ng ? d.NZ : d.NZ + 2 * NG;
    const int o = ng ? 0 : NG;
    const long long n = (long long)nx * ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((long long)nx * ny));
        fld[at(d, i - o, j - o, k - o)] = blk[t];
    }
}

// the reference's array after its ghost update, into the host block layout;
// xf: 0 the field, 1 C_G, 2 rho, 3 mu of C_L
template <int K>
__global__ void k3_pack(Dom3 d, Phase ph, const double *fld, double *blk, int ng, int xf)
{
    const int nx = ng ? d.NX : d.NX + 2 * NG, ny = ng ? d.NY : d.NY + 2 * NG, nz = ng ? d.NZ : d.NZ + 2 * NG;
    const int o = ng ? 0 : NG;
    const long long n = (long long)nx * ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx) - o, j = (int)((t / nx) % ny) - o, k = (int)(t / ((long long)nx * ny)) - o;
        double v = ng ? fld[at(d, i, j, k)] : rd<K>(d, fld, i, j, k);
        if (xf == 1) v = ph.cg(v);
        else if (xf == 2) v = ph.rho(v);
        else if (xf == 3) v = ph.mu(v);
        // rho and mu are computed on the G range only: the positions their
        // ghost update leaves alone keep the zeros of the allocation
        if (xf >= 2 && !written<K>(d, i, j, k)) v = 0.0;
        blk[t] = v;
    }
}

__global__ void k3_flush(double *buf, size_t n, double v)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) buf[t] = v;
}

struct GpuExec {
    cudaStream_t stream = nullptr;
    Sc3 *sc = nullptr;         // device scalars
    Sc3 *sc_host = nullptr;    // pinned mirror
    int *int_host = nullptr;   // pinned word
    double *part = nullptr;    // NSLOT x pstride partial sums
    size_t pstride = 0;        // doubles per slot: 4 per block of the largest reduction grid
    Pend pend{};
    long long launches = 0;
    cudaError_t err = cudaSuccess;
    size_t field_elems = 0;    // doubles per padded field
    long long origin = 0;      // offset of element (0,0,0) in a field
    // per-solver device time (pvof_set_solver_timing): events around each solve
    int timing = 0;
    cudaEvent_t tev[2] = {nullptr, nullptr};
    double sol_ms[3] = {0.0, 0.0, 0.0};

    void tic()
    {
        if (timing) cudaEventRecord(tev[0], stream);
    }
    void toc(int solver)
    {
        if (!timing) return;
        float t = 0.f;
        if (cudaEventRecord(tev[1], stream) == cudaSuccess && cudaEventSynchronize(tev[1]) == cudaSuccess &&
            cudaEventElapsedTime(&t, tev[0], tev[1]) == cudaSuccess)
            sol_ms[solver] += t;
    }

    void note()
    {
        launches++;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess && err == cudaSuccess) err = e;
    }
    static int blocks(const Range &r, int cap)
    {
        const long long nrows = (long long)(r.j1 - r.j0) * (r.k1 - r.k0);
        long long b = (nrows + WPB - 1) / WPB;
        if (b < 1) b = 1;
        if (b > cap) b = cap;
        return (int)b;
    }
    static bool empty(const Range &r) { return r.i1 <= r.i0 || r.j1 <= r.j0 || r.k1 <= r.k0; }

    template <class F>
    void cells(const Range &r, const int *gate, F f)
    {
        if (empty(r)) return;
        k3_cells<<<blocks(r, NBC), TPB, 0, stream>>>(r, gate, f);
        note();
    }
    template <int N, bool MAX = false, class F>
    void reduce(const Range &r, const int *gate, int slot, F f)
    {
        const int nb = blocks(r, NBR);
        k3_reduce<N, MAX><<<nb, TPB, 0, stream>>>(r, gate, part + (size_t)slot * pstride, f);
        note();
        pend.nb[slot] = empty(r) ? 0 : nb;
        pend.nq[slot] = N;
        pend.mx[slot] = MAX ? 1 : 0;
        pend.mask |= 1u << slot;
    }
    template <class F>
    void scalar(const int *gate, F f)
    {
        pend.stride = pstride;
        k3_scalar<<<1, TPB, 0, stream>>>(part, pend, gate, sc, f);
        note();
        pend.mask = 0;
    }
    // the pressure PCG iteration's three passes (k3p_*)
    static dim3 pgrid(const Dom3 &d)
    {
        return dim3((unsigned)((d.NX - 1 + 63) / 64), (unsigned)((d.NY - 1 + 7) / 8), (unsigned)((d.NZ - 1 + PKB - 1) / PKB));
    }
    // the partials of these passes use the last slot, which the generic
    // reductions of the pressure loop do not touch
    template <class F>
    void p_apply(const Dom3 &d, const double *CX, const double *CY, const double *CZ, const double *X, double *AD,
                 const int *gate, F then)
    {
        k3p_apply<<<pgrid(d), dim3(32, 8), 0, stream>>>(d, CX, CY, CZ, X, AD, gate, part + (size_t)(NSLOT - 1) * pstride,
                                                        sc, then);
        note();
    }
    template <class F>
    void p_update(const Dom3 &d, double *PHI, double *R, const double *DD, const double *AD, const double *M,
                  const int *gate, F then)
    {
        k3p_update<<<pgrid(d), dim3(32, 8), 0, stream>>>(d, PHI, R, DD, AD, M, gate, sc,
                                                         part + (size_t)(NSLOT - 1) * pstride, then);
        note();
    }
    void p_dir(const Dom3 &d, const double *R, const double *M, double *DD, const int *gate)
    {
        k3p_dir<<<pgrid(d), dim3(32, 8), 0, stream>>>(d, R, M, DD, gate, sc);
        note();
    }
    // spectral preconditioner: spectrum, tridiagonal tables, launch shapes
    double2 *spec = nullptr;
    double *tri_cp = nullptr, *tri_im = nullptr;
    SpecDims sd{};
    double spec_scale = 0.0;
    double2 *tw_x = nullptr, *tw_z = nullptr;   // exp(-2 pi i q / n), q < n/2
    // z = s (-L)^-1 (s r) over the physical cells (the k3s_* kernels), then
    // r.z and the scalar step then(sc, r.z) in the last block
    // x transforms: one pair of rows per nt_x threads, g_x pairs per block
    static long long spec_xblocks(const SpecDims &sd)
    {
        return (((long long)sd.K * sd.ny + 1) / 2 + sd.g_x - 1) / sd.g_x;
    }
    template <class F>
    void spec_apply(const Dom3 &d, const double *R, const double *M, double *Z, const int *gate, F then)
    {
        const size_t smx = (size_t)(sd.N / 2 + sd.g_x * sd.N) * sizeof(double2);
        const size_t smz = (size_t)(sd.K / 2 + sd.ch_z * sd.K) * sizeof(double2);
        const unsigned gx = (unsigned)spec_xblocks(sd);
        const unsigned gz = (unsigned)(sd.ny * ((sd.H + sd.ch_z - 1) / sd.ch_z));
        // one thread per system, a few thousand systems: blocks of 32 spread them over every SM
        const unsigned gt = (unsigned)(((long long)sd.K * sd.H + 31) / 32);
        k3s_fwd_x<<<gx, 256, smx, stream>>>(d, sd, R, M, spec, tw_x, gate);
        note();
        k3s_z<<<gz, 256, smz, stream>>>(sd, spec, tw_z, -1.0, gate);
        note();
        k3s_tri<<<gt, 32, 0, stream>>>(sd, spec, tri_cp, tri_im, spec_scale, gate);
        note();
        k3s_z<<<gz, 256, smz, stream>>>(sd, spec, tw_z, 1.0, gate);
        note();
        k3s_inv_x<<<gx, 256, smx, stream>>>(d, sd, spec, M, R, Z, tw_x, gate, part + (size_t)(NSLOT - 1) * pstride, sc,
                                             then);
        note();
    }
    void p_dir_z(const Dom3 &d, const double *Z, double *DD, const int *gate)
    {
        k3p_dir_z<<<pgrid(d), dim3(32, 8), 0, stream>>>(d, Z, DD, gate, sc);
        note();
    }
    int read_int(const int *p)
    {
        if (cudaMemcpyAsync(int_host, p, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            if (err == cudaSuccess) err = cudaGetLastError();
            return 0;
        }
        return *int_host;
    }
    double read_double(const double *p)
    {
        Sc3 s = read_scalars();
        const char *base = reinterpret_cast<const char *>(sc);
        return *reinterpret_cast<const double *>(reinterpret_cast<const char *>(&s) + (reinterpret_cast<const char *>(p) - base));
    }
    Sc3 read_scalars()
    {
        if (cudaMemcpyAsync(sc_host, sc, sizeof(Sc3), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            if (err == cudaSuccess) err = cudaGetLastError();
        }
        return *sc_host;
    }
    void zero(double *fld)
    {
        const cudaError_t e = cudaMemsetAsync(fld - origin, 0, field_elems * sizeof(double), stream);
        if (e != cudaSuccess && err == cudaSuccess) err = e;
    }
    int status()
    {
        if (err != cudaSuccess) return fail(PVOF_ECUDA, std::string("CUDA: ") + cudaGetErrorString(err));
        return PVOF_OK;
    }
};

struct Handle {
    Box3<GpuExec> b;
    int device = 0;
    double *mem = nullptr;      // all fields
    double *tables = nullptr;   // metrics, weights, maps (doubles)
    int *itables = nullptr;     // map sources
    double *stage = nullptr;    // staging block for host copies
    size_t stage_elems = 0;
    double *flush = nullptr;
    size_t flush_elems = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

static size_t block_elems(const Dom3 &d, bool ng)
{
    return ng ? (size_t)d.NX * d.NY * d.NZ : (size_t)(d.NX + 2 * NG) * (d.NY + 2 * NG) * (d.NZ + 2 * NG);
}

#define CK3(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(PVOF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int destroy(Handle *h)
{
    if (!h) return PVOF_OK;
    cudaSetDevice(h->device);
    GpuExec &x = h->b.x;
    if (x.stream) cudaStreamSynchronize(x.stream);
    cudaFree(h->mem);
    cudaFree(h->tables);
    cudaFree(h->itables);
    cudaFree(h->stage);
    cudaFree(h->flush);
    cudaFree(x.sc);
    cudaFree(x.part);
    cudaFree(x.spec);
    cudaFree(x.tri_cp);
    cudaFree(x.tri_im);
    cudaFree(x.tw_x);
    cudaFree(x.tw_z);
    cudaFreeHost(x.sc_host);
    cudaFreeHost(x.int_host);
    for (int q = 0; q < 2; q++) {
        if (h->ev[q]) cudaEventDestroy(h->ev[q]);
        if (x.tev[q]) cudaEventDestroy(x.tev[q]);
    }
    if (x.stream) cudaStreamDestroy(x.stream);
    delete h;
    return PVOF_OK;
}

// the spectral preconditioner's launch shapes, tables and spectrum (host
// tables in FP64 from the same modified wave numbers as the operator)
static int spec_setup(GpuExec &x, const Dom3 &d, const pvof_grid_desc *g)
{
    SpecDims &sd = x.sd;
    sd.N = d.NX - 1;
    sd.K = d.NZ - 1;
    sd.ny = d.NY - 1;
    sd.H = sd.N / 2 + 1;
    sd.logN = 0;
    while ((1 << sd.logN) < sd.N) sd.logN++;
    sd.logK = 0;
    while ((1 << sd.logK) < sd.K) sd.logK++;
    sd.nt_x = std::min(256, sd.N / 2);
    sd.g_x = 256 / sd.nt_x;
    int ch = (int)((48 * 1024 / sizeof(double2) - sd.K / 2) / sd.K);
    sd.ch_z = 1;
    while (sd.ch_z * 2 <= std::min(ch, 16)) sd.ch_z *= 2;
    sd.nt_z = 256 / sd.ch_z;
    const double idy2 = d.idy2;
    x.spec_scale = (1.0 / idy2) / ((double)sd.N * (double)sd.K);
    const size_t n = (size_t)sd.K * sd.ny * sd.H;
    std::vector<double> cp(n), im(n);
    const double pi = 3.14159265358979323846;
    for (int kz = 0; kz < sd.K; kz++)
        for (int kx = 0; kx < sd.H; kx++) {
            const double lam = (d.idx2 * (2.0 - 2.0 * std::cos(2.0 * pi * kx / sd.N)) +
                                d.idz2 * (2.0 - 2.0 * std::cos(2.0 * pi * kz / sd.K))) / idy2;
            double cprev = 0.0;
            for (int j = 0; j < sd.ny; j++) {
                const double b = ((j == 0 || j == sd.ny - 1) ? 1.0 : 2.0) + lam;
                const double m = b + cprev;
                const size_t q = ((size_t)kz * sd.ny + j) * sd.H + kx;
                im[q] = 1.0 / m;
                cp[q] = -1.0 / m;
                cprev = cp[q];
            }
        }
    (void)g;
    std::vector<double2> twx((size_t)sd.N / 2), twz((size_t)sd.K / 2);
    for (int q = 0; q < sd.N / 2; q++) twx[q] = make_double2(std::cos(2.0 * pi * q / sd.N), -std::sin(2.0 * pi * q / sd.N));
    for (int q = 0; q < sd.K / 2; q++) twz[q] = make_double2(std::cos(2.0 * pi * q / sd.K), -std::sin(2.0 * pi * q / sd.K));
    if (cudaMalloc(&x.tw_x, twx.size() * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&x.tw_z, twz.size() * sizeof(double2)) != cudaSuccess ||
        cudaMemcpy(x.tw_x, twx.data(), twx.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(x.tw_z, twz.data(), twz.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(PVOF_ENOMEM, "twiddle tables");
    if (cudaMalloc(&x.spec, n * sizeof(double2)) != cudaSuccess || cudaMalloc(&x.tri_cp, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&x.tri_im, n * sizeof(double)) != cudaSuccess)
        return fail(PVOF_ENOMEM, "device memory for the spectral preconditioner");
    if (cudaMemcpy(x.tri_cp, cp.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(x.tri_im, im.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(PVOF_ECUDA, "spectral tables upload");
    return PVOF_OK;
}

int create(const pvof_grid_desc *g, const pvof_params *p, int device, Handle **out)
{
    *out = nullptr;
    if (!g->periodic[0] || g->periodic[1] || !g->periodic[2])
        return fail(PVOF_EINVAL, "the 3D mode needs x and z periodic and walls in y");
    if (g->NXM < 8 || g->NYM < 8 || g->NZM < 8) return fail(PVOF_EINVAL, "the 3D mode needs at least 8 cells per direction");
    if (p->pressure_warm_start) return fail(PVOF_EINVAL, "the pressure warm starts are 2D only");
    if (p->pressure_preconditioner < 0 || p->pressure_preconditioner > 1)
        return fail(PVOF_EINVAL, "pressure_preconditioner must be 0 (Jacobi) or 1 (spectral)");
    if (p->pressure_preconditioner) {
        auto pow2 = [](int n) { return n >= 2 && n <= 1024 && (n & (n - 1)) == 0; };
        if (!pow2(g->NXM) || !pow2(g->NZM) || g->NYM > 4096)
            return fail(PVOF_EINVAL, "the 3D spectral preconditioner needs power-of-two x and z cell counts up to 1024");
    }
    if (p->stencil_fp32 < 0 || p->stencil_fp32 > 1) return fail(PVOF_EINVAL, "stencil_fp32 must be 0 or 1");
    const double hx = (g->xmax - g->xmin) / g->NXM, hy = (g->ymax - g->ymin) / g->NYM, hz = (g->zmax - g->zmin) / g->NZM;
    if (!(hx > 0 && hy > 0 && hz > 0)) return fail(PVOF_EINVAL, "empty box");
    CK3(cudaSetDevice(device));
    Handle *h = new Handle();
    h->device = device;
    Box3<GpuExec> &b = h->b;
    b.g = *g;
    b.p = *p;
    b.ph.rho_g = p->rho2 / p->rho1;
    b.ph.mu_g = p->mu2 / p->mu1;
    Dom3 &d = b.d;
    d.NX = g->NXM + 1;
    d.NY = g->NYM + 1;
    d.NZ = g->NZM + 1;
    d.P = ((OX + d.NX + NG) + 7) / 8 * 8;
    d.S = (long long)d.P * (d.NY + 2 * NG);
    GpuExec &x = b.x;
    x.field_elems = (size_t)d.S * (size_t)(d.NZ + 2 * NG);
    x.origin = (long long)NG * d.S + (long long)NG * d.P + OX;
    auto bail = [&](int rc) { destroy(h); return rc; };
    if (cudaStreamCreateWithFlags(&x.stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(PVOF_ECUDA, "stream"));
    // fields (zeroed once: never-written positions read as the reference's zero-initialised arrays)
    const int nfields = F3_COUNT + 2;
    if (cudaMalloc(&h->mem, x.field_elems * sizeof(double) * nfields) != cudaSuccess)
        return bail(fail(PVOF_ENOMEM, "device memory for the 3D fields"));
    if (cudaMemsetAsync(h->mem, 0, x.field_elems * sizeof(double) * nfields, x.stream) != cudaSuccess)
        return bail(fail(PVOF_ECUDA, "memset"));
    for (int q = 0; q < F3_COUNT; q++) b.f[q] = h->mem + (size_t)q * x.field_elems + x.origin;
    b.vd[0] = b.f[F3_VD];
    b.vd[1] = h->mem + (size_t)F3_COUNT * x.field_elems + x.origin;
    b.vd[2] = h->mem + (size_t)(F3_COUNT + 1) * x.field_elems + x.origin;
    // tables: metrics per axis (8 arrays), weights, map multipliers; map sources
    HostAxis ax[3];
    const bool per[3] = {true, false, true};
    const double lo[3] = {g->xmin, g->ymin, g->zmin}, hi[3] = {g->xmax, g->ymax, g->zmax};
    const int N[3] = {d.NX, d.NY, d.NZ};
    for (int a = 0; a < 3; a++) {
        host_axis_metrics(ax[a], N[a], lo[a], hi[a], per[a]);
        host_axis_maps(ax[a], N[a], per[a], false, false, false, a, g->wall[PVOF_BOTTOM], g->wall[PVOF_TOP]);
    }
    std::vector<double> dt_;
    std::vector<int> it_;
    std::vector<size_t> doff, ioff;
    auto addd = [&](const std::vector<double> &v) { doff.push_back(dt_.size()); dt_.insert(dt_.end(), v.begin(), v.end()); };
    auto addi = [&](const std::vector<int> &v) { ioff.push_back(it_.size()); it_.insert(it_.end(), v.begin(), v.end()); };
    for (int a = 0; a < 3; a++) {
        addd(ax[a].idf); addd(ax[a].idc); addd(ax[a].df); addd(ax[a].dc); addd(ax[a].w);
        for (int kind = 0; kind < K_COUNT; kind++) {
            addd(ax[a].mul[kind]);
            addi(ax[a].src[kind]);
        }
    }
    if (cudaMalloc(&h->tables, dt_.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->itables, it_.size() * sizeof(int)) != cudaSuccess)
        return bail(fail(PVOF_ENOMEM, "device memory for the tables"));
    if (cudaMemcpy(h->tables, dt_.data(), dt_.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->itables, it_.data(), it_.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(PVOF_ECUDA, "table upload"));
    size_t qd = 0, qi = 0;
    for (int a = 0; a < 3; a++) {
        const double *idf = h->tables + doff[qd++] + NG, *idc = h->tables + doff[qd++] + NG;
        const double *df = h->tables + doff[qd++] + NG, *dc = h->tables + doff[qd++] + NG;
        const double *w = h->tables + doff[qd++] + NG;
        if (a == 0) { d.idx_u = idf; d.idx_c = idc; d.dx_u = df; d.dx_c = dc; d.wx = w; }
        if (a == 1) { d.idy_v = idf; d.idy_c = idc; d.dy_v = df; d.dy_c = dc; d.wy = w; }
        if (a == 2) { d.idz_w = idf; d.idz_c = idc; d.dz_w = df; d.dz_c = dc; d.wz = w; }
        for (int kind = 0; kind < K_COUNT; kind++) {
            Axis A{h->itables + ioff[qi++], h->tables + doff[qd++]};
            if (a == 0) d.map[kind].x = A;
            if (a == 1) d.map[kind].y = A;
            if (a == 2) d.map[kind].z = A;
        }
    }
    d.idx2 = ax[0].idc[1 + NG] * ax[0].idc[1 + NG];
    d.idy2 = ax[1].idc[1 + NG] * ax[1].idc[1 + NG];
    d.idz2 = ax[2].idc[1 + NG] * ax[2].idc[1 + NG];
    d.idx_u1 = ax[0].idf[1 + NG];
    if (p->pressure_preconditioner && spec_setup(x, d, g) < 0) return bail(PVOF_ENOMEM);
    {
        // one partial sum per block of the largest reduction grid: the
        // generic sums, the pressure passes and the spectral inverse-x pass
        const dim3 pg = GpuExec::pgrid(d);
        size_t nb = std::max((size_t)NBR, (size_t)pg.x * pg.y * pg.z);
        if (p->pressure_preconditioner) nb = std::max(nb, (size_t)GpuExec::spec_xblocks(x.sd));
        x.pstride = 4 * nb;
    }
    if (cudaMalloc(&x.sc, sizeof(Sc3)) != cudaSuccess || cudaMalloc(&x.part, sizeof(double) * NSLOT * x.pstride) != cudaSuccess)
        return bail(fail(PVOF_ENOMEM, "device scalars"));
    cudaMemsetAsync(x.sc, 0, sizeof(Sc3), x.stream);
    cudaMemsetAsync(x.part, 0, sizeof(double) * NSLOT * x.pstride, x.stream);
    if (cudaMallocHost(&x.sc_host, sizeof(Sc3)) != cudaSuccess || cudaMallocHost(&x.int_host, sizeof(int)) != cudaSuccess)
        return bail(fail(PVOF_ENOMEM, "pinned scalars"));
    h->stage_elems = block_elems(d, false);
    if (cudaMalloc(&h->stage, h->stage_elems * sizeof(double)) != cudaSuccess)
        return bail(fail(PVOF_ENOMEM, "staging block"));
    for (int q = 0; q < 2; q++)
        if (cudaEventCreate(&h->ev[q]) != cudaSuccess || cudaEventCreate(&x.tev[q]) != cudaSuccess)
            return bail(fail(PVOF_ECUDA, "event"));
    if (cudaStreamSynchronize(x.stream) != cudaSuccess) return bail(fail(PVOF_ECUDA, "set-up"));
    *out = h;
    return PVOF_OK;
}

// field of the ABI -> (slot, ghost kind, no-ghost, derived quantity)
struct FieldRef {
    int slot, kind, ng, xf;
};
static bool field_ref(const Handle *h, int field, bool upload, FieldRef &r)
{
    r = FieldRef{-1, K_SCALAR, 0, 0};
    switch (field) {
    case PVOF_F_C_L: r.slot = F3_CL; break;
    case PVOF_F_F: r.slot = (upload || !h->b.initialized) ? F3_F : F3_CL; break;
    case PVOF_F_C_G: if (upload) return false; r.slot = F3_CL; r.xf = 1; break;
    case PVOF_F_RHO: if (upload) return false; r.slot = F3_CL; r.xf = 2; break;
    case PVOF_F_MU: if (upload) return false; r.slot = F3_CL; r.xf = 3; break;
    case PVOF_F_PSI_LG: r.slot = F3_PSI; break;
    case PVOF_F_CH_RHS_N:
    case PVOF_F_CH_RHS_CUR: r.slot = F3_RN; break;
    case PVOF_F_U: r.slot = F3_U; r.kind = K_U; break;
    case PVOF_F_V: r.slot = F3_V; r.kind = K_V; break;
    case PVOF_F_W: r.slot = F3_W; r.kind = K_W; break;
    case PVOF_F_P: r.slot = F3_P; r.kind = K_PRESSURE; break;
    case PVOF_F_DELTAP: r.slot = F3_DP; r.kind = K_PRESSURE; break;
    case PVOF_F_P_RHS: r.slot = F3_PRHS; r.kind = K_WRAP_C; break;
    case PVOF_F_U_EXPLICIT: case PVOF_F_U_EXPLICIT_OLD: r.slot = F3_U_EXO; r.ng = 1; break;
    case PVOF_F_V_EXPLICIT: case PVOF_F_V_EXPLICIT_OLD: r.slot = F3_V_EXO; r.ng = 1; break;
    case PVOF_F_W_EXPLICIT: case PVOF_F_W_EXPLICIT_OLD: r.slot = F3_W_EXO; r.ng = 1; break;
    case PVOF_F_U_VISC_EXPLICIT: case PVOF_F_U_VISC_EXPLICIT_OLD: r.slot = F3_U_VXO; r.ng = 1; break;
    case PVOF_F_V_VISC_EXPLICIT: case PVOF_F_V_VISC_EXPLICIT_OLD: r.slot = F3_V_VXO; r.ng = 1; break;
    case PVOF_F_W_VISC_EXPLICIT: case PVOF_F_W_VISC_EXPLICIT_OLD: r.slot = F3_W_VXO; r.ng = 1; break;
    case PVOF_F_U_RHS: r.slot = F3_U_RHS; r.ng = 1; break;
    case PVOF_F_V_RHS: r.slot = F3_V_RHS; r.ng = 1; break;
    case PVOF_F_W_RHS: r.slot = F3_W_RHS; r.ng = 1; break;
    case PVOF_F_FSIG_OLD_X: r.slot = F3_FSO_X; r.ng = 1; break;
    case PVOF_F_FSIG_OLD_Y: r.slot = F3_FSO_Y; r.ng = 1; break;
    case PVOF_F_FSIG_OLD_Z: r.slot = F3_FSO_Z; r.ng = 1; break;
    case PVOF_F_FSIG_NEW_X: r.slot = F3_FSN_X; r.ng = 1; break;
    case PVOF_F_FSIG_NEW_Y: r.slot = F3_FSN_Y; r.ng = 1; break;
    case PVOF_F_FSIG_NEW_Z: r.slot = F3_FSN_Z; r.ng = 1; break;
    default: return false;
    }
    return true;
}

static bool is_ng_field(int field)
{
    return (field >= PVOF_F_U_EXPLICIT && field <= PVOF_F_FSIG_NEW_Y) || (field >= PVOF_F_W_EXPLICIT && field <= PVOF_F_FSIG_NEW_Z);
}

size_t block_count(const Handle *h, int field)
{
    if (field < 0 || field >= PVOF_F_COUNT) return 0;
    return block_elems(h->b.d, is_ng_field(field));
}

int upload(Handle *h, int field, const double *host, size_t count)
{
    FieldRef r;
    if (!field_ref(h, field, true, r)) return fail(PVOF_EINVAL, "this field cannot be uploaded in the 3D mode");
    const size_t n = block_elems(h->b.d, r.ng);
    if (count != n) return fail(PVOF_EINVAL, "block size mismatch");
    CK3(cudaSetDevice(h->device));
    GpuExec &x = h->b.x;
    CK3(cudaMemcpyAsync(h->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, x.stream));
    k3_unpack<<<592, 256, 0, x.stream>>>(h->b.d, h->b.f[r.slot], h->stage, r.ng);
    x.note();
    CK3(cudaStreamSynchronize(x.stream));
    return x.status();
}

int download(Handle *h, int field, double *host, size_t count)
{
    FieldRef r;
    if (!field_ref(h, field, false, r)) return fail(PVOF_EINVAL, "this field is not kept in the 3D mode");
    const size_t n = block_elems(h->b.d, r.ng);
    if (count != n) return fail(PVOF_EINVAL, "block size mismatch");
    CK3(cudaSetDevice(h->device));
    GpuExec &x = h->b.x;
    const Dom3 &d = h->b.d;
    const double *fld = h->b.f[r.slot];
    switch (r.kind) {
    case K_U: k3_pack<K_U><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    case K_V: k3_pack<K_V><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    case K_W: k3_pack<K_W><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    case K_PRESSURE: k3_pack<K_PRESSURE><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    case K_WRAP_C: k3_pack<K_WRAP_C><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    default: k3_pack<K_SCALAR><<<592, 256, 0, x.stream>>>(d, h->b.ph, fld, h->stage, r.ng, r.xf); break;
    }
    x.note();
    CK3(cudaMemcpyAsync(host, h->stage, n * sizeof(double), cudaMemcpyDeviceToHost, x.stream));
    CK3(cudaStreamSynchronize(x.stream));
    return x.status();
}

int synchronize(Handle *h)
{
    CK3(cudaSetDevice(h->device));
    CK3(cudaStreamSynchronize(h->b.x.stream));
    return h->b.x.status();
}

int set_stage(Handle *h, int stage, double dt)
{
    if (stage < 0 || stage > 2 || !(dt > 0.0)) return fail(PVOF_EINVAL, "stage must be 0..2 and dt positive");
    h->b.stage = stage;
    h->b.dt = dt;
    return PVOF_OK;
}

int initialize(Handle *h)
{
    CK3(cudaSetDevice(h->device));
    const int rc = h->b.initialize();
    if (rc < 0) return rc;
    CK3(cudaStreamSynchronize(h->b.x.stream));
    return h->b.x.status();
}

int substep(Handle *h, pvof_stats *st)
{
    CK3(cudaSetDevice(h->device));
    if (!h->b.initialized) return fail(PVOF_EINVAL, "pvof_initialize() first");
    if (!(h->b.dt > 0.0)) return fail(PVOF_EINVAL, "pvof_set_stage() first");
    const int rc = h->b.substep(st);
    if (rc == PVOF_EDIVERGED) return fail(rc, "the outer Poisson loop did not reach div < 1e-6 in 10 passes");
    return rc;
}

int run_steps(Handle *h, int nsteps, double dt, pvof_stats *st)
{
    CK3(cudaSetDevice(h->device));
    if (!h->b.initialized) return fail(PVOF_EINVAL, "pvof_initialize() first");
    if (nsteps < 0 || !(dt > 0.0)) return fail(PVOF_EINVAL, "nsteps >= 0 and dt > 0");
    const int rc = h->b.run_steps(nsteps, dt, st);
    if (rc == PVOF_EDIVERGED) return fail(rc, "the outer Poisson loop did not reach div < 1e-6 in 10 passes");
    return rc;
}

int liquid_mass(Handle *h, double *m)
{
    CK3(cudaSetDevice(h->device));
    return h->b.liquid_mass(m);
}

long long launch_count(const Handle *h) { return h->b.x.launches; }

int set_solver_timing(Handle *h, int on)
{
    h->b.x.timing = on ? 1 : 0;
    for (int k = 0; k < 3; k++) {
        h->b.x.sol_ms[k] = 0.0;
        h->b.sol_launches[k] = h->b.sol_iters[k] = h->b.sol_cell_iters[k] = 0;
    }
    return PVOF_OK;
}

int solver_timing(const Handle *h, int solver, double *ms, long long *launches, long long *iters, long long *cell_iters)
{
    if (solver < 0 || solver > 2) return fail(PVOF_EINVAL, "bad solver index");
    if (ms) *ms = h->b.x.sol_ms[solver];
    if (launches) *launches = h->b.sol_launches[solver];
    if (iters) *iters = h->b.sol_iters[solver];
    if (cell_iters) *cell_iters = h->b.sol_cell_iters[solver];
    return PVOF_OK;
}
double clamp_total(const Handle *h) { return h->b.clamp_total; }

int timer_start(Handle *h)
{
    CK3(cudaSetDevice(h->device));
    CK3(cudaEventRecord(h->ev[0], h->b.x.stream));
    return PVOF_OK;
}

int timer_stop(Handle *h, double *ms)
{
    CK3(cudaSetDevice(h->device));
    CK3(cudaEventRecord(h->ev[1], h->b.x.stream));
    CK3(cudaEventSynchronize(h->ev[1]));
    float t = 0.f;
    CK3(cudaEventElapsedTime(&t, h->ev[0], h->ev[1]));
    *ms = t;
    return h->b.x.status();
}

// writes a buffer twice the size of the L2 so the next launch starts cold
int flush_l2(Handle *h)
{
    CK3(cudaSetDevice(h->device));
    if (!h->flush) {
        int l2 = 0;
        CK3(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->device));
        h->flush_elems = (size_t)2 * (size_t)l2 / sizeof(double);
        CK3(cudaMalloc(&h->flush, h->flush_elems * sizeof(double)));
    }
    k3_flush<<<592, 256, 0, h->b.x.stream>>>(h->flush, h->flush_elems, 0.0);
    CK3(cudaGetLastError());
    return PVOF_OK;
}

}  // namespace pvof3
