// Constant-density Poisson solver by Fourier transform in the periodic x
// direction and tridiagonal solves in the wall-normal y direction:
// Pressure_solve_xz_period (Eulerian/lsolver/psolve_fft.c:638-983) with its
// coefficients (Pressure_calc_coeff, :467-591) and the Thomas algorithm
// (tridiag, :141-163), for the planar 2D mode (one z plane: the z transform of
// the reference is the identity there).
//
//   1. every row j: real forward transform of length N = NX-1 in FFTW's
//      half-complex order (Re X_0 .. Re X_{N/2}, Im X_{(N+1)/2-1} .. Im X_1),
//      times 1/N;
//   2. every half-complex index i: tridiagonal solve along y of
//      (as, ap - 2 (1 - cos(2 pi wave(i) / N)) / dx^2, an), with the mean
//      mode pinned to zero at j = 0 (Neumann walls);
//   3. every row: unnormalised inverse transform.
//
// The transforms are radix-2 in shared memory for N a power of two (a direct
// transform for other N), one CTA per row; the Thomas solves run one thread
// per wavenumber down the columns, so a warp reads 32 consecutive doubles of
// a row per step.
#include <cmath>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

// Forward (sign = -1) or inverse (+1) complex transform of a[0..N) in shared
// memory, N a power of two, by the CTA: bit reversal, then log2(N) stages.
__device__ void fft_pow2(double2 *a, int N, int logN, double sign)
{
    for (int t = threadIdx.x; t < N; t += blockDim.x) {
        const int r = (int)(__brev((unsigned)t) >> (32 - logN));
        if (r > t) { double2 x = a[t]; a[t] = a[r]; a[r] = x; }
    }
    __syncthreads();
    for (int len = 2; len <= N; len <<= 1) {
        const int half = len >> 1;
        for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
            const int g = t / half, pos = t - g * half;
            const int i0 = g * len + pos, i1 = i0 + half;
            double s, c;
            sincospi(2.0 * pos / len, &s, &c);
            s *= sign;
            const double2 u = a[i0], v = a[i1];
            const double2 w = make_double2(v.x * c - v.y * s, v.x * s + v.y * c);
            a[i0] = make_double2(u.x + w.x, u.y + w.y);
            a[i1] = make_double2(u.x - w.x, u.y - w.y);
        }
        __syncthreads();
    }
}

// exp(sign 2 pi i k n / N) by reducing k n modulo N first
__device__ __forceinline__ void twiddle(long long kn, int N, double sign, double &c, double &s)
{
    const long long m = kn % N;
    sincospi(2.0 * (double)m / (double)N, &s, &c);
    s *= sign;
}

// step 1: hc[j][k] = half-complex forward transform of rhs[j][0..N) times inx
__global__ void k_fft_forward(Dom d, int N, int logN, const double *__restrict__ rhs, double *__restrict__ hc, double inx)
{
    extern __shared__ double2 sm[];
    const int j = blockIdx.x;
    const int P = d.P;
    if (logN >= 0) {
        for (int n = threadIdx.x; n < N; n += blockDim.x) sm[n] = make_double2(AT_(rhs, n, j), 0.0);
        __syncthreads();
        fft_pow2(sm, N, logN, -1.0);
        for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) AT_(hc, k, j) = sm[k].x * inx;
        for (int k = 1 + threadIdx.x; k < (N + 1) / 2; k += blockDim.x) AT_(hc, N - k, j) = sm[k].y * inx;
    } else {
        double *x = reinterpret_cast<double *>(sm);
        for (int n = threadIdx.x; n < N; n += blockDim.x) x[n] = AT_(rhs, n, j);
        __syncthreads();
        for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) {
            double re = 0.0, im = 0.0;
            for (int n = 0; n < N; n++) {
                double c, s;
                twiddle((long long)k * n, N, -1.0, c, s);
                re += x[n] * c;
                im += x[n] * s;
            }
            AT_(hc, k, j) = re * inx;
            if (k > 0 && k < (N + 1) / 2) AT_(hc, N - k, j) = im * inx;
        }
    }
}

// step 2: tridiag (psolve_fft.c:141-163) along y for every half-complex index
// i; as/ap/an per row, mw[i] the modified wavenumber; gam is scratch
__global__ void k_fft_tridiag(Dom d, int N, int NYp, const double *__restrict__ as_, const double *__restrict__ ap_,
                              const double *__restrict__ an_, const double *__restrict__ mw, double *__restrict__ hc,
                              double *__restrict__ gam)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int P = d.P;
    auto a = [&](int j) { return (i == 0 && j == 0) ? 0.0 : as_[j]; };
    auto c = [&](int j) { return (i == 0 && j == 0) ? 0.0 : an_[j]; };
    auto b = [&](int j) { return (i == 0 && j == 0) ? 1.0 : ap_[j] - 0.0 - mw[i]; };
    auto r = [&](int j) { return (i == 0 && j == 0) ? 0.0 : AT_(hc, i, j); };
    double bet = b(0);
    AT_(hc, i, 0) = r(0) / bet;
    for (int j = 1; j < NYp; j++) {
        const double g = c(j - 1) / bet;
        AT_(gam, i, j) = g;
        bet = b(j) - a(j) * g;
        AT_(hc, i, j) = (r(j) - a(j) * AT_(hc, i, j - 1)) / bet;
    }
    for (int j = NYp - 2; j >= 0; j--) AT_(hc, i, j) = AT_(hc, i, j) - AT_(gam, i, j + 1) * AT_(hc, i, j + 1);
}

// step 3: out[j][0..N) = unnormalised inverse transform of the half-complex row
__global__ void k_fft_inverse(Dom d, int N, int logN, const double *__restrict__ hc, double *__restrict__ out)
{
    extern __shared__ double2 sm[];
    const int j = blockIdx.x;
    const int P = d.P;
    auto X = [&](int k) {   // Hermitian spectrum from the half-complex row
        if (k == 0) return make_double2(AT_(hc, 0, j), 0.0);
        if (2 * k == N) return make_double2(AT_(hc, k, j), 0.0);
        if (k < (N + 1) / 2) return make_double2(AT_(hc, k, j), AT_(hc, N - k, j));
        return make_double2(AT_(hc, N - k, j), -AT_(hc, k, j));
    };
    if (logN >= 0) {
        for (int k = threadIdx.x; k < N; k += blockDim.x) sm[k] = X(k);
        __syncthreads();
        fft_pow2(sm, N, logN, 1.0);
        for (int n = threadIdx.x; n < N; n += blockDim.x) AT_(out, n, j) = sm[n].x;
    } else {
        for (int k = threadIdx.x; k < N; k += blockDim.x) sm[k] = X(k);
        __syncthreads();
        for (int n = threadIdx.x; n < N; n += blockDim.x) {
            double re = 0.0;
            for (int k = 0; k < N; k++) {
                double c, s;
                twiddle((long long)k * n, N, 1.0, c, s);
                re += sm[k].x * c - sm[k].y * s;
            }
            AT_(out, n, j) = re;
        }
    }
}

}  // namespace pvof
