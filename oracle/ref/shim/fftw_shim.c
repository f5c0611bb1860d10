/*
 * O(N^2) evaluation of the FFTW3 transform definitions used by the reference
 * (see fftw3.h).  Test infrastructure for the CPU oracle build only.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct pvof_fftw_plan_s {
    int n;
    int kind;      /* r2r kind, or 100 + sign for complex DFT */
    void *in, *out;
};

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->n = n; p->kind = kind; p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->n = n; p->kind = 100 + sign; p->in = in; p->out = out;
    return p;
}

static void r2r(int n, int kind, const double *x, double *y)
{
    const double pi = 3.14159265358979323846;
    double *t = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; k++) {
        double s = 0.0;
        if (kind == FFTW_R2HC) {
            /* y[k] = Re X_k for k <= n/2, y[n-k] = Im X_k for 0 < k < (n+1)/2 */
            int kk = (k <= n / 2) ? k : n - k;
            for (int j = 0; j < n; j++) {
                double a = 2.0 * pi * (double)j * (double)kk / (double)n;
                s += (k <= n / 2) ? x[j] * cos(a) : -x[j] * sin(a);
            }
        } else if (kind == FFTW_HC2R) {
            /* y[j] = sum_k X_k exp(+2 pi i j k / n), Hermitian X */
            int j = k;
            s = x[0];
            for (int q = 1; q < (n + 1) / 2; q++) {
                double a = 2.0 * pi * (double)j * (double)q / (double)n;
                s += 2.0 * (x[q] * cos(a) - x[n - q] * sin(a));
            }
            if (n % 2 == 0)
                s += x[n / 2] * ((j % 2) ? -1.0 : 1.0);
        } else if (kind == FFTW_REDFT10) {
            for (int j = 0; j < n; j++)
                s += 2.0 * x[j] * cos(pi * ((double)j + 0.5) * (double)k / (double)n);
        } else if (kind == FFTW_REDFT01) {
            s = x[0];
            for (int j = 1; j < n; j++)
                s += 2.0 * x[j] * cos(pi * (double)j * ((double)k + 0.5) / (double)n);
        } else {
            abort();
        }
        t[k] = s;
    }
    memcpy(y, t, sizeof(double) * (size_t)n);
    free(t);
}

static void dft(int n, int sign, const fftw_complex *x, fftw_complex *y)
{
    const double pi = 3.14159265358979323846;
    double *t = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < n; k++) {
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n; j++) {
            double a = (double)sign * 2.0 * pi * (double)j * (double)k / (double)n;
            re += x[j][0] * cos(a) - x[j][1] * sin(a);
            im += x[j][0] * sin(a) + x[j][1] * cos(a);
        }
        t[2 * k] = re;
        t[2 * k + 1] = im;
    }
    memcpy(y, t, sizeof(double) * 2 * (size_t)n);
    free(t);
}

void fftw_execute_r2r(const fftw_plan p, double *in, double *out) { r2r(p->n, p->kind, in, out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) { dft(p->n, p->kind - 100, in, out); }
void fftw_execute(const fftw_plan p)
{
    if (p->kind >= 99)
        dft(p->n, p->kind - 100, (const fftw_complex *)p->in, (fftw_complex *)p->out);
    else
        r2r(p->n, p->kind, (const double *)p->in, (double *)p->out);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
void fftw_cleanup(void) {}
