/*
 * Minimal FFTW3-compatible interface written for this project so that the
 * reference's C sources compile and link without FFTW.  Plans hold the
 * transform kind and length; execution is a direct O(N^2) evaluation of the
 * published FFTW transform definitions (R2HC, HC2R, REDFT10, REDFT01 and the
 * complex DFT).  Test infrastructure for the CPU oracle build only.
 */
#ifndef PVOF_SHIM_FFTW3_H
#define PVOF_SHIM_FFTW3_H

#include <stddef.h>

typedef double fftw_complex[2];
typedef struct pvof_fftw_plan_s *fftw_plan;
typedef int fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_R2HC 0
#define FFTW_HC2R 1
#define FFTW_REDFT10 5
#define FFTW_REDFT01 6
#define FFTW_MEASURE 0U
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_r2r(const fftw_plan p, double *in, double *out);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#endif
