/*
 * Minimal FFTW3 API subset, written for this project so that the reference
 * IP-Glasma sources can be compiled unmodified in a container without FFTW.
 *
 * TEST INFRASTRUCTURE ONLY: part of the CPU oracle build (oracle/_ref). The
 * shipped library never links this file.
 *
 * Only the symbols the reference uses are declared (FFT.h:64-97,
 * FFT.cpp:75-78,550-553). Conventions follow FFTW's documented definition:
 * FFTW_FORWARD computes Y[k] = sum_j X[j] exp(-2 pi i j k / n), FFTW_BACKWARD
 * uses exp(+2 pi i ...), neither is normalised, arrays are row-major.
 */
#ifndef IPG_SHIM_FFTW3_H
#define IPG_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct ipg_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride,
                             int idist, fftw_complex *out, const int *onembed,
                             int ostride, int odist, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif
