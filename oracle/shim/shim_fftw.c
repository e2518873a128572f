/*
 * FFTW3 API subset for the CPU oracle build (TEST INFRASTRUCTURE ONLY).
 *
 * A plain textbook Cooley-Tukey radix-2 decimation-in-time transform for
 * power-of-two lengths and a direct O(n^2) DFT otherwise. Twiddle factors are
 * evaluated directly with cos/sin (no recurrences) so the transform error stays
 * at the level of a few ulps times log2(n), comparable to FFTW.
 *
 * Sign convention (FFTW manual, "What FFTW Really Computes"):
 *   FFTW_FORWARD  (-1): Y[k] = sum_j X[j] exp(-2 pi i jk/n)
 *   FFTW_BACKWARD (+1): Y[k] = sum_j X[j] exp(+2 pi i jk/n)
 * Multi-dimensional transforms are row-major products of 1D transforms; no
 * normalisation is applied.
 */
#include "fftw3.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct ipg_fftw_plan_s {
    int n0, n1;      /* 2D extents (n0 slow, n1 fast) */
    int howmany;     /* batch count */
    int idist, odist;
    fftw_complex *in, *out;
    int sign;
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
void fftw_cleanup_threads(void) {}

static fftw_plan make_plan(int n0, int n1, int howmany, fftw_complex *in,
                           int idist, fftw_complex *out, int odist, int sign) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n0 = n0;
    p->n1 = n1;
    p->howmany = howmany;
    p->in = in;
    p->out = out;
    p->idist = idist;
    p->odist = odist;
    p->sign = sign;
    return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(n0, n1, 1, in, n0 * n1, out, n0 * n1, sign);
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride,
                             int idist, fftw_complex *out, const int *onembed,
                             int ostride, int odist, int sign, unsigned flags) {
    (void)inembed;
    (void)onembed;
    (void)flags;
    if (rank != 2 || istride != 1 || ostride != 1) {
        fprintf(stderr, "shim fftw: only rank-2 unit-stride plans supported\n");
        abort();
    }
    return make_plan(n[0], n[1], howmany, in, idist, out, odist, sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place 1D transform of n complex values spaced by `stride` (in units of
 * complex elements) in `x`, using `tmp` (n complex) as scratch. */
static void fft1d(double *x, int n, int stride, int sign, double *tmp) {
    int i, k;
    for (i = 0; i < n; i++) {
        tmp[2 * i] = x[2 * (size_t)i * stride];
        tmp[2 * i + 1] = x[2 * (size_t)i * stride + 1];
    }
    if (is_pow2(n)) {
        int bits = 0, j, len;
        while ((1 << bits) < n) bits++;
        /* bit-reversal permutation */
        for (i = 0; i < n; i++) {
            int r = 0;
            for (j = 0; j < bits; j++) r |= ((i >> j) & 1) << (bits - 1 - j);
            if (r > i) {
                double t0 = tmp[2 * i], t1 = tmp[2 * i + 1];
                tmp[2 * i] = tmp[2 * r];
                tmp[2 * i + 1] = tmp[2 * r + 1];
                tmp[2 * r] = t0;
                tmp[2 * r + 1] = t1;
            }
        }
        for (len = 2; len <= n; len <<= 1) {
            int half = len >> 1;
            for (k = 0; k < half; k++) {
                double ang = 2.0 * M_PI * (double)k / (double)len;
                double wr = cos(ang), wi = sign * sin(ang);
                for (i = k; i < n; i += len) {
                    double ar = tmp[2 * i], ai = tmp[2 * i + 1];
                    double br = tmp[2 * (i + half)], bi = tmp[2 * (i + half) + 1];
                    double tr = br * wr - bi * wi;
                    double ti = br * wi + bi * wr;
                    tmp[2 * i] = ar + tr;
                    tmp[2 * i + 1] = ai + ti;
                    tmp[2 * (i + half)] = ar - tr;
                    tmp[2 * (i + half) + 1] = ai - ti;
                }
            }
        }
        for (i = 0; i < n; i++) {
            x[2 * (size_t)i * stride] = tmp[2 * i];
            x[2 * (size_t)i * stride + 1] = tmp[2 * i + 1];
        }
    } else {
        for (k = 0; k < n; k++) {
            double sr = 0.0, si = 0.0;
            for (i = 0; i < n; i++) {
                long m = ((long)i * (long)k) % n;
                double ang = 2.0 * M_PI * (double)m / (double)n;
                double wr = cos(ang), wi = sign * sin(ang);
                sr += tmp[2 * i] * wr - tmp[2 * i + 1] * wi;
                si += tmp[2 * i] * wi + tmp[2 * i + 1] * wr;
            }
            x[2 * (size_t)k * stride] = sr;
            x[2 * (size_t)k * stride + 1] = si;
        }
    }
}

void fftw_execute(const fftw_plan p) {
    int b, r, c;
    int n0 = p->n0, n1 = p->n1;
    size_t ntot = (size_t)n0 * n1;
    int nmax = n0 > n1 ? n0 : n1;
    double *tmp = (double *)malloc(sizeof(double) * 2 * nmax);
    /* FFTW_FORWARD = -1 means exp(-i...), i.e. the sine term carries sign -1 */
    int sgn = p->sign;
    for (b = 0; b < p->howmany; b++) {
        double *src = (double *)(p->in + (size_t)b * p->idist);
        double *dst = (double *)(p->out + (size_t)b * p->odist);
        if (dst != src) memmove(dst, src, sizeof(fftw_complex) * ntot);
        for (r = 0; r < n0; r++) fft1d(dst + 2 * (size_t)r * n1, n1, 1, sgn, tmp);
        for (c = 0; c < n1; c++) fft1d(dst + 2 * (size_t)c, n0, n1, sgn, tmp);
    }
    free(tmp);
}
