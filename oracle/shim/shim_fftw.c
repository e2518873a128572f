/*
 * FFTW3 API subset for the CPU oracle build (TEST INFRASTRUCTURE ONLY).
 *
 * A plain textbook Cooley-Tukey radix-2 decimation-in-time transform for
 * power-of-two lengths and a direct O(n^2) DFT otherwise. Twiddle factors are
 * evaluated directly with cos/sin (no recurrences) so the transform error stays
 * at the level of a few ulps times log2(n), comparable to FFTW.
 *
 * The power-of-two twiddles and the bit-reversal permutation are tabulated
 * once per plan: the stage-`len` twiddle of index k is the table entry
 * m = k n/len, whose angle (2 pi m)/n equals (2 pi k)/len to the bit (the
 * factors differ by a power of two), so the tables change the speed, not the
 * numbers. Columns are transformed in blocks of adjacent columns so that
 * each cache line of the matrix is fetched once per block.
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
    double *tw0, *tw1; /* power-of-two twiddles (cos, sign sin) of n0, n1 */
    int *rev0, *rev1;  /* bit-reversal permutations of n0, n1 */
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

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* twiddles w_m = exp(sign 2 pi i m/n), m < n/2, as (cos, sign sin) pairs, and
 * the bit-reversal permutation of n; NULL for other lengths */
static void make_tables(int n, int sign, double **tw, int **rev) {
    int m, i, j, bits = 0;
    *tw = NULL;
    *rev = NULL;
    if (!is_pow2(n)) return;
    while ((1 << bits) < n) bits++;
    *tw = (double *)malloc(sizeof(double) * (n > 1 ? n : 2));
    *rev = (int *)malloc(sizeof(int) * n);
    for (m = 0; m < n / 2; m++) {
        double ang = 2.0 * M_PI * (double)m / (double)n;
        (*tw)[2 * m] = cos(ang);
        (*tw)[2 * m + 1] = sign * sin(ang);
    }
    for (i = 0; i < n; i++) {
        int r = 0;
        for (j = 0; j < bits; j++) r |= ((i >> j) & 1) << (bits - 1 - j);
        (*rev)[i] = r;
    }
}

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
    make_tables(n0, sign, &p->tw0, &p->rev0);
    make_tables(n1, sign, &p->tw1, &p->rev1);
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

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->tw0);
    free(p->tw1);
    free(p->rev0);
    free(p->rev1);
    free(p);
}

/* In-place radix-2 transform of the n contiguous complex values in tmp, with
 * the plan's tables for n. */
static void fft_pow2(double *tmp, int n, const double *tw, const int *rev) {
    int i, k, len;
    for (i = 0; i < n; i++) {
        int r = rev[i];
        if (r > i) {
            double t0 = tmp[2 * i], t1 = tmp[2 * i + 1];
            tmp[2 * i] = tmp[2 * r];
            tmp[2 * i + 1] = tmp[2 * r + 1];
            tmp[2 * r] = t0;
            tmp[2 * r + 1] = t1;
        }
    }
    for (len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (i = 0; i < n; i += len) {
            double *a = tmp + 2 * i, *b = tmp + 2 * (i + half);
            for (k = 0; k < half; k++) {
                double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
                double ar = a[2 * k], ai = a[2 * k + 1];
                double br = b[2 * k], bi = b[2 * k + 1];
                double tr = br * wr - bi * wi;
                double ti = br * wi + bi * wr;
                a[2 * k] = ar + tr;
                a[2 * k + 1] = ai + ti;
                b[2 * k] = ar - tr;
                b[2 * k + 1] = ai - ti;
            }
        }
    }
}

/* direct DFT of the n values in tmp into x (spaced by `stride`) */
static void dft_direct(const double *tmp, double *x, int n, int stride, int sign) {
    int i, k;
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

enum { COL_BLOCK = 8 };

void fftw_execute(const fftw_plan p) {
    int b, r, c, q, i;
    int n0 = p->n0, n1 = p->n1;
    size_t ntot = (size_t)n0 * n1;
    int nmax = n0 > n1 ? n0 : n1;
    double *tmp = (double *)malloc(sizeof(double) * 2 * nmax * COL_BLOCK);
    /* FFTW_FORWARD = -1 means exp(-i...), i.e. the sine term carries sign -1 */
    int sgn = p->sign;
    for (b = 0; b < p->howmany; b++) {
        double *src = (double *)(p->in + (size_t)b * p->idist);
        double *dst = (double *)(p->out + (size_t)b * p->odist);
        if (dst != src) memmove(dst, src, sizeof(fftw_complex) * ntot);
        /* rows: contiguous */
        for (r = 0; r < n0; r++) {
            double *row = dst + 2 * (size_t)r * n1;
            memcpy(tmp, row, sizeof(double) * 2 * n1);
            if (p->tw1) {
                fft_pow2(tmp, n1, p->tw1, p->rev1);
                memcpy(row, tmp, sizeof(double) * 2 * n1);
            } else {
                dft_direct(tmp, row, n1, 1, sgn);
            }
        }
        /* columns, COL_BLOCK adjacent ones at a time */
        for (c = 0; c < n1; c += COL_BLOCK) {
            int nb = n1 - c < COL_BLOCK ? n1 - c : COL_BLOCK;
            for (i = 0; i < n0; i++) {
                const double *s = dst + 2 * ((size_t)i * n1 + c);
                for (q = 0; q < nb; q++) {
                    tmp[2 * ((size_t)q * n0 + i)] = s[2 * q];
                    tmp[2 * ((size_t)q * n0 + i) + 1] = s[2 * q + 1];
                }
            }
            for (q = 0; q < nb; q++) {
                double *col = tmp + 2 * (size_t)q * n0;
                if (p->tw0) fft_pow2(col, n0, p->tw0, p->rev0);
                else dft_direct(col, dst + 2 * (size_t)(c + q), n0, n1, sgn);
            }
            if (p->tw0) {
                for (i = 0; i < n0; i++) {
                    double *d = dst + 2 * ((size_t)i * n1 + c);
                    for (q = 0; q < nb; q++) {
                        d[2 * q] = tmp[2 * ((size_t)q * n0 + i)];
                        d[2 * q + 1] = tmp[2 * ((size_t)q * n0 + i) + 1];
                    }
                }
            }
        }
    }
    free(tmp);
}
