/*
 * CPU restatement of IP-Glasma's per-event hot path. TEST INFRASTRUCTURE
 * ONLY: the parity tests compare the CUDA library against it; the shipped
 * library never links it. See ipg_oracle.h for the interface and how the
 * restatement is pinned to the reference.
 *
 * Each function follows the reference file:line given in its comment, in
 * the reference's order of operations wherever that is cheap to keep (3x3
 * products accumulate k = 0, 1, 2; sums are left to right), so that most
 * stages agree with the reference to the last bits.
 */
#include "ipg_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/ipg_eig4.h"

typedef struct {
    double r, i;
} cx;
typedef struct {
    cx m[9];
} mat;

static const double HBARC = 0.1973269718; /* Phys_consts.h */

/* ---------------------------------------------------------------------- */
/* complex 3x3 algebra (Matrix.cpp:100-289)                               */
/* ---------------------------------------------------------------------- */
static inline cx cmul(cx a, cx b) {
    cx c = {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
    return c;
}
static inline cx cadd(cx a, cx b) {
    cx c = {a.r + b.r, a.i + b.i};
    return c;
}
static inline cx csub(cx a, cx b) {
    cx c = {a.r - b.r, a.i - b.i};
    return c;
}
static inline cx conjc(cx a) {
    cx c = {a.r, -a.i};
    return c;
}
static inline cx cscale(cx a, double s) {
    cx c = {a.r * s, a.i * s};
    return c;
}

static mat m_load(const double *p) {
    mat a;
    for (int k = 0; k < 9; k++) {
        a.m[k].r = p[2 * k];
        a.m[k].i = p[2 * k + 1];
    }
    return a;
}
static void m_store(double *p, const mat *a) {
    for (int k = 0; k < 9; k++) {
        p[2 * k] = a->m[k].r;
        p[2 * k + 1] = a->m[k].i;
    }
}
static mat m_id(void) {
    mat a;
    memset(&a, 0, sizeof(a));
    a.m[0].r = a.m[4].r = a.m[8].r = 1.0;
    return a;
}
static mat m_zero(void) {
    mat a;
    memset(&a, 0, sizeof(a));
    return a;
}
/* operator* (Matrix.cpp:100-118) */
static mat m_mul(mat a, mat b) {
    mat c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            c.m[3 * i + j] = cadd(cadd(cmul(a.m[3 * i], b.m[j]), cmul(a.m[3 * i + 1], b.m[3 + j])),
                                  cmul(a.m[3 * i + 2], b.m[6 + j]));
    return c;
}
/* prodABconj: A B^dag (Matrix.cpp:208-245) */
static mat m_mul_nd(mat a, mat b) {
    mat c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            c.m[3 * i + j] =
                cadd(cadd(cmul(a.m[3 * i], conjc(b.m[3 * j])), cmul(a.m[3 * i + 1], conjc(b.m[3 * j + 1]))),
                     cmul(a.m[3 * i + 2], conjc(b.m[3 * j + 2])));
    return c;
}
/* prodAconjB: A^dag B (Matrix.cpp:247-284) */
static mat m_mul_dn(mat a, mat b) {
    mat c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            c.m[3 * i + j] = cadd(cadd(cmul(conjc(a.m[i]), b.m[j]), cmul(conjc(a.m[3 + i]), b.m[3 + j])),
                                  cmul(conjc(a.m[6 + i]), b.m[6 + j]));
    return c;
}
static mat m_dag(mat a) {
    mat c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.m[3 * i + j] = conjc(a.m[3 * j + i]);
    return c;
}
static mat m_add(mat a, mat b) {
    for (int k = 0; k < 9; k++) a.m[k] = cadd(a.m[k], b.m[k]);
    return a;
}
static mat m_sub(mat a, mat b) {
    for (int k = 0; k < 9; k++) a.m[k] = csub(a.m[k], b.m[k]);
    return a;
}
/* double * Matrix */
static mat m_sc(double s, mat a) {
    for (int k = 0; k < 9; k++) a.m[k] = cscale(a.m[k], s);
    return a;
}
/* complex * Matrix: a(i) * s, full complex product */
static mat m_csc(cx s, mat a) {
    for (int k = 0; k < 9; k++) a.m[k] = cmul(a.m[k], s);
    return a;
}
static cx m_tr(mat a) { return cadd(cadd(a.m[0], a.m[4]), a.m[8]); }
/* traceOfProdcutOfMatrix(M1, M2) = sum_ij M1(i,j) M2(j,i), i then j */
static cx m_trmul(mat a, mat b) {
    cx t = {0., 0.};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) t = cadd(t, cmul(a.m[3 * i + j], b.m[3 * j + i]));
    return t;
}
/* traceless part as the reference forms it: X - (tr X / 3) * one */
static mat m_tl(mat a) {
    cx t = m_tr(a);
    cx s = {t.r / 3.0, t.i / 3.0};
    return m_sub(a, m_csc(s, m_id()));
}

/* generators t^a = lambda_a / 2 (Group.cpp:111-193) */
static mat gen(int a) {
    mat t = m_zero();
    switch (a) {
        case 0: t.m[1].r = 0.5; t.m[3].r = 0.5; break;
        case 1: t.m[1].i = -0.5; t.m[3].i = 0.5; break;
        case 2: t.m[0].r = 0.5; t.m[4].r = -0.5; break;
        case 3: t.m[2].r = 0.5; t.m[6].r = 0.5; break;
        case 4: t.m[2].i = -0.5; t.m[6].i = 0.5; break;
        case 5: t.m[5].r = 0.5; t.m[7].r = 0.5; break;
        case 6: t.m[5].i = -0.5; t.m[7].i = 0.5; break;
        default:
            t.m[0].r = 1. / (2. * sqrt(3.));
            t.m[4].r = 1. / (2. * sqrt(3.));
            t.m[8].r = -1. / (sqrt(3.));
    }
    return t;
}

/* ---------------------------------------------------------------------- */
/* MT19937-64 and the polar Gaussian (Random.cpp:1-204), restated from    */
/* Matsumoto & Nishimura's published 64-bit algorithm                     */
/* ---------------------------------------------------------------------- */
typedef struct {
    uint64_t mt[312];
    int mti;
    int iset;
    double gset;
} rng_t;

static void rng_seed(rng_t *r, uint64_t seed) {
    r->mt[0] = seed;
    for (int i = 1; i < 312; i++)
        r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
    r->mti = 312;
    r->iset = 0;
    r->gset = 0.;
}

static uint64_t rng_next(rng_t *r) {
    static const uint64_t MAG[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    uint64_t x;
    if (r->mti >= 312) {
        int i;
        for (i = 0; i < 312 - 156; i++) {
            x = (r->mt[i] & UM) | (r->mt[i + 1] & LM);
            r->mt[i] = r->mt[i + 156] ^ (x >> 1) ^ MAG[x & 1ULL];
        }
        for (; i < 311; i++) {
            x = (r->mt[i] & UM) | (r->mt[i + 1] & LM);
            r->mt[i] = r->mt[i - 156] ^ (x >> 1) ^ MAG[x & 1ULL];
        }
        x = (r->mt[311] & UM) | (r->mt[0] & LM);
        r->mt[311] = r->mt[155] ^ (x >> 1) ^ MAG[x & 1ULL];
        r->mti = 0;
    }
    x = r->mt[r->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

static double rng_real3(rng_t *r) {
    return ((double)(rng_next(r) >> 12) + 0.5) * (1.0 / 4503599627370496.0);
}

static double rng_gauss(rng_t *r) {
    if (r->iset == 0) {
        double v1, v2, rsq, fac;
        do {
            v1 = 2.0 * rng_real3(r) - 1.0;
            v2 = 2.0 * rng_real3(r) - 1.0;
            rsq = v1 * v1 + v2 * v2;
        } while (rsq > 1. || rsq == 0.);
        fac = sqrt(-2.0 * log(rsq) / rsq);
        r->gset = v1 * fac;
        r->iset = 1;
        return v2 * fac;
    }
    r->iset = 0;
    return r->gset;
}

void ipgo_gauss_stream(uint64_t seed, long count, double *out) {
    rng_t r;
    rng_seed(&r, seed);
    for (long k = 0; k < count; k++) out[k] = rng_gauss(&r);
}

/* ---------------------------------------------------------------------- */
/* SU(3) exponential (Matrix.cpp:310-426, Init.cpp:3483-3499)             */
/* ---------------------------------------------------------------------- */
static void expm_coeff(const double *Q, double complex res[9]) {
    const double sqrt3 = sqrt(3.);
    double c0 = sqrt3 * (Q[0] * Q[0] * Q[7] + Q[1] * Q[1] * Q[7] + Q[2] * Q[2] * Q[7]);
    c0 -= Q[7] * Q[7] * Q[7] / sqrt3;
    c0 -= (sqrt3 / 2.) * (Q[3] * Q[3] * Q[7] + Q[4] * Q[4] * Q[7] + Q[5] * Q[5] * Q[7] +
                          Q[6] * Q[6] * Q[7]);
    c0 += 3. * (Q[0] * Q[3] * Q[5] + Q[0] * Q[4] * Q[6] + Q[1] * Q[4] * Q[5] - Q[1] * Q[3] * Q[6]);
    c0 += 1.5 * (Q[2] * Q[3] * Q[3] + Q[2] * Q[4] * Q[4] - Q[2] * Q[5] * Q[5] - Q[2] * Q[6] * Q[6]);
    c0 /= 12.;
    double c1 = 0.;
    for (int a = 0; a < 8; a++) c1 += Q[a] * Q[a];
    c1 *= 0.25;
    double c0max = fmax(1e-15, 2. * pow(c1 / 3., 1.5));
    if (!(c0max >= 1e-15)) c0max = 1e-15; /* std::max(1e-15, NaN) keeps 1e-15 */
    const double th = acos(c0 / c0max) / 3.;
    const double u = sqrt(c1 / 3.) * cos(th);
    const double w = sqrt(c1) * sin(th);
    const double xi0 = sin(w) / w;
    const double den = 9. * u * u - w * w;
    const double complex iu = I * u;
    const double cosw = cos(w);
    const double complex exp2iu = cexp(2. * iu);
    const double complex expmiu = cexp(-iu);
    double complex f0 = (u * u - w * w) * exp2iu +
                        expmiu * (8. * u * u * cosw + 2. * iu * xi0 * (3. * u * u + w * w));
    f0 /= den;
    double complex f1 = 2. * u * exp2iu - expmiu * (2. * u * cosw - I * (3. * u * u - w * w) * xi0);
    f1 /= den;
    double complex f2 = exp2iu - expmiu * (cosw + 3. * iu * xi0);
    f2 /= den;
    const double complex u0 = f0 + 2. / 3. * c1 * f2;
    f1 /= (0.5 * f2);
    double complex ua[8];
    for (int i = 0; i < 8; i++) ua[i] = f1 * Q[i];
    ua[0] += (Q[3] * Q[5] + Q[4] * Q[6] + 2. / sqrt3 * Q[0] * Q[7]);
    ua[1] += (2. * Q[1] * Q[7] / sqrt3 - Q[3] * Q[6] + Q[4] * Q[5]);
    ua[2] += (2. * Q[2] * Q[7] / sqrt3 + 0.5 * Q[3] * Q[3] + 0.5 * Q[4] * Q[4] - 0.5 * Q[5] * Q[5] -
              0.5 * Q[6] * Q[6]);
    ua[3] += (-1. / sqrt3 * Q[3] * Q[7] + Q[0] * Q[5] - Q[1] * Q[6] + Q[2] * Q[3]);
    ua[4] += (-1. / sqrt3 * Q[4] * Q[7] + Q[0] * Q[6] + Q[1] * Q[5] + Q[2] * Q[4]);
    ua[5] += (-1. / sqrt3 * Q[5] * Q[7] + Q[0] * Q[3] + Q[1] * Q[4] - Q[2] * Q[5]);
    ua[6] += (-1. / sqrt3 * Q[6] * Q[7] + Q[0] * Q[4] - Q[1] * Q[3] - Q[2] * Q[6]);
    ua[7] += (Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2] - Q[7] * Q[7] - 0.5 * Q[3] * Q[3] -
              0.5 * Q[4] * Q[4] - 0.5 * Q[5] * Q[5] - 0.5 * Q[6] * Q[6]) /
             sqrt3;
    res[0] = u0;
    for (int i = 0; i < 8; i++) res[i + 1] = ua[i] * 0.5 * f2;
    for (int i = 0; i < 9; i++)
        if (isnan(creal(res[i])) || isnan(cimag(res[i]))) res[i] = 0;
}

static mat exp_from(const double *in) {
    double complex c[9];
    expm_coeff(in, c);
    if (fabs(creal(c[0])) < 1e-15) return m_id();
    /* U0 * one + U1 t0 + ... + U8 t7, summed left to right */
    cx s0 = {creal(c[0]), cimag(c[0])};
    mat acc = m_csc(s0, m_id());
    for (int a = 0; a < 8; a++) {
        cx s = {creal(c[a + 1]), cimag(c[a + 1])};
        acc = m_add(acc, m_csc(s, gen(a)));
    }
    return acc;
}

void ipgo_expm(const double in[8], double out[18]) {
    mat m = exp_from(in);
    m_store(out, &m);
}

/* ---------------------------------------------------------------------- */
/* Poisson solve with the reference's centred FFT (FFT.cpp:492-605)       */
/* ---------------------------------------------------------------------- */
static void fft1(double *x, int n, int stride, int sign, double *tmp) {
    for (int i = 0; i < n; i++) {
        tmp[2 * i] = x[2 * (size_t)i * stride];
        tmp[2 * i + 1] = x[2 * (size_t)i * stride + 1];
    }
    if ((n & (n - 1)) == 0) {
        int bits = 0;
        while ((1 << bits) < n) bits++;
        for (int i = 0; i < n; i++) {
            int r = 0;
            for (int b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
            if (r > i) {
                double t0 = tmp[2 * i], t1 = tmp[2 * i + 1];
                tmp[2 * i] = tmp[2 * r];
                tmp[2 * i + 1] = tmp[2 * r + 1];
                tmp[2 * r] = t0;
                tmp[2 * r + 1] = t1;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int h = len >> 1;
            for (int k = 0; k < h; k++) {
                const double ang = 2.0 * M_PI * (double)k / (double)len;
                const double wr = cos(ang), wi = sign * sin(ang);
                for (int i = k; i < n; i += len) {
                    const double br = tmp[2 * (i + h)], bi = tmp[2 * (i + h) + 1];
                    const double tr = br * wr - bi * wi, ti = br * wi + bi * wr;
                    const double ar = tmp[2 * i], ai = tmp[2 * i + 1];
                    tmp[2 * i] = ar + tr;
                    tmp[2 * i + 1] = ai + ti;
                    tmp[2 * (i + h)] = ar - tr;
                    tmp[2 * (i + h) + 1] = ai - ti;
                }
            }
        }
        for (int i = 0; i < n; i++) {
            x[2 * (size_t)i * stride] = tmp[2 * i];
            x[2 * (size_t)i * stride + 1] = tmp[2 * i + 1];
        }
    } else {
        for (int k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (int i = 0; i < n; i++) {
                const long m = ((long)i * k) % n;
                const double ang = 2.0 * M_PI * (double)m / (double)n;
                const double wr = cos(ang), wi = sign * sin(ang);
                sr += tmp[2 * i] * wr - tmp[2 * i + 1] * wi;
                si += tmp[2 * i] * wi + tmp[2 * i + 1] * wr;
            }
            x[2 * (size_t)k * stride] = sr;
            x[2 * (size_t)k * stride + 1] = si;
        }
    }
}

/* fftnComplex(data, data, nn, isign): shift, FFTW-sign transform, 1/N^2 on
 * the inverse, shift back. isign = 1 -> exp(-i..), -1 -> exp(+i..). */
static void fftn_centred(double *d, int N, int isign, double *work, double *tmp) {
    const int h = N / 2;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            const int ni = (i + h) % N, nj = (j + h) % N; /* input[(i+N/2)%N] = data[i] */
            work[2 * ((size_t)ni * N + nj)] = d[2 * ((size_t)i * N + j)];
            work[2 * ((size_t)ni * N + nj) + 1] = d[2 * ((size_t)i * N + j) + 1];
        }
    const int sgn = (isign == 1) ? -1 : 1;
    for (int r = 0; r < N; r++) fft1(work + 2 * (size_t)r * N, N, 1, sgn, tmp);
    for (int c = 0; c < N; c++) fft1(work + 2 * (size_t)c, N, N, sgn, tmp);
    if (isign == -1) {
        const double ntot = (double)N * N;
        for (size_t k = 0; k < 2 * (size_t)N * N; k++) work[k] /= ntot;
    }
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            const int ni = (i + h) % N, nj = (j + h) % N;
            d[2 * ((size_t)i * N + j)] = work[2 * ((size_t)ni * N + nj)];
            d[2 * ((size_t)i * N + j) + 1] = work[2 * ((size_t)ni * N + nj) + 1];
        }
}

void ipgo_wilson_lines(int N, int Ny, double L, double g, double m_GeV, double uvdamp,
                       const double *g2mu2, const double *xi, double *V) {
    const size_t n = (size_t)N * N;
    const double a = L / N;
    const double m = m_GeV * a / HBARC;
    const double uvd = uvdamp / a * HBARC;
    double *rho = (double *)malloc(sizeof(double) * 2 * n * 8);
    double *work = (double *)malloc(sizeof(double) * 2 * n);
    double *tmp = (double *)malloc(sizeof(double) * 2 * N);
    double *col = (double *)malloc(sizeof(double) * 2 * n);
    for (size_t p = 0; p < n; p++) {
        mat one = m_id();
        m_store(V + 18 * p, &one);
    }
    for (int k = 0; k < Ny; k++) {
        /* rho^a = g sqrt(g2mu2/Ny) xi (Init.cpp:1695-1705) */
        for (size_t pos = 0; pos < n; pos++)
            for (int c = 0; c < 8; c++) {
                const double amp = g * sqrt(g2mu2[pos] / (double)Ny);
                rho[2 * (c * n + pos)] = amp * xi[((size_t)k * n + pos) * 8 + c];
                rho[2 * (c * n + pos) + 1] = 0.;
            }
        for (int c = 0; c < 8; c++) {
            double *d = rho + 2 * c * n;
            fftn_centred(d, N, 1, work, tmp);
            /* Init.cpp:1712-1742 */
            for (int i = 0; i < N; i++)
                for (int j = 0; j < N; j++) {
                    const double kx = 2. * M_PI * (-0.5 + (double)i / (double)N);
                    const double ky = 2. * M_PI * (-0.5 + (double)j / (double)N);
                    const double kt2 = 4. * (sin(kx / 2.) * sin(kx / 2.) + sin(ky / 2.) * sin(ky / 2.));
                    const size_t q = (size_t)i * N + j;
                    if (m == 0) {
                        if (kt2 != 0) {
                            d[2 * q] *= (1. / kt2);
                            d[2 * q + 1] *= (1. / kt2);
                        } else {
                            d[2 * q] = 0.;
                            d[2 * q + 1] = 0.;
                        }
                    } else {
                        const double f = (1. / (kt2 + m * m)) * exp(-sqrt(kt2) * uvd);
                        d[2 * q] *= f;
                        d[2 * q + 1] *= f;
                    }
                }
            fftn_centred(d, N, -1, work, tmp);
        }
        /* V <- exp(-i A t) V (Init.cpp:1750-1768) */
        for (size_t pos = 0; pos < n; pos++) {
            double in[8];
            for (int c = 0; c < 8; c++) in[c] = -rho[2 * (c * n + pos)];
            mat e = exp_from(in);
            mat v = m_load(V + 18 * pos);
            v = m_mul(e, v);
            m_store(V + 18 * pos, &v);
        }
    }
    free(rho);
    free(work);
    free(tmp);
    free(col);
}

/* ---------------------------------------------------------------------- */
/* tau = 0 (Init.cpp:2437-2691, 3344-3481, solveAxb 47-63)                */
/* ---------------------------------------------------------------------- */
static void lu_solve(double J[64], const double F[8], double x[8]) {
    int perm[8];
    for (int i = 0; i < 8; i++) perm[i] = i;
    for (int col = 0; col < 7; col++) {
        int piv = col;
        double best = fabs(J[col * 8 + col]);
        for (int row = col + 1; row < 8; row++)
            if (fabs(J[row * 8 + col]) > best) {
                best = fabs(J[row * 8 + col]);
                piv = row;
            }
        if (piv != col) {
            for (int k = 0; k < 8; k++) {
                double t = J[col * 8 + k];
                J[col * 8 + k] = J[piv * 8 + k];
                J[piv * 8 + k] = t;
            }
            int t = perm[col];
            perm[col] = perm[piv];
            perm[piv] = t;
        }
        const double d = J[col * 8 + col];
        if (d != 0.0)
            for (int row = col + 1; row < 8; row++) {
                const double l = J[row * 8 + col] / d;
                J[row * 8 + col] = l;
                for (int k = col + 1; k < 8; k++) J[row * 8 + k] = J[row * 8 + k] - l * J[col * 8 + k];
            }
    }
    double y[8];
    for (int i = 0; i < 8; i++) y[i] = F[perm[i]];
    for (int i = 1; i < 8; i++) {
        double acc = y[i];
        for (int j = 0; j < i; j++) acc -= J[i * 8 + j] * y[j];
        y[i] = acc;
    }
    for (int i = 7; i >= 0; i--) {
        double acc = y[i];
        for (int j = i + 1; j < 8; j++) acc -= J[i * 8 + j] * y[j];
        y[i] = acc / J[i * 8 + i];
    }
    for (int i = 0; i < 8; i++) x[i] = y[i];
}

/* findUInForwardLightconeChun without the random restarts: returns the
 * iteration count, or -1 when a restart would have been drawn */
static int newton_link(mat U1, mat U2, mat *Usol_out) {
    mat T[8];
    for (int a = 0; a < 8; a++) T[a] = gen(a);
    const mat U0 = m_mul(U1, U2);
    const mat S = m_add(U1, U2);
    const mat Sd = m_dag(S);
    cx tc[8];
    mat MA[8];
    for (int a = 0; a < 8; a++) {
        tc[a] = m_tr(m_mul(T[a], m_sub(S, Sd)));
        MA[a] = m_mul(T[a], S);
    }
    double alpha[8] = {0, 0, 0, 0, 0, 0, 0, 0}, dal[8], Fa[8], J[64];
    mat Usol = m_mul(exp_from(alpha), U0);
    mat Usd = m_dag(Usol);
    double Fzero = 10.;
    int iter = 0;
    while (Fzero > 1e-6 && iter < 2000) {
        iter++;
        Fzero = 0.;
        mat Mt = m_sub(m_mul(S, Usd), m_mul(Usol, Sd));
        for (int a = 0; a < 8; a++) {
            cx tl = m_trmul(T[a], Mt);
            cx tr = cadd(tc[a], tl);
            Fa[a] = -tr.i;
            Fzero += fabs(Fa[a]);
        }
        int good = 1;
        for (int b = 0; b < 8; b++) {
            double d = fmax(0.001, fmin(10., 0.01 * fabs(alpha[b])));
            alpha[b] = alpha[b] + d;
            mat M2 = m_dag(m_mul(exp_from(alpha), U0));
            M2 = m_mul(S, m_sub(M2, Usd));
            double mcheck = 0.;
            for (int a = 0; a < 8; a++) {
                cx tl = m_trmul(T[a], M2);
                J[a * 8 + b] = 2. * tl.i / d;
                mcheck += fabs(J[a * 8 + b]);
                if (mcheck < 1e-15) good = 0;
            }
            alpha[b] = alpha[b] - d;
        }
        if (!good)
            for (int b = 0; b < 8; b++) {
                mat M3 = m_mul(T[b], Usd);
                for (int a = 0; a < 8; a++) J[a * 8 + b] = -2. * m_trmul(MA[a], M3).r;
            }
        lu_solve(J, Fa, dal);
        for (int a = 0; a < 8; a++)
            if (fabs(dal[a]) > 1e5) return -1;
        for (int a = 0; a < 8; a++) alpha[a] = alpha[a] + dal[a];
        Usol = m_mul(exp_from(alpha), U0);
        Usd = m_dag(Usol);
    }
    *Usol_out = Usol;
    return Fzero > 1e-6 ? -1 : iter;
}

int ipgo_tau0(int N, double g, const double *VA, const double *VB, double *Ux, double *Uy,
              double *pi, int *newton_iters) {
    const size_t n = (size_t)N * N;
    mat *u1x = (mat *)malloc(sizeof(mat) * n), *u2x = (mat *)malloc(sizeof(mat) * n);
    mat *u1y = (mat *)malloc(sizeof(mat) * n), *u2y = (mat *)malloc(sizeof(mat) * n);
    mat *ux = (mat *)malloc(sizeof(mat) * n), *uy = (mat *)malloc(sizeof(mat) * n);
    int restarts = 0;
#define VAT(V, p) (m_load((V) + 18 * (p)))
    for (size_t pos = 0; pos < n; pos++) {
        const int i = (int)(pos / N), j = (int)(pos % N);
        const size_t pX = (size_t)(i + 1 < N ? i + 1 : N - 1) * N + j;
        const size_t pY = (size_t)i * N + (j + 1 < N ? j + 1 : N - 1);
        mat a = VAT(VA, pos), b = VAT(VB, pos);
        u1x[pos] = m_mul(a, m_dag(VAT(VA, pX)));
        u1y[pos] = m_mul(a, m_dag(VAT(VA, pY)));
        u2x[pos] = m_mul(b, m_dag(VAT(VB, pX)));
        u2y[pos] = m_mul(b, m_dag(VAT(VB, pY)));
    }
#pragma omp parallel for reduction(+ : restarts) schedule(dynamic, 64)
    for (long pos = 0; pos < (long)n; pos++) {
        int itx = newton_link(u1x[pos], u2x[pos], &ux[pos]);
        int ity = newton_link(u1y[pos], u2y[pos], &uy[pos]);
        restarts += (itx < 0) + (ity < 0);
        if (newton_iters) {
            newton_iters[2 * pos] = itx;
            newton_iters[2 * pos + 1] = ity;
        }
    }
    /* "minus" stencil and pi = (-2i/g) E1 (Init.cpp:2521-2584, 2664-2681) */
    for (size_t pos = 0; pos < n; pos++) {
        const int i = (int)(pos / N), j = (int)(pos % N);
        const size_t mX = (size_t)(i > 0 ? i - 1 : 0) * N + j;
        const size_t mY = (size_t)i * N + (j > 0 ? j - 1 : 0);
        mat D = m_sub(u1x[pos], u2x[pos]), Dd = m_sub(m_dag(u1x[pos]), m_dag(u2x[pos]));
        mat U = ux[pos], Ud = m_dag(U);
        mat t = m_add(m_sub(m_sub(m_mul(D, Ud), D), m_mul(U, Dd)), Dd);
        D = m_sub(u1x[mX], u2x[mX]);
        Dd = m_sub(m_dag(u1x[mX]), m_dag(u2x[mX]));
        U = ux[mX];
        Ud = m_dag(U);
        t = m_sub(m_add(m_add(m_sub(t, m_mul(Ud, D)), D), m_mul(Dd, U)), Dd);
        D = m_sub(u1y[pos], u2y[pos]);
        Dd = m_sub(m_dag(u1y[pos]), m_dag(u2y[pos]));
        U = uy[pos];
        Ud = m_dag(U);
        t = m_add(m_sub(m_sub(m_add(t, m_mul(D, Ud)), D), m_mul(U, Dd)), Dd);
        D = m_sub(u1y[mY], u2y[mY]);
        Dd = m_sub(m_dag(u1y[mY]), m_dag(u2y[mY]));
        U = uy[mY];
        Ud = m_dag(U);
        t = m_sub(m_add(m_add(m_sub(t, m_mul(Ud, D)), D), m_mul(Dd, U)), Dd);
        mat E1 = m_sc(1. / 8., t);
        cx s = {0., -2. / g};
        mat p = m_csc(s, E1);
        m_store(pi + 18 * pos, &p);
        m_store(Ux + 18 * pos, &ux[pos]);
        m_store(Uy + 18 * pos, &uy[pos]);
    }
    free(u1x);
    free(u2x);
    free(u1y);
    free(u2y);
    free(ux);
    free(uy);
    return restarts;
}

/* ---------------------------------------------------------------------- */
/* leapfrog (Evolution.cpp:35-293)                                         */
/* ---------------------------------------------------------------------- */
#define AT(F, p) (m_load((F) + 18 * (size_t)(p)))

void ipgo_evolve_phi(int N, double dtau, double tau, double *phi, const double *pi) {
    const size_t n = (size_t)N * N;
    for (size_t p = 0; p < n; p++) {
        mat f = m_add(AT(phi, p), m_sc((tau + dtau / 2.) * dtau, AT(pi, p)));
        m_store(phi + 18 * p, &f);
    }
}

void ipgo_evolve_u(int N, double g, double dtau, double tau, double *Ux, double *Uy,
                   const double *E1, const double *E2) {
    const size_t n = (size_t)N * N;
    const cx c = {0., g * g * dtau / (tau + dtau / 2.)};
    for (size_t p = 0; p < n; p++) {
        for (int d = 0; d < 2; d++) {
            mat X = m_csc(c, AT(d ? E2 : E1, p));
            mat t2 = m_add(m_id(), m_sc(1. / 2., X));
            mat t1 = m_mul(X, t2);
            t2 = m_add(m_id(), m_sc(1. / 1., t1));
            mat u = m_mul(t2, AT(d ? Uy : Ux, p));
            m_store((d ? Uy : Ux) + 18 * p, &u);
        }
    }
}

void ipgo_evolve_pi(int N, double dtau, double tau, const double *Ux, const double *Uy,
                    const double *phi, double *pi) {
    const size_t n = (size_t)N * N;
    for (size_t pos = 0; pos < n; pos++) {
        const int i = (int)(pos / N), j = (int)(pos % N);
        const size_t pX = (size_t)(i + 1 < N ? i + 1 : N - 1) * N + j;
        const size_t pY = (size_t)i * N + (j + 1 < N ? j + 1 : N - 1);
        const size_t mX = (size_t)(i > 0 ? i - 1 : 0) * N + j;
        const size_t mY = (size_t)i * N + (j > 0 ? j - 1 : 0);
        const mat ux = AT(Ux, pos), uy = AT(Uy, pos);
        const mat phX = m_mul(ux, m_mul_nd(AT(phi, pX), ux));
        const mat phY = m_mul(uy, m_mul_nd(AT(phi, pY), uy));
        const mat uxm = AT(Ux, mX), uym = AT(Uy, mY);
        const mat phmX = m_mul(m_mul_dn(uxm, AT(phi, mX)), uxm);
        const mat phmY = m_mul(m_mul_dn(uym, AT(phi, mY)), uym);
        mat br = m_sub(m_add(m_add(m_add(phX, phmX), phY), phmY), m_sc(4., AT(phi, pos)));
        mat p = m_add(AT(pi, pos), m_sc(dtau / (tau), br));
        m_store(pi + 18 * pos, &p);
    }
}

void ipgo_evolve_e(int N, double g, double dtau, double tau, const double *Ux,
                   const double *Uy, const double *phi, double *E1, double *E2) {
    const size_t n = (size_t)N * N;
    const cx ia = {0. * tau * dtau / (2. * g * g), 1. * tau * dtau / (2. * g * g)};
    const cx ib = {0. * dtau / tau, 1. * dtau / tau};
    for (size_t pos = 0; pos < n; pos++) {
        const int i = (int)(pos / N), j = (int)(pos % N);
        const size_t pX = (size_t)(i + 1 < N ? i + 1 : N - 1) * N + j;
        const size_t pY = (size_t)i * N + (j + 1 < N ? j + 1 : N - 1);
        const size_t mX = (size_t)(i > 0 ? i - 1 : 0) * N + j;
        const size_t mY = (size_t)i * N + (j > 0 ? j - 1 : 0);
        const size_t mXpY = (size_t)(i > 0 ? i - 1 : 0) * N + (j + 1 < N ? j + 1 : N - 1);
        const size_t pXmY = (size_t)(i + 1 < N ? i + 1 : N - 1) * N + (j > 0 ? j - 1 : 0);
        const mat ux = AT(Ux, pos), uy = AT(Uy, pos), ph = AT(phi, pos);
        mat phN = m_mul(ux, m_mul_nd(AT(phi, pX), ux));
        const mat U12 = m_mul(m_mul(ux, AT(Uy, pX)), m_mul_nd(m_dag(AT(Ux, pY)), uy));
        const mat U1m2 = m_mul(m_mul_nd(ux, AT(Uy, pXmY)), m_mul_dn(AT(Ux, mY), AT(Uy, mY)));
        const mat U2m1 = m_mul(m_mul_nd(uy, AT(Ux, mXpY)), m_mul_dn(AT(Uy, mX), AT(Ux, mX)));
        const mat U12d = m_dag(U12);
        mat t1 = m_sub(m_sub(m_add(U12, U1m2), U12d), m_dag(U1m2));
        t1 = m_tl(t1);
        mat t2 = m_sub(m_mul(phN, ph), m_mul(ph, phN));
        mat En = m_add(AT(E1, pos), m_add(m_csc(ia, t1), m_csc(ib, t2)));
        En = m_tl(En);
        m_store(E1 + 18 * pos, &En);
        t1 = m_sub(m_sub(m_add(U12d, U2m1), U12), m_dag(U2m1));
        t1 = m_tl(t1);
        phN = m_mul(uy, m_mul_nd(AT(phi, pY), uy));
        t2 = m_sub(m_mul(phN, ph), m_mul(ph, phN));
        En = m_add(AT(E2, pos), m_add(m_csc(ia, t1), m_csc(ib, t2)));
        En = m_tl(En);
        m_store(E2 + 18 * pos, &En);
    }
}

/* ---------------------------------------------------------------------- */
/* T^{mu nu} (Evolution.cpp:659-1246)                                     */
/* ---------------------------------------------------------------------- */
static inline double retr(mat a) { return m_tr(a).r; }
static inline double imtr(mat a) { return m_tr(a).i; }
static mat fwd(mat u, mat a) { return m_mul(m_mul(u, a), m_dag(u)); } /* U A U^dag */
static mat bwd(mat u, mat a) { return m_mul(m_mul(m_dag(u), a), u); } /* U^dag A U */
static mat tl_diff(mat a, mat b) { return m_tl(m_sub(a, b)); }
static mat m4(mat a, mat b, mat c, mat d) { return m_mul(m_mul(m_mul(a, b), c), d); }

void ipgo_tmunu(int N, double L, double g, double dtau, int it, const double *Ux,
                const double *Uy, const double *E1, const double *E2, const double *phi,
                const double *pi, double *T10) {
    const size_t n = (size_t)N * N;
    const double a = L / N, tau = it * dtau;
    const double a4 = pow(a, 4.), a5 = pow(a, 5.), a6 = pow(a, 6.);
#define IX(ii, jj) ((size_t)(ii) * N + (jj))
#define CL(v) ((v) < 0 ? 0 : ((v) > N - 1 ? N - 1 : (v)))
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            const size_t pos = IX(i, j), pX = IX(CL(i + 1), j), pY = IX(i, CL(j + 1));
            const size_t pXY = IX(CL(i + 1), CL(j + 1));
            const size_t mX = IX(CL(i - 1), j), mY = IX(i, CL(j - 1));
            const size_t mXpY = IX(CL(i - 1), CL(j + 1)), pXmY = IX(CL(i + 1), CL(j - 1));
            const size_t p2X = IX(CL(i + 2), j), p2Y = IX(i, CL(j + 2));
            const size_t p2XY = IX(CL(i + 2), CL(j + 1)), pX2Y = IX(CL(i + 1), CL(j + 2));
            const mat e1 = AT(E1, pos), e2 = AT(E2, pos), e1p = AT(E1, pY), e2p = AT(E2, pX);
            const mat p0 = AT(pi, pos), pX_ = AT(pi, pX), pY_ = AT(pi, pY), pXY_ = AT(pi, pXY);
            const double trE = retr(m_mul(e1, e1)) + retr(m_mul(e1p, e1p)) +
                               retr(m_mul(e2, e2)) + retr(m_mul(e2p, e2p));
            const double trEx = -retr(m_mul(e1, e1)) - retr(m_mul(e1p, e1p)) +
                                retr(m_mul(e2, e2)) + retr(m_mul(e2p, e2p));
            const double trEy = retr(m_mul(e1, e1)) + retr(m_mul(e1p, e1p)) -
                                retr(m_mul(e2, e2)) - retr(m_mul(e2p, e2p));
            const double trP = retr(m_mul(p0, p0)) + retr(m_mul(pX_, pX_)) +
                               retr(m_mul(pY_, pY_)) + retr(m_mul(pXY_, pXY_));
            const double ge = g * g / tau / tau;
            double Ttt = ge * trE / 2. + trP / 4.;
            double Txx = ge * trEx / 2. + trP / 4.;
            double Tyy = ge * trEy / 2. + trP / 4.;
            double Tee = 1. / tau / tau * (ge * trE / 2. - trP / 4.);

            const mat ux = AT(Ux, pos), uy = AT(Uy, pos);
            const mat uxpX = AT(Ux, pX), uxpY = AT(Ux, pY), uypX = AT(Uy, pX), uypY = AT(Uy, pY);
            double B = 0.;
            if (i != N - 1) {
                const mat pl = m_mul(ux, m_mul(uypX, m_mul(m_dag(uxpY), m_dag(uy))));
                B = 2. / pow(g, 2.) * (3. - retr(pl));
            }
            const mat f0 = AT(phi, pos), fX = AT(phi, pX), fY = AT(phi, pY), fXY = AT(phi, pXY);
            const mat ptX = fwd(ux, fX), ptY = fwd(uy, fY);
            const mat ptXY1 = fwd(uxpY, fXY), ptXY2 = fwd(uypX, fXY);
            const mat d1 = m_sub(f0, ptX), d2 = m_sub(fY, ptXY1), d3 = m_sub(f0, ptY), d4 = m_sub(fX, ptXY2);
            const double P1 = retr(m_mul(d1, d1)), P2 = retr(m_mul(d2, d2));
            const double P3 = retr(m_mul(d3, d3)), P4 = retr(m_mul(d4, d4));
            Ttt = Ttt + 2. / pow(g, 2.) * (3. - (i == N - 1 ? 3. : 3. - B * pow(g, 2.) / 2.)) * 0. + B +
                  0.5 / tau / tau * (P1 + P2 + P3 + P4);
            Txx = Txx + B + 0.5 / tau / tau * (P1 + P2 - P3 - P4);
            Tyy = Tyy + B + 0.5 / tau / tau * (-P1 - P2 + P3 + P4);
            Tee = Tee + 1. / tau / tau * (-B + 0.5 / tau / tau * (P1 + P2 + P3 + P4));
            T10[0 * n + pos] = Ttt * 1 / a4;
            T10[1 * n + pos] = Txx * 1 / a4;
            T10[2 * n + pos] = Tyy * 1 / a4;
            T10[3 * n + pos] = Tee * 1 / a6;

            /* off-diagonal components, the expressions of Evolution.cpp:1045-1226 */
            const mat uxmX = AT(Ux, mX), uymX = AT(Uy, mX), uxmXpY = AT(Ux, mXpY);
            const mat uxpXpY = AT(Ux, pXY), uyp2X = AT(Uy, p2X);
            const mat uymY = AT(Uy, mY), uxmY = AT(Ux, mY), uypXmY = AT(Uy, pXmY);
            const mat uypXpY = AT(Uy, pXY), uxp2Y = AT(Ux, p2Y);
            const mat Dx = m_dag(ux), Dy = m_dag(uy), DxpY = m_dag(uxpY), DypX = m_dag(uypX);
            const mat DxmX = m_dag(uxmX), DymX = m_dag(uymX), DxmXpY = m_dag(uxmXpY);
            const mat DxpX = m_dag(uxpX), DxpXpY = m_dag(uxpXpY), Dyp2X = m_dag(uyp2X);
            const mat DymY = m_dag(uymY), DxmY = m_dag(uxmY), DypXmY = m_dag(uypXmY);
            const mat DypY = m_dag(uypY), DypXpY = m_dag(uypXpY), Dxp2Y = m_dag(uxp2Y);
            const mat P_a = m4(uy, uxpY, DypX, Dx), P_b = m4(ux, uypX, DxpY, Dy);
            const mat Q1 = m4(DxmX, uymX, uxmXpY, Dy), Q1d = m4(uy, DxmXpY, DymX, uxmX);
            const mat R1 = m4(uypX, uxpXpY, Dyp2X, DxpX), R1d = m4(uxpX, uyp2X, DxpXpY, DypX);
            const mat S1 = m4(Dx, uy, uxpY, DypX), S1d = m4(uypX, DxpY, Dy, ux);
            const mat Q3 = m4(DymY, uxmY, uypXmY, Dx), Q3d = m4(ux, DypXmY, DxmY, uymY);
            const mat R3 = m4(uxpY, uypXpY, Dxp2Y, DypY), R3d = m4(uypY, uxp2Y, DypXpY, DxpY);
            const mat S3 = m4(Dy, ux, uypX, DxpY), S3d = m4(uxpY, DypX, Dx, uy);
            const mat fmX = AT(phi, mX), fmY = AT(phi, mY), fmXpY = AT(phi, mXpY), fpXmY = AT(phi, pXmY);
            const mat f2X = AT(phi, p2X), f2Y = AT(phi, p2Y), f2XY = AT(phi, p2XY), fX2Y = AT(phi, pX2Y);
            {
                mat K = m_add(tl_diff(P_a, P_b), tl_diff(Q1, Q1d));
                mat Kp = m_add(tl_diff(R1, R1d), tl_diff(S1, S1d));
                const double mag = imtr(m_add(m_mul(e2, K), m_mul(e2p, Kp)));
                mat el = m_mul(p0, m_sub(fwd(ux, fX), bwd(uxmX, fmX)));
                el = m_add(el, m_mul(pY_, m_sub(fwd(uxpY, fXY), bwd(uxmXpY, fmXpY))));
                el = m_add(el, m_mul(pX_, m_sub(fwd(uxpX, f2X), bwd(ux, f0))));
                el = m_add(el, m_mul(pXY_, m_sub(fwd(uxpXpY, f2XY), bwd(uxpY, fY))));
                T10[4 * n + pos] = (2. / tau / 8. * mag - 2. / 8. / tau * retr(el)) * 1 / a4;
            }
            {
                mat K = m_add(tl_diff(P_b, P_a), tl_diff(Q3, Q3d));
                mat Kp = m_add(tl_diff(R3, R3d), tl_diff(S3, S3d));
                const double mag = imtr(m_add(m_mul(e1, K), m_mul(e1p, Kp)));
                mat el = m_mul(p0, m_sub(fwd(uy, fY), bwd(uymY, fmY)));
                el = m_add(el, m_mul(pX_, m_sub(fwd(uypX, fXY), bwd(uypXmY, fpXmY))));
                el = m_add(el, m_mul(pY_, m_sub(fwd(uypY, f2Y), bwd(uy, f0))));
                el = m_add(el, m_mul(pXY_, m_sub(fwd(uypXpY, fX2Y), bwd(uypX, fX))));
                T10[5 * n + pos] = (2. / tau / 8. * mag - 2. / 8. / tau * retr(el)) * 1 / a4;
            }
            const mat dX = m_sub(ptX, f0), dY = m_sub(ptY, f0);
            const mat dXY1 = m_sub(ptXY1, fY), dXY2 = m_sub(ptXY2, fX);
            {
                mat t = m_add(m_add(m_add(m_mul(e1, dX), m_mul(e1p, dXY1)), m_mul(e2, dY)), m_mul(e2p, dXY2));
                T10[6 * n + pos] = (g / tau / tau / tau * retr(t)) * 1 / a5;
            }
            {
                mat ea = m_add(e1, fwd(uy, e1p)), eb = m_add(e2, fwd(ux, e2p));
                mat t = m_mul(m_sc(-1. / 4. * g * g, ea), eb);
                mat wy = m_mul(m_mul(uy, dXY1), Dy), wx = m_mul(m_mul(ux, dXY2), Dx);
                mat q = m_add(m_add(m_add(m_mul(dX, dY), m_mul(wy, dY)), m_mul(dX, wx)), m_mul(wy, wx));
                t = m_add(t, m_sc(1. / 4., q));
                T10[7 * n + pos] = (2. / tau / tau * retr(t)) * 1 / a4;
            }
            {
                mat e = m_add(m_mul(e1, m_add(p0, fwd(ux, pX_))), m_mul(e1p, m_add(pY_, fwd(uxpY, pXY_))));
                mat K = m_add(tl_diff(P_b, P_a), tl_diff(Q1d, Q1));
                mat Kp = m_add(tl_diff(S1d, S1), tl_diff(R1d, R1));
                mat m = m_add(m_mul(K, dY), m_mul(Kp, dXY2));
                const double v = 1. / 4. * g * retr(e) + 1. / 8. / g * imtr(m);
                T10[8 * n + pos] = (-2. / tau / tau * v) * 1 / a5;
            }
            {
                mat e = m_add(m_mul(e2, m_add(p0, fwd(uy, pY_))), m_mul(e2p, m_add(pX_, fwd(uypX, pXY_))));
                mat K = m_add(tl_diff(P_a, P_b), tl_diff(Q3d, Q3));
                mat Kp = m_add(tl_diff(S3d, S3), tl_diff(R3d, R3));
                mat m = m_add(m_mul(K, dX), m_mul(Kp, dXY1));
                const double v = 1. / 4. * g * retr(e) + 1. / 8. / g * imtr(m);
                T10[9 * n + pos] = (-2. / tau / tau * v) * 1 / a5;
            }
        }
#undef IX
#undef CL
}

/* ---------------------------------------------------------------------- */
/* Landau matching (MyEigen.cpp:25-314)                                   */
/* ---------------------------------------------------------------------- */
int ipgo_landau(int N, double L, double dtau, int it, const double *T10, double *eps_out,
                double *u4, double *pi10) {
    const size_t n = (size_t)N * N;
    const double a = L / N;
    double ux = 0., uy = 0., ueta = 0., utau = 0., eps = 0.;
    int nofound = 0;
    for (int si = 0; si < N; si++)
        for (int sj = 0; sj < N; sj++) {
            const size_t pos = (size_t)si * N + sj;
            const double Ttt = T10[0 * n + pos], Txx = T10[1 * n + pos], Tyy = T10[2 * n + pos];
            const double Tee = T10[3 * n + pos], Ttx = T10[4 * n + pos], Tty = T10[5 * n + pos];
            const double Tte = T10[6 * n + pos], Txy = T10[7 * n + pos], Txe = T10[8 * n + pos];
            const double Tye = T10[9 * n + pos];
            const double t2d = (it * dtau * a) * (it * dtau * a);
            const double data[16] = {Ttt, -Ttx, -Tty, -t2d * Tte, Ttx, -Txx, -Txy, -t2d * Txe,
                                     Tty, -Txy, -Tyy, -t2d * Tye, Tte, -Txe, -Tye, -t2d * Tee};
            double er[4], ei[4], vr[16], vi[16];
            ipg_eig4(data, er, ei, vr, vi);
            double ceps = Ttt, cu[4] = {1., 0., 0., 0.};
            int found = 0;
            const double tau2 = a * it * dtau * a * it * dtau;
            for (int i = 0; i < 4; i++) {
                double sqr = 0., eur = 0.;
                for (int j = 0; j < 4; j++) {
                    const double zr = vr[4 * i + j], zi = vi[4 * i + j];
                    const double z2r = zr * zr - zi * zi;
                    eur += z2r;
                    if (j == 0) sqr += z2r;
                    else if (j < 3) sqr -= z2r;
                    else sqr -= (tau2 * zr) * zr - (tau2 * zi) * zi;
                }
                const double factor = sqrt(fabs(eur / sqr));
                if (sqr > 0) {
                    eps = er[i];
                    if (fabs(ei[i]) > 0.001 && si > 0 && sj > 0 && si < N - 5 && sj < N - 5) eps = Ttt;
                }
                double s2 = 0.;
                for (int j = 0; j < 4; j++) {
                    const double zr = vr[4 * i + j] * factor, zi = vi[4 * i + j] * factor;
                    const double z2r = zr * zr - zi * zi;
                    if (j == 0) s2 += z2r;
                    else if (j < 3) s2 -= z2r;
                    else s2 -= (tau2 * zr) * zr - (tau2 * zi) * zi;
                }
                if (s2 > 0) {
                    int change = 0;
                    found++;
                    for (int j = 0; j < 4; j++) {
                        double zr = vr[4 * i + j] * factor, zi = vi[4 * i + j] * factor;
                        if (j == 0 && zr < 0) {
                            change = 1;
                            zr = -zr;
                            zi = -zi;
                        }
                        if (j > 0 && change == 1) {
                            zr = -zr;
                            zi = -zi;
                        }
                        if (j == 0) utau = (eps > 0.1) ? zr : 1.;
                        if (j == 1) ux = (eps > 0.1) ? zr : 0.;
                        if (j == 2) uy = (eps > 0.1) ? zr : 0.;
                        if (j == 3) ueta = (eps > 0.1) ? zr : 0.;
                        if (fabs(zi) > 0.001 && eps > 0.001 && si > 10 && sj > 10 && si < N - 10 &&
                            sj < N - 10) {
                            utau = 1.;
                            ux = 0.;
                            uy = 0.;
                            ueta = 0.;
                            eps = Ttt;
                        }
                    }
                    cu[0] = utau;
                    cu[1] = ux;
                    cu[2] = uy;
                    cu[3] = ueta;
                    ceps = eps;
                }
            }
            nofound += found == 0;
            eps_out[pos] = ceps;
            for (int k = 0; k < 4; k++) u4[k * n + pos] = cu[k];
            double *P = pi10;
            if (utau == 1 && ux == 0 && uy == 0 && ueta == 0) {
                for (int k = 0; k < 10; k++) P[k * n + pos] = 0.;
            } else {
                P[0 * n + pos] = Ttt - 4. / 3. * eps * utau * utau + eps / 3.;
                P[1 * n + pos] = Txx - 4. / 3. * eps * ux * ux - eps / 3.;
                P[2 * n + pos] = Tyy - 4. / 3. * eps * uy * uy - eps / 3.;
                P[3 * n + pos] = Tee - 4. / 3. * eps * ueta * ueta - eps / 3. / it / dtau / a / it / dtau / a;
                P[4 * n + pos] = Ttx - 4. / 3. * eps * utau * ux;
                P[5 * n + pos] = Tty - 4. / 3. * eps * utau * uy;
                P[6 * n + pos] = Tte - 4. / 3. * eps * utau * ueta;
                P[7 * n + pos] = Txy - 4. / 3. * eps * ux * uy;
                P[8 * n + pos] = Txe - 4. / 3. * eps * ux * ueta;
                P[9 * n + pos] = Tye - 4. / 3. * eps * uy * ueta;
            }
        }
    return nofound;
}

/* ---------------------------------------------------------------------- */
/* Gauss law (Evolution.cpp:295-364) and eccentricity (1280-1810)         */
/* ---------------------------------------------------------------------- */
double ipgo_gauss_law(int N, const double *Ux, const double *Uy, const double *E1,
                      const double *E2, const double *phi, const double *pi) {
    double largest = 0;
    const size_t n = (size_t)N * N;
    for (size_t pos = 0; pos < n; pos++) {
        const int i = (int)(pos / N), j = (int)(pos % N);
        const size_t mX = (size_t)(i > 0 ? i - 1 : 0) * N + j;
        const size_t mY = (size_t)i * N + (j > 0 ? j - 1 : 0);
        const mat uxm = AT(Ux, mX), uym = AT(Uy, mY);
        mat G = m_sub(m_mul(m_mul(m_dag(uxm), AT(E1, mX)), uxm), AT(E1, pos));
        G = m_add(G, m_mul(m_mul(m_dag(uym), AT(E2, mY)), uym));
        G = m_sub(G, AT(E2, pos));
        const mat f = AT(phi, pos), p = AT(pi, pos);
        const cx iu = {0., 1.};
        G = m_sub(G, m_csc(iu, m_sub(m_mul(f, p), m_mul(p, f))));
        double sq = 0.;
        for (int k = 0; k < 9; k++) sq += G.m[k].r * G.m[k].r + G.m[k].i * G.m[k].i;
        sq *= 0.5;
        if (sq > largest) largest = sq;
    }
    return largest;
}

void ipgo_eccentricity(int N, double L, const double *eps, const double *utau, double ecc[6],
                       double psi[6]) {
    const double a = L / N;
    double avx = 0, avy = 0, tot = 0;
    for (int ix = 0; ix < N; ix++)
        for (int iy = 0; iy < N; iy++) {
            const size_t pos = (size_t)ix * N + iy;
            const double x = -L / 2. + a * ix, y = -L / 2. + a * iy;
            const double w = (eps[pos] < 0.) ? 0. : eps[pos] * utau[pos];
            avx += x * w;
            avy += y * w;
            tot += w;
        }
    avx /= tot;
    avy /= tot;
    double avr[6] = {0}, cs[6] = {0}, sn[6] = {0};
    for (int ix = 2; ix < N - 2; ix++)
        for (int iy = 2; iy < N - 2; iy++) {
            const size_t pos = (size_t)ix * N + iy;
            const double x = -L / 2. + a * ix - avx, y = -L / 2. + a * iy - avy;
            double ph;
            if (x >= 0) {
                ph = atan(y / x);
                if (x == 0) ph = (y >= 0) ? M_PI / 2. : 3. * M_PI / 2.;
            } else {
                ph = atan(y / x) + M_PI;
            }
            const double w = (eps[pos] < 0.) ? 0. : eps[pos] * utau[pos];
            const double r = sqrt(x * x + y * y);
            const int pw[6] = {3, 2, 3, 4, 5, 6};
            for (int k = 0; k < 6; k++) {
                double rp = 1.;
                for (int q = 0; q < pw[k]; q++) rp *= r;
                avr[k] += rp * w;
                cs[k] += rp * cos((k + 1) * ph) * w;
                sn[k] += rp * sin((k + 1) * ph) * w;
            }
        }
    for (int k = 0; k < 6; k++) {
        psi[k] = (atan(sn[k] / cs[k]) + M_PI) / (k + 1);
        ecc[k] = sqrt(cs[k] * cs[k] + sn[k] * sn[k]) / avr[k];
    }
}

/* ---------------------------------------------------------------------- */
/* whole event (Init::setV, Init::init tau=0, Evolution::run)             */
/* ---------------------------------------------------------------------- */
void ipgo_run_event(int N, int Ny, double L, double g, double m_GeV, double uvdamp,
                    double maxtime, double dtau_override, const double *g2muA,
                    const double *g2muB, const double *xiA, const double *xiB, double *VA_out,
                    double *VB_out, double *tau0_Ux, double *tau0_Uy, double *tau0_pi,
                    double *eps, double *u4, double *pi10, double *T10, double *scalars) {
    const size_t n = (size_t)N * N, bytes = sizeof(double) * 18 * n;
    const double a = L / N;
    double dtau;
    if (dtau_override > 0) {
        dtau = dtau_override;
    } else {
        const int steps = (int)(10 * maxtime / a) + 1;
        dtau = maxtime / (steps * a);
    }
    const int itmax = (int)(maxtime / (a * dtau) + 0.1);
    double *VA = malloc(bytes), *VB = malloc(bytes);
    double *Ux = malloc(bytes), *Uy = malloc(bytes), *E1 = calloc(18 * n, sizeof(double));
    double *E2 = calloc(18 * n, sizeof(double)), *phi = calloc(18 * n, sizeof(double));
    double *pi = malloc(bytes);
    double *T = malloc(sizeof(double) * 10 * n), *e = malloc(sizeof(double) * n);
    double *u = malloc(sizeof(double) * 4 * n), *p10 = malloc(sizeof(double) * 10 * n);
    ipgo_wilson_lines(N, Ny, L, g, m_GeV, uvdamp, g2muA, xiA, VA);
    ipgo_wilson_lines(N, Ny, L, g, m_GeV, uvdamp, g2muB, xiB, VB);
    if (VA_out) memcpy(VA_out, VA, bytes);
    if (VB_out) memcpy(VB_out, VB, bytes);
    const int restarts = ipgo_tau0(N, g, VA, VB, Ux, Uy, pi, NULL);
    if (tau0_Ux) memcpy(tau0_Ux, Ux, bytes);
    if (tau0_Uy) memcpy(tau0_Uy, Uy, bytes);
    if (tau0_pi) memcpy(tau0_pi, pi, bytes);
    ipgo_evolve_phi(N, dtau, 0., phi, pi);
    ipgo_evolve_u(N, g, dtau, 0., Ux, Uy, E1, E2);
    for (int it = 1; it <= itmax; it++) {
        if (it == itmax) {
            ipgo_tmunu(N, L, g, dtau, it, Ux, Uy, E1, E2, phi, pi, T);
            ipgo_landau(N, L, dtau, it, T, e, u, p10);
        }
        if (it < itmax) {
            ipgo_evolve_pi(N, dtau, it * dtau, Ux, Uy, phi, pi);
            ipgo_evolve_e(N, g, dtau, it * dtau, Ux, Uy, phi, E1, E2);
            ipgo_evolve_phi(N, dtau, it * dtau, phi, pi);
            ipgo_evolve_u(N, g, dtau, it * dtau, Ux, Uy, E1, E2);
        } else {
            ipgo_evolve_pi(N, dtau / 2., it * dtau, Ux, Uy, phi, pi);
            ipgo_evolve_e(N, g, dtau / 2., it * dtau, Ux, Uy, phi, E1, E2);
        }
    }
    double ecc[6], psi[6];
    ipgo_eccentricity(N, L, e, u, ecc, psi);
    if (scalars) {
        scalars[0] = ipgo_gauss_law(N, Ux, Uy, E1, E2, phi, pi);
        scalars[1] = ecc[1];
        scalars[2] = itmax;
        scalars[3] = dtau;
        scalars[4] = restarts;
    }
    if (eps) memcpy(eps, e, sizeof(double) * n);
    if (u4) memcpy(u4, u, sizeof(double) * 4 * n);
    if (pi10) memcpy(pi10, p10, sizeof(double) * 10 * n);
    if (T10) memcpy(T10, T, sizeof(double) * 10 * n);
    free(VA);
    free(VB);
    free(Ux);
    free(Uy);
    free(E1);
    free(E2);
    free(phi);
    free(pi);
    free(T);
    free(e);
    free(u);
    free(p10);
}

/* ---- output files (MyEigen.cpp:329-1045) -------------------------------- */

/* bilinear resampling stencil at output point (x, y): lattice index of the
 * lower corner by floor((x + L/2)/a + 1e-10) (MyEigen.cpp:409-412), upper
 * neighbours clamped at N-1, fractions over the OUTPUT spacing ha
 * (MyEigen.cpp:430, 455) */
typedef struct {
    int p[4];
    double fx, fy;
} wstencil;

static wstencil w_stencil(int N, double L, double ha, double x, double y) {
    const double a = L / N;
    const int xpos = (int)floor((x + L / 2.) / a + 0.0000000001);
    const int ypos = (int)floor((y + L / 2.) / a + 0.0000000001);
    const int xup = xpos < N - 1 ? xpos + 1 : xpos;
    const int yup = ypos < N - 1 ? ypos + 1 : ypos;
    wstencil s;
    s.fx = (x - (-L / 2. + a * xpos)) / ha;
    s.fy = (y - (-L / 2. + a * ypos)) / ha;
    s.p[0] = xpos * N + ypos;
    s.p[1] = xup * N + ypos;
    s.p[2] = xpos * N + yup;
    s.p[3] = xup * N + yup;
    return s;
}

/* one interpolated field; a pair of neighbours counts only if both indices
 * are in (0, N*N) (MyEigen.cpp:500-514) */
static double w_interp(const wstencil *s, int nn, const double *f, int absval) {
    double v[4];
    for (int k = 0; k < 4; k++) v[k] = absval ? fabs(f[s->p[k]]) : f[s->p[k]];
    const int ok1 = s->p[0] > 0 && s->p[0] < nn && s->p[1] > 0 && s->p[1] < nn;
    const int ok2 = s->p[2] > 0 && s->p[2] < nn && s->p[3] > 0 && s->p[3] < nn;
    const double x1 = ok1 ? (1 - s->fx) * v[0] + s->fx * v[1] : 0.;
    const double x2 = ok2 ? (1 - s->fx) * v[2] + s->fx * v[3] : 0.;
    return (1. - s->fy) * x1 + s->fy * x2;
}

static const double w_hbarc = 0.1973269718;

int ipgo_write_hydro(const char *path, int N, double L, int sizeOutput,
                     double LOutput, int etaSizeOutput, double detaOutput,
                     int it, double dtau, const double *eps, const double *u4,
                     const double *pi10, double gfactor, double *Etot) {
    const double a = L / N, ha = LOutput / sizeOutput, tau0 = it * dtau * a;
    const int nn = N * N;
    const size_t n = (size_t)nn;
    /* pi10 rows: tautau xx yy etaeta taux tauy taueta xy xeta yeta; printed
     * as tautau taux tauy taueta xx xy xeta yy yeta etaeta */
    static const int order[10] = {0, 4, 5, 6, 1, 7, 8, 2, 9, 3};
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    fprintf(f, "# dummy 1 etamax= %d xmax= %d ymax= %d deta= %g dx= %g dy= %g tau= %g\n",
            etaSizeOutput, sizeOutput, sizeOutput, detaOutput, ha, ha, tau0);
    double etot = 0.;
    for (int ieta = 0; ieta < etaSizeOutput; ieta++) {
        const double eta = -(etaSizeOutput - 1) / 2. * detaOutput + detaOutput * ieta;
        for (int ix = 0; ix < sizeOutput; ix++) {
            for (int iy = 0; iy < sizeOutput; iy++) {
                const double x = -LOutput / 2. + ha * ix;
                const double y = -LOutput / 2. + ha * iy;
                fprintf(f, "%g %g %g ", eta, x, y);
                if (fabs(x) < L / 2. && fabs(y) < L / 2.) {
                    const wstencil s = w_stencil(N, L, ha, x, y);
                    const double e = w_interp(&s, nn, eps, 1);
                    const double ux = w_interp(&s, nn, u4 + n, 0);
                    const double uy = w_interp(&s, nn, u4 + 2 * n, 0);
                    const double ue = w_interp(&s, nn, u4 + 3 * n, 0);
                    /* u^tau from the normalisation (MyEigen.cpp:751-753) */
                    const double ut = sqrt(1. + ux * ux + uy * uy + tau0 * tau0 * ue * ue);
                    const double ew = fabs(w_hbarc * e * gfactor);
                    etot += ew * ha * ha * it * dtau * a;
                    if (ew > 0.0000000001) {
                        fprintf(f, "%g %g %g %g %g", ew, ut, ux, uy, ue);
                        for (int k = 0; k < 10; k++)
                            fprintf(f, " %g", w_interp(&s, nn, pi10 + order[k] * n, 0) * gfactor);
                        fputc('\n', f);
                        continue;
                    }
                }
                fprintf(f, "0 1 0 0 0 0 0 0 0 0 0 0 0 0 0\n");
            }
        }
        fputc('\n', f);
    }
    if (Etot) *Etot = etot;
    return fclose(f) != 0;
}

int ipgo_write_tmunu(const char *path, int N, double L, int sizeOutput,
                     double LOutput, int etaSizeOutput, double detaOutput,
                     int it, double dtau, const double *T10, double gfactor) {
    const double a = L / N, ha = LOutput / sizeOutput, tau0 = it * dtau * a;
    const int nn = N * N;
    const size_t n = (size_t)nn;
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    fprintf(f, "# dummy 1 etamax= %d xmax= %d ymax= %d deta= %g dx= %g dy= %g\n",
            etaSizeOutput, sizeOutput, sizeOutput, detaOutput, ha, ha);
    for (int iy = 0; iy < sizeOutput; iy++) {
        for (int ix = 0; ix < sizeOutput; ix++) {
            const double x = -LOutput / 2. + ha * ix;
            const double y = -LOutput / 2. + ha * iy;
            fprintf(f, "%d %d ", ix, iy);
            if (fabs(x) < L / 2. && fabs(y) < L / 2.) {
                const wstencil s = w_stencil(N, L, ha, x, y);
                double t[10];
                for (int k = 0; k < 10; k++) t[k] = w_interp(&s, nn, T10 + k * n, 0);
                /* T10 rows: tautau xx yy etaeta taux tauy taueta xy xeta yeta;
                 * sign and tau factors of MyEigen.cpp:1017-1027 */
                if (t[0] * gfactor * w_hbarc > 1e-16) {
                    fprintf(f, "%g %g %g %g %g %g %g %g %g %g\n", t[0] * gfactor * w_hbarc,
                            t[1] * gfactor * w_hbarc, t[2] * gfactor * w_hbarc,
                            tau0 * tau0 * t[3] * gfactor * w_hbarc, -t[4] * gfactor * w_hbarc,
                            -t[5] * gfactor * w_hbarc, -tau0 * t[6] * gfactor * w_hbarc,
                            -t[7] * gfactor * w_hbarc, -tau0 * t[9] * gfactor * w_hbarc,
                            -tau0 * t[8] * gfactor * w_hbarc);
                    continue;
                }
            }
            fprintf(f, "%g %g %g 0 0 0 0 0 0 0\n", 1e-16, 1e-16 / 2., 1e-16 / 2.);
        }
        fputc('\n', f);
    }
    return fclose(f) != 0;
}
