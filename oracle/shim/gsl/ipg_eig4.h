/*
 * Eigenvalues and right eigenvectors of a general real 4x4 matrix, used by
 * the oracle's GSL subset in place of gsl_eigen_nonsymmv (TEST
 * INFRASTRUCTURE ONLY).
 *
 * Method (published algorithms, written for this project):
 *  1. Householder reduction of a copy of A to upper Hessenberg form.
 *  2. Francis implicit double-shift QR iteration on the active unreduced
 *     block (Golub & Van Loan, "Matrix Computations", Alg. 7.5.1/7.5.2),
 *     with the classical ad-hoc exceptional shift after 10 and 20 sweeps
 *     without deflation; 1x1 and 2x2 diagonal blocks give the eigenvalues,
 *     stored at their block positions, a complex pair with the positive
 *     imaginary part first.
 *  3. For each eigenvalue lambda, a null vector of (A - lambda I) from
 *     Gaussian elimination with complete pivoting: elimination stops after
 *     three steps or when the remaining block is below a rank tolerance;
 *     the last free unknown is set to 1, the others to 0, and the pivot
 *     unknowns follow by back substitution.
 *  4. Each eigenvector is scaled to unit Euclidean norm and rotated so that
 *     its largest-modulus component is real and positive.
 *
 * GSL fixes only the norm of an eigenvector (GSL manual, gsl_eigen_nonsymmv);
 * the phase convention of step 4 is this project's.
 *
 * Output layout: er[i] + i*ei[i] is eigenvalue i and
 * (vr[4*i+j] + i*vi[4*i+j]), j = 0..3, its eigenvector.
 */
#ifndef IPG_EIG4_H
#define IPG_EIG4_H

#include <float.h>
#include <math.h>

static void ipg_eig4_hessenberg(double h[4][4]) {
    int k, i, j;
    for (k = 0; k < 2; k++) {
        double v[4] = {0, 0, 0, 0}, nrm2 = 0.0, alpha, vtv;
        for (i = k + 1; i < 4; i++) nrm2 += h[i][k] * h[i][k];
        if (nrm2 == 0.0) continue;
        alpha = (h[k + 1][k] >= 0.0 ? -1.0 : 1.0) * sqrt(nrm2);
        for (i = k + 1; i < 4; i++) v[i] = h[i][k];
        v[k + 1] -= alpha;
        vtv = 0.0;
        for (i = k + 1; i < 4; i++) vtv += v[i] * v[i];
        if (vtv == 0.0) continue;
        /* left: rows k+1..3 */
        for (j = 0; j < 4; j++) {
            double d = 0.0;
            for (i = k + 1; i < 4; i++) d += v[i] * h[i][j];
            d *= 2.0 / vtv;
            for (i = k + 1; i < 4; i++) h[i][j] -= d * v[i];
        }
        /* right: columns k+1..3 */
        for (i = 0; i < 4; i++) {
            double d = 0.0;
            for (j = k + 1; j < 4; j++) d += h[i][j] * v[j];
            d *= 2.0 / vtv;
            for (j = k + 1; j < 4; j++) h[i][j] -= d * v[j];
        }
        for (i = k + 2; i < 4; i++) h[i][k] = 0.0;
    }
}

/* Householder reflector P = I - beta v v^T with P x = alpha e1 for a 2- or
 * 3-vector; returns 0 when x is zero (no reflection). */
static int ipg_eig4_reflector(int len, const double *x, double *v,
                              double *beta) {
    double nrm2 = 0.0, alpha, vtv = 0.0;
    int i;
    for (i = 0; i < len; i++) nrm2 += x[i] * x[i];
    if (nrm2 == 0.0) return 0;
    alpha = (x[0] >= 0.0 ? -1.0 : 1.0) * sqrt(nrm2);
    for (i = 0; i < len; i++) v[i] = x[i];
    v[0] -= alpha;
    for (i = 0; i < len; i++) vtv += v[i] * v[i];
    if (vtv == 0.0) return 0;
    *beta = 2.0 / vtv;
    return 1;
}

static void ipg_eig4_apply(double h[4][4], int len, int r0, const double *v,
                           double beta, int lo, int hi, int cfirst,
                           int rlast) {
    int i, j;
    /* left on rows r0..r0+len-1, columns cfirst..hi */
    for (j = cfirst; j <= hi; j++) {
        double d = 0.0;
        for (i = 0; i < len; i++) d += v[i] * h[r0 + i][j];
        d *= beta;
        for (i = 0; i < len; i++) h[r0 + i][j] -= d * v[i];
    }
    /* right on columns r0..r0+len-1, rows lo..rlast */
    for (i = lo; i <= rlast; i++) {
        double d = 0.0;
        for (j = 0; j < len; j++) d += h[i][r0 + j] * v[j];
        d *= beta;
        for (j = 0; j < len; j++) h[i][r0 + j] -= d * v[j];
    }
}

/* eigenvalues of the Hessenberg matrix h (destroyed); returns the number of
 * double-shift sweeps, or -1 if the iteration limit was hit */
static int ipg_eig4_qr(double h[4][4], double er[4], double ei[4]) {
    int hi = 3, its = 0, total = 0, i, j;
    double anorm = 0.0;
    for (i = 0; i < 4; i++)
        for (j = (i > 0 ? i - 1 : 0); j < 4; j++) anorm += fabs(h[i][j]);
    while (hi >= 0) {
        int lo = hi;
        while (lo > 0) {
            double s = fabs(h[lo - 1][lo - 1]) + fabs(h[lo][lo]);
            if (s == 0.0) s = anorm;
            if (fabs(h[lo][lo - 1]) <= DBL_EPSILON * s) {
                h[lo][lo - 1] = 0.0;
                break;
            }
            lo--;
        }
        if (lo == hi) {
            er[hi] = h[hi][hi];
            ei[hi] = 0.0;
            hi -= 1;
            its = 0;
            continue;
        }
        if (lo == hi - 1) {
            double a = h[lo][lo], b = h[lo][hi], c = h[hi][lo], d = h[hi][hi];
            double half = 0.5 * (a - d);
            double disc = half * half + b * c;
            if (disc >= 0.0) {
                double r = sqrt(disc);
                double zz = half + (half >= 0.0 ? r : -r);
                er[lo] = d + zz;
                er[hi] = (zz != 0.0) ? d - b * c / zz : d + zz;
                ei[lo] = 0.0;
                ei[hi] = 0.0;
            } else {
                double r = sqrt(-disc);
                er[lo] = d + half;
                er[hi] = d + half;
                ei[lo] = r;
                ei[hi] = -r;
            }
            hi -= 2;
            its = 0;
            continue;
        }
        if (total >= 120) return -1;
        {
            double tr, det, x[3], v[3], beta;
            int k;
            if (its == 10 || its == 20) {
                double w = fabs(h[hi][hi - 1]) + fabs(h[hi - 1][hi - 2]);
                tr = 1.5 * w;
                det = w * w;
            } else {
                tr = h[hi - 1][hi - 1] + h[hi][hi];
                det = h[hi - 1][hi - 1] * h[hi][hi] - h[hi - 1][hi] * h[hi][hi - 1];
            }
            x[0] = h[lo][lo] * h[lo][lo] + h[lo][lo + 1] * h[lo + 1][lo] -
                   tr * h[lo][lo] + det;
            x[1] = h[lo + 1][lo] * (h[lo][lo] + h[lo + 1][lo + 1] - tr);
            x[2] = h[lo + 1][lo] * h[lo + 2][lo + 1];
            for (k = lo; k <= hi - 2; k++) {
                if (k > lo) {
                    x[0] = h[k][k - 1];
                    x[1] = h[k + 1][k - 1];
                    x[2] = h[k + 2][k - 1];
                }
                if (ipg_eig4_reflector(3, x, v, &beta)) {
                    int rlast = (k + 3 <= hi) ? k + 3 : hi;
                    ipg_eig4_apply(h, 3, k, v, beta, lo, hi,
                                   (k > lo ? k - 1 : lo), rlast);
                    if (k > lo) {
                        h[k + 1][k - 1] = 0.0;
                        h[k + 2][k - 1] = 0.0;
                    }
                }
            }
            x[0] = h[hi - 1][hi - 2];
            x[1] = h[hi][hi - 2];
            if (ipg_eig4_reflector(2, x, v, &beta)) {
                ipg_eig4_apply(h, 2, hi - 1, v, beta, lo, hi, hi - 2, hi);
                h[hi][hi - 2] = 0.0;
            }
            its++;
            total++;
        }
    }
    return total;
}

/* null vector of the complex matrix (A - lambda I) */
static void ipg_eig4_nullvec(const double a[16], double lr, double li,
                             double vr[4], double vi[4]) {
    double mr[4][4], mi[4][4], yr[4], yi[4], scale = 0.0, tol2;
    int cp[4], i, j, k, rank = 3;
    for (i = 0; i < 4; i++)
        for (j = 0; j < 4; j++) {
            mr[i][j] = a[4 * i + j] - (i == j ? lr : 0.0);
            mi[i][j] = (i == j ? -li : 0.0);
            if (fabs(mr[i][j]) + fabs(mi[i][j]) > scale)
                scale = fabs(mr[i][j]) + fabs(mi[i][j]);
        }
    tol2 = (64.0 * DBL_EPSILON * scale) * (64.0 * DBL_EPSILON * scale);
    for (j = 0; j < 4; j++) cp[j] = j;
    for (k = 0; k < 3; k++) {
        int pi = k, pj = k;
        double best = -1.0;
        for (i = k; i < 4; i++)
            for (j = k; j < 4; j++) {
                double m2 = mr[i][j] * mr[i][j] + mi[i][j] * mi[i][j];
                if (m2 > best) {
                    best = m2;
                    pi = i;
                    pj = j;
                }
            }
        if (best <= tol2) {
            rank = k;
            break;
        }
        if (pi != k)
            for (j = 0; j < 4; j++) {
                double t = mr[k][j];
                mr[k][j] = mr[pi][j];
                mr[pi][j] = t;
                t = mi[k][j];
                mi[k][j] = mi[pi][j];
                mi[pi][j] = t;
            }
        if (pj != k) {
            int t = cp[k];
            cp[k] = cp[pj];
            cp[pj] = t;
            for (i = 0; i < 4; i++) {
                double s = mr[i][k];
                mr[i][k] = mr[i][pj];
                mr[i][pj] = s;
                s = mi[i][k];
                mi[i][k] = mi[i][pj];
                mi[i][pj] = s;
            }
        }
        {
            double dr = mr[k][k], di = mi[k][k], den = dr * dr + di * di;
            for (i = k + 1; i < 4; i++) {
                double fr = (mr[i][k] * dr + mi[i][k] * di) / den;
                double fi = (mi[i][k] * dr - mr[i][k] * di) / den;
                for (j = k; j < 4; j++) {
                    mr[i][j] -= fr * mr[k][j] - fi * mi[k][j];
                    mi[i][j] -= fr * mi[k][j] + fi * mr[k][j];
                }
            }
        }
    }
    for (j = 0; j < 4; j++) {
        yr[j] = 0.0;
        yi[j] = 0.0;
    }
    yr[3] = 1.0;
    for (i = rank - 1; i >= 0; i--) {
        double sr = 0.0, si = 0.0, dr = mr[i][i], di = mi[i][i], den;
        for (j = i + 1; j < 4; j++) {
            sr += mr[i][j] * yr[j] - mi[i][j] * yi[j];
            si += mr[i][j] * yi[j] + mi[i][j] * yr[j];
        }
        den = dr * dr + di * di;
        yr[i] = -(sr * dr + si * di) / den;
        yi[i] = -(si * dr - sr * di) / den;
    }
    for (j = 0; j < 4; j++) {
        vr[cp[j]] = yr[j];
        vi[cp[j]] = yi[j];
    }
    {
        double n2 = 0.0, best = -1.0, pr, pim, mod, inv;
        int m = 0;
        for (j = 0; j < 4; j++) {
            double m2 = vr[j] * vr[j] + vi[j] * vi[j];
            n2 += m2;
            if (m2 > best) {
                best = m2;
                m = j;
            }
        }
        mod = sqrt(best);
        inv = 1.0 / (sqrt(n2) * mod);
        /* multiply by conj(v_m)/|v_m| / |v| */
        pr = vr[m] * inv;
        pim = -vi[m] * inv;
        for (j = 0; j < 4; j++) {
            double r = vr[j] * pr - vi[j] * pim;
            double s = vr[j] * pim + vi[j] * pr;
            vr[j] = r;
            vi[j] = s;
        }
        vi[m] = 0.0;
    }
}

/* returns the QR sweep count, or -1 if the QR iteration did not converge */
static int ipg_eig4(const double a[16], double er[4], double ei[4],
                    double vr[16], double vi[16]) {
    double h[4][4];
    int i, j, status;
    for (i = 0; i < 4; i++)
        for (j = 0; j < 4; j++) h[i][j] = a[4 * i + j];
    ipg_eig4_hessenberg(h);
    status = ipg_eig4_qr(h, er, ei);
    if (status < 0) {
        /* leave the unconverged diagonal as the eigenvalue estimate */
        for (i = 0; i < 4; i++) {
            er[i] = h[i][i];
            ei[i] = 0.0;
        }
    }
    for (i = 0; i < 4; i++) ipg_eig4_nullvec(a, er[i], ei[i], vr + 4 * i, vi + 4 * i);
    return status;
}

#endif
