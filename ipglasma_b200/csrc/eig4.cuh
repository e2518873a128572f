// Eigenvalues and right eigenvectors of a general real 4x4 matrix, one per
// thread, for the Landau matching of T^mu_nu (replaces gsl_eigen_nonsymmv,
// MyEigen.cpp:78-93).
//
// Method (published algorithms):
//  1. Householder reduction to upper Hessenberg form.
//  2. Francis implicit double-shift QR (Golub & Van Loan, "Matrix
//     Computations", Alg. 7.5.1/7.5.2) on the active unreduced block, with the
//     classical exceptional shift after 10 and 20 sweeps without deflation;
//     eigenvalues are stored at their diagonal-block positions, a complex
//     pair with the positive imaginary part first.
//  3. Eigenvectors as null vectors of (A - lambda I) by Gaussian elimination
//     with complete pivoting (at most three steps, rank tolerance
//     64 eps max|A - lambda I|), last free unknown = 1, back substitution.
//  4. Unit Euclidean norm (the GSL convention), phase chosen so the largest
//     component is real and positive.
#pragma once

#include <cfloat>

namespace ipg {

__device__ __forceinline__ void eig4_hessenberg(double h[4][4]) {
#pragma unroll
    for (int k = 0; k < 2; k++) {
        double v[4] = {0, 0, 0, 0}, nrm2 = 0.0;
#pragma unroll
        for (int i = k + 1; i < 4; i++) nrm2 += h[i][k] * h[i][k];
        if (nrm2 == 0.0) continue;
        const double alpha = (h[k + 1][k] >= 0.0 ? -1.0 : 1.0) * sqrt(nrm2);
#pragma unroll
        for (int i = k + 1; i < 4; i++) v[i] = h[i][k];
        v[k + 1] -= alpha;
        double vtv = 0.0;
#pragma unroll
        for (int i = k + 1; i < 4; i++) vtv += v[i] * v[i];
        if (vtv == 0.0) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            double d = 0.0;
#pragma unroll
            for (int i = k + 1; i < 4; i++) d += v[i] * h[i][j];
            d *= 2.0 / vtv;
#pragma unroll
            for (int i = k + 1; i < 4; i++) h[i][j] -= d * v[i];
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            double d = 0.0;
#pragma unroll
            for (int j = k + 1; j < 4; j++) d += h[i][j] * v[j];
            d *= 2.0 / vtv;
#pragma unroll
            for (int j = k + 1; j < 4; j++) h[i][j] -= d * v[j];
        }
#pragma unroll
        for (int i = k + 2; i < 4; i++) h[i][k] = 0.0;
    }
}

__device__ __forceinline__ int eig4_reflector(int len, const double *x,
                                              double *v, double *beta) {
    double nrm2 = 0.0, vtv = 0.0;
#pragma unroll
    for (int i = 0; i < len; i++) nrm2 += x[i] * x[i];
    if (nrm2 == 0.0) return 0;
    const double alpha = (x[0] >= 0.0 ? -1.0 : 1.0) * sqrt(nrm2);
#pragma unroll
    for (int i = 0; i < len; i++) v[i] = x[i];
    v[0] -= alpha;
#pragma unroll
    for (int i = 0; i < len; i++) vtv += v[i] * v[i];
    if (vtv == 0.0) return 0;
    *beta = 2.0 / vtv;
    return 1;
}

__device__ __forceinline__ void eig4_apply(double h[4][4], int len, int r0,
                                           const double *v, double beta, int lo,
                                           int hi, int cfirst, int rlast) {
#pragma unroll
    for (int j = cfirst; j <= hi; j++) {
        double d = 0.0;
#pragma unroll
        for (int i = 0; i < len; i++) d += v[i] * h[r0 + i][j];
        d *= beta;
#pragma unroll
        for (int i = 0; i < len; i++) h[r0 + i][j] -= d * v[i];
    }
#pragma unroll
    for (int i = lo; i <= rlast; i++) {
        double d = 0.0;
#pragma unroll
        for (int j = 0; j < len; j++) d += h[i][r0 + j] * v[j];
        d *= beta;
#pragma unroll
        for (int j = 0; j < len; j++) h[i][r0 + j] -= d * v[j];
    }
}

// The QR iteration's active block [lo, hi] moves at run time; it is
// dispatched to code specialised for each (lo, hi) a 4 x 4 matrix can have, so
// every index into h, er and ei is a compile-time constant and the matrix
// stays in registers. The arithmetic and its order are those of the
// textbook iteration.

// deflation scan from HI down: the first negligible subdiagonal entry is set
// to zero and bounds the active block from below
template <int HI>
__device__ __forceinline__ int eig4_find_lo(double h[4][4], double anorm) {
    int lo = HI;
    bool found = false;
#pragma unroll
    for (int l = HI; l > 0; l--) {
        if (found) continue;
        double s = fabs(h[l - 1][l - 1]) + fabs(h[l][l]);
        if (s == 0.0) s = anorm;
        if (fabs(h[l][l - 1]) <= DBL_EPSILON * s) {
            h[l][l - 1] = 0.0;
            found = true;
            lo = l;
        } else {
            lo = l - 1;
        }
    }
    return lo;
}

// one Francis double-shift sweep on the unreduced block [LO, HI]
template <int LO, int HI>
__device__ __forceinline__ void eig4_sweep(double h[4][4], int its) {
    double tr, det, x[3], v[3], beta;
    if (its == 10 || its == 20) {
        const double w = fabs(h[HI][HI - 1]) + fabs(h[HI - 1][HI - 2]);
        tr = 1.5 * w;
        det = w * w;
    } else {
        tr = h[HI - 1][HI - 1] + h[HI][HI];
        det = h[HI - 1][HI - 1] * h[HI][HI] - h[HI - 1][HI] * h[HI][HI - 1];
    }
    x[0] = h[LO][LO] * h[LO][LO] + h[LO][LO + 1] * h[LO + 1][LO] - tr * h[LO][LO] + det;
    x[1] = h[LO + 1][LO] * (h[LO][LO] + h[LO + 1][LO + 1] - tr);
    x[2] = h[LO + 1][LO] * h[LO + 2][LO + 1];
#pragma unroll
    for (int k = LO; k <= HI - 2; k++) {
        if (k > LO) {
            x[0] = h[k][k - 1];
            x[1] = h[k + 1][k - 1];
            x[2] = h[k + 2][k - 1];
        }
        if (eig4_reflector(3, x, v, &beta)) {
            const int rlast = (k + 3 <= HI) ? k + 3 : HI;
            eig4_apply(h, 3, k, v, beta, LO, HI, (k > LO ? k - 1 : LO), rlast);
            if (k > LO) {
                h[k + 1][k - 1] = 0.0;
                h[k + 2][k - 1] = 0.0;
            }
        }
    }
    x[0] = h[HI - 1][HI - 2];
    x[1] = h[HI][HI - 2];
    if (eig4_reflector(2, x, v, &beta)) {
        eig4_apply(h, 2, HI - 1, v, beta, LO, HI, HI - 2, HI);
        h[HI][HI - 2] = 0.0;
    }
}

// the eigenvalues of the 2 x 2 block at rows HI-1, HI
template <int HI>
__device__ __forceinline__ void eig4_block2(const double h[4][4], double er[4], double ei[4]) {
    constexpr int LO = HI - 1;
    const double a = h[LO][LO], b = h[LO][HI], c = h[HI][LO], d = h[HI][HI];
    const double half = 0.5 * (a - d);
    const double disc = half * half + b * c;
    if (disc >= 0.0) {
        const double r = sqrt(disc);
        const double zz = half + (half >= 0.0 ? r : -r);
        er[LO] = d + zz;
        er[HI] = (zz != 0.0) ? d - b * c / zz : d + zz;
        ei[LO] = 0.0;
        ei[HI] = 0.0;
    } else {
        const double r = sqrt(-disc);
        er[LO] = d + half;
        er[HI] = d + half;
        ei[LO] = r;
        ei[HI] = -r;
    }
}

// returns the number of sweeps, or -1 when the sweep limit was reached
__device__ __forceinline__ int eig4_qr(double h[4][4], double er[4], double ei[4]) {
    int hi = 3, its = 0, total = 0;
    double anorm = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = (i > 0 ? i - 1 : 0); j < 4; j++) anorm += fabs(h[i][j]);
    while (hi >= 0) {
        const int lo = hi == 3   ? eig4_find_lo<3>(h, anorm)
                       : hi == 2 ? eig4_find_lo<2>(h, anorm)
                       : hi == 1 ? eig4_find_lo<1>(h, anorm)
                                 : 0;
        if (lo == hi) {
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q == hi) {
                    er[q] = h[q][q];
                    ei[q] = 0.0;
                }
            hi -= 1;
            its = 0;
            continue;
        }
        if (lo == hi - 1) {
            if (hi == 3)
                eig4_block2<3>(h, er, ei);
            else if (hi == 2)
                eig4_block2<2>(h, er, ei);
            else
                eig4_block2<1>(h, er, ei);
            hi -= 2;
            its = 0;
            continue;
        }
        if (total >= 120) return -1;
        if (hi == 3 && lo == 0)
            eig4_sweep<0, 3>(h, its);
        else if (hi == 3)
            eig4_sweep<1, 3>(h, its);
        else
            eig4_sweep<0, 2>(h, its);
        its++;
        total++;
    }
    return total;
}

// Every index below is a compile-time constant after unrolling (the pivot
// rows and columns are applied by selects over the candidates, the rank by
// guards), so the 4 x 4 complex work matrix and the vector stay in
// registers instead of local memory; the arithmetic and its order are those
// of plain complete-pivoting elimination.
__device__ __forceinline__ void eig4_nullvec(const double a[16], double lr, double li,
                                             double vr[4], double vi[4]) {
    double mr[4][4], mi[4][4], yr[4], yi[4], scale = 0.0;
    int cp[4], rank = 3;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            mr[i][j] = a[4 * i + j] - (i == j ? lr : 0.0);
            mi[i][j] = (i == j ? -li : 0.0);
            if (fabs(mr[i][j]) + fabs(mi[i][j]) > scale)
                scale = fabs(mr[i][j]) + fabs(mi[i][j]);
        }
    const double tol2 = (64.0 * DBL_EPSILON * scale) * (64.0 * DBL_EPSILON * scale);
#pragma unroll
    for (int j = 0; j < 4; j++) cp[j] = j;
    bool stop = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (stop) continue;
        int pi = k, pj = k;
        double best = -1.0;
#pragma unroll
        for (int i = k; i < 4; i++)
#pragma unroll
            for (int j = k; j < 4; j++) {
                const double m2 = mr[i][j] * mr[i][j] + mi[i][j] * mi[i][j];
                if (m2 > best) {
                    best = m2;
                    pi = i;
                    pj = j;
                }
            }
        if (best <= tol2) {
            rank = k;
            stop = true;
            continue;
        }
        // row k <-> row pi
#pragma unroll
        for (int r = k + 1; r < 4; r++)
            if (pi == r)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    double t = mr[k][j];
                    mr[k][j] = mr[r][j];
                    mr[r][j] = t;
                    t = mi[k][j];
                    mi[k][j] = mi[r][j];
                    mi[r][j] = t;
                }
        // column k <-> column pj, and the unknowns' order with it
#pragma unroll
        for (int c = k + 1; c < 4; c++)
            if (pj == c) {
                const int t = cp[k];
                cp[k] = cp[c];
                cp[c] = t;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    double u = mr[i][k];
                    mr[i][k] = mr[i][c];
                    mr[i][c] = u;
                    u = mi[i][k];
                    mi[i][k] = mi[i][c];
                    mi[i][c] = u;
                }
            }
        const double dr = mr[k][k], di = mi[k][k], den = dr * dr + di * di;
#pragma unroll
        for (int i = k + 1; i < 4; i++) {
            const double fr = (mr[i][k] * dr + mi[i][k] * di) / den;
            const double fi = (mi[i][k] * dr - mr[i][k] * di) / den;
#pragma unroll
            for (int j = k; j < 4; j++) {
                const double pr = fr * mr[k][j] - fi * mi[k][j];
                const double pim = fr * mi[k][j] + fi * mr[k][j];
                mr[i][j] -= pr;
                mi[i][j] -= pim;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        yr[j] = 0.0;
        yi[j] = 0.0;
    }
    yr[3] = 1.0;
#pragma unroll
    for (int i = 2; i >= 0; i--) {
        if (i >= rank) continue;
        double sr = 0.0, si = 0.0;
        const double dr = mr[i][i], di = mi[i][i];
#pragma unroll
        for (int j = i + 1; j < 4; j++) {
            sr += mr[i][j] * yr[j] - mi[i][j] * yi[j];
            si += mr[i][j] * yi[j] + mi[i][j] * yr[j];
        }
        const double den = dr * dr + di * di;
        yr[i] = -(sr * dr + si * di) / den;
        yi[i] = -(si * dr - sr * di) / den;
    }
    // v[cp[j]] = y[j]
#pragma unroll
    for (int t = 0; t < 4; t++) {
        vr[t] = cp[0] == t ? yr[0] : cp[1] == t ? yr[1] : cp[2] == t ? yr[2] : yr[3];
        vi[t] = cp[0] == t ? yi[0] : cp[1] == t ? yi[1] : cp[2] == t ? yi[2] : yi[3];
    }
    double n2 = 0.0, best = -1.0;
    int m = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const double m2 = vr[j] * vr[j] + vi[j] * vi[j];
        n2 += m2;
        if (m2 > best) {
            best = m2;
            m = j;
        }
    }
    const double inv = 1.0 / (sqrt(n2) * sqrt(best));
    const double vrm = m == 0 ? vr[0] : m == 1 ? vr[1] : m == 2 ? vr[2] : vr[3];
    const double vim = m == 0 ? vi[0] : m == 1 ? vi[1] : m == 2 ? vi[2] : vi[3];
    const double pr = vrm * inv, pim = -vim * inv;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const double r = vr[j] * pr - vi[j] * pim;
        const double s = vr[j] * pim + vi[j] * pr;
        vr[j] = r;
        vi[j] = j == m ? 0.0 : s;
    }
}

__device__ __forceinline__ int eig4(const double a[16], double er[4], double ei[4],
                    double vr[16], double vi[16]) {
    double h[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) h[i][j] = a[4 * i + j];
    eig4_hessenberg(h);
    const int status = eig4_qr(h, er, ei);
    if (status < 0) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            er[i] = h[i][i];
            ei[i] = 0.0;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) eig4_nullvec(a, er[i], ei[i], vr + 4 * i, vi + 4 * i);
    return status;
}

}  // namespace ipg
