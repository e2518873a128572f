// SU(3) exponential exp(i Q_a t^a) in closed form and the Gell-Mann basis.
//
// Follows Matrix::expmCoeff (Matrix.cpp:310-426), the Cayley-Hamilton form of
// Morningstar & Peardon (Phys. Rev. D 69, 054501, 2004): the nine complex
// coefficients (u0, u_a) of exp(iQ) = u0 1 + sum_a u_a t^a, with any NaN
// coefficient set to zero, and Init::getUfromExponent (Init.cpp:3483-3499),
// which returns the identity when |Re u0| < 1e-15.
#pragma once

#include "su3.cuh"

namespace ipg {

// generator constants t^7 = diag(c8, c8, -2 c8) with c8 = 1/(2 sqrt 3)
#define IPG_C8 (1. / (2. * 1.7320508075688772))
#define IPG_INV_SQRT3 (1. / 1.7320508075688772)

__device__ __forceinline__ C<double> cdiv_real(C<double> a, double d) {
    return {a.r / d, a.i / d};
}

__device__ __forceinline__ C<double> cdiv(C<double> a, C<double> b) {
    // Smith's algorithm for a / b
    if (fabs(b.r) >= fabs(b.i)) {
        double r = b.i / b.r, den = b.r + b.i * r;
        return {(a.r + a.i * r) / den, (a.i - a.r * r) / den};
    } else {
        double r = b.r / b.i, den = b.r * r + b.i;
        return {(a.r * r + a.i) / den, (a.i * r - a.r) / den};
    }
}

// coefficients of exp(i Q.t); returns them in u[0..8]
__device__ __forceinline__ void expm_coeff(const double Q[8], C<double> u[9]) {
    const double sqrt3 = sqrt(3.);
    double c0 = sqrt3 * (Q[0] * Q[0] * Q[7] + Q[1] * Q[1] * Q[7] + Q[2] * Q[2] * Q[7]);
    c0 -= Q[7] * Q[7] * Q[7] / sqrt3;
    c0 -= (sqrt3 / 2.) * (Q[3] * Q[3] * Q[7] + Q[4] * Q[4] * Q[7] +
                          Q[5] * Q[5] * Q[7] + Q[6] * Q[6] * Q[7]);
    c0 += 3. * (Q[0] * Q[3] * Q[5] + Q[0] * Q[4] * Q[6] + Q[1] * Q[4] * Q[5] -
                Q[1] * Q[3] * Q[6]);
    c0 += 1.5 * (Q[2] * Q[3] * Q[3] + Q[2] * Q[4] * Q[4] - Q[2] * Q[5] * Q[5] -
                 Q[2] * Q[6] * Q[6]);
    c0 /= 12.;
    double c1 = 0.;
#pragma unroll
    for (int a = 0; a < 8; a++) c1 += Q[a] * Q[a];
    c1 *= 0.25;
    // (c1/3)^{3/2} as t sqrt(t): same value as pow() to rounding, without the
    // log/exp pair
    const double t3 = c1 / 3.;
    const double st3 = sqrt(t3);
    const double c0max = fmax(1e-15, 2. * (t3 * st3));
    const double theta3 = acos(c0 / c0max) / 3.;
    double sth, cth;
    sincos(theta3, &sth, &cth);
    const double uu = st3 * cth;
    const double w = sqrt(c1) * sth;
    double sw, cosw;
    sincos(w, &sw, &cosw);
    const double xi0 = sw / w;
    const double den = 9. * uu * uu - w * w;
    // one reciprocal for the three f's (a NaN or infinity from den = 0
    // propagates as with three divisions and is zeroed below)
    const double rden = 1. / den;
    // e^{-iu} directly, e^{2iu} by the double-angle identities
    double su, cu;
    sincos(uu, &su, &cu);
    const C<double> exp2iu = {(cu - su) * (cu + su), 2. * su * cu};
    const C<double> expmiu = {cu, -su};
    // f0 = (u^2 - w^2) e^{2iu} + e^{-iu} (8 u^2 cos w + 2 i u xi0 (3u^2 + w^2))
    C<double> f0, f1, f2;
    {
        C<double> inner = {8. * uu * uu * cosw, 2. * uu * xi0 * (3. * uu * uu + w * w)};
        C<double> t = cmul(expmiu, inner);
        f0 = {((uu * uu - w * w) * exp2iu.r + t.r) * rden,
              ((uu * uu - w * w) * exp2iu.i + t.i) * rden};
    }
    {
        // f1 = 2u e^{2iu} - e^{-iu} (2u cos w - i (3u^2 - w^2) xi0)
        C<double> inner = {2. * uu * cosw, -(3. * uu * uu - w * w) * xi0};
        C<double> t = cmul(expmiu, inner);
        f1 = {(2. * uu * exp2iu.r - t.r) * rden, (2. * uu * exp2iu.i - t.i) * rden};
    }
    {
        // f2 = e^{2iu} - e^{-iu} (cos w + 3 i u xi0)
        C<double> inner = {cosw, 3. * uu * xi0};
        C<double> t = cmul(expmiu, inner);
        f2 = {(exp2iu.r - t.r) * rden, (exp2iu.i - t.i) * rden};
    }
    C<double> u0 = {f0.r + 2. / 3. * c1 * f2.r, f0.i + 2. / 3. * c1 * f2.i};
    // f1 / (f2 / 2) = f1 conj(f2) * 2 / |f2|^2
    {
        const double r2 = 2. / (f2.r * f2.r + f2.i * f2.i);
        f1 = {(f1.r * f2.r + f1.i * f2.i) * r2, (f1.i * f2.r - f1.r * f2.i) * r2};
    }
    double lin[8];
    lin[0] = Q[3] * Q[5] + Q[4] * Q[6] + 2. / sqrt3 * Q[0] * Q[7];
    lin[1] = 2. * Q[1] * Q[7] / sqrt3 - Q[3] * Q[6] + Q[4] * Q[5];
    lin[2] = 2. * Q[2] * Q[7] / sqrt3 + 0.5 * Q[3] * Q[3] + 0.5 * Q[4] * Q[4] -
             0.5 * Q[5] * Q[5] - 0.5 * Q[6] * Q[6];
    lin[3] = -1. / sqrt3 * Q[3] * Q[7] + Q[0] * Q[5] - Q[1] * Q[6] + Q[2] * Q[3];
    lin[4] = -1. / sqrt3 * Q[4] * Q[7] + Q[0] * Q[6] + Q[1] * Q[5] + Q[2] * Q[4];
    lin[5] = -1. / sqrt3 * Q[5] * Q[7] + Q[0] * Q[3] + Q[1] * Q[4] - Q[2] * Q[5];
    lin[6] = -1. / sqrt3 * Q[6] * Q[7] + Q[0] * Q[4] - Q[1] * Q[3] - Q[2] * Q[6];
    lin[7] = (Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2] - Q[7] * Q[7] -
              0.5 * Q[3] * Q[3] - 0.5 * Q[4] * Q[4] - 0.5 * Q[5] * Q[5] -
              0.5 * Q[6] * Q[6]) /
             sqrt3;
    const C<double> hf2 = {0.5 * f2.r, 0.5 * f2.i};
    u[0] = u0;
#pragma unroll
    for (int a = 0; a < 8; a++) {
        C<double> ua = {f1.r * Q[a] + lin[a], f1.i * Q[a]};
        u[a + 1] = cmul(ua, hf2);
    }
#pragma unroll
    for (int k = 0; k < 9; k++)
        if (isnan(u[k].r) || isnan(u[k].i)) u[k] = {0., 0.};
}

// exp(i in.t) as a 3x3 matrix (Init::getUfromExponent)
__device__ __forceinline__ M3<double> exp_from_coeff(const double in[8]) {
    C<double> u[9];
    expm_coeff(in, u);
    M3<double> r;
    if (fabs(u[0].r) < 1e-15) {
        set_identity(r);
        return r;
    }
    const double c8 = IPG_C8, s3 = IPG_INV_SQRT3;
    // u0*1 + sum_a u_a t^a, t^a = lambda_a / 2 (Group.cpp:111-193)
    r.m[0] = {u[0].r + 0.5 * u[3].r + c8 * u[8].r, u[0].i + 0.5 * u[3].i + c8 * u[8].i};
    r.m[4] = {u[0].r - 0.5 * u[3].r + c8 * u[8].r, u[0].i - 0.5 * u[3].i + c8 * u[8].i};
    r.m[8] = {u[0].r - s3 * u[8].r, u[0].i - s3 * u[8].i};
    // (0,1) = u1/2 - i u2/2 ; (1,0) = u1/2 + i u2/2
    r.m[1] = {0.5 * u[1].r + 0.5 * u[2].i, 0.5 * u[1].i - 0.5 * u[2].r};
    r.m[3] = {0.5 * u[1].r - 0.5 * u[2].i, 0.5 * u[1].i + 0.5 * u[2].r};
    r.m[2] = {0.5 * u[4].r + 0.5 * u[5].i, 0.5 * u[4].i - 0.5 * u[5].r};
    r.m[6] = {0.5 * u[4].r - 0.5 * u[5].i, 0.5 * u[4].i + 0.5 * u[5].r};
    r.m[5] = {0.5 * u[6].r + 0.5 * u[7].i, 0.5 * u[6].i - 0.5 * u[7].r};
    r.m[7] = {0.5 * u[6].r - 0.5 * u[7].i, 0.5 * u[6].i + 0.5 * u[7].r};
    return r;
}

// tr(t^a M) for the Gell-Mann generators, a = 0..7
__device__ __forceinline__ void trace_ta(const M3<double> &m, C<double> out[8]) {
    const double c8 = IPG_C8, s3 = IPG_INV_SQRT3;
    out[0] = {0.5 * m.m[1].r + 0.5 * m.m[3].r, 0.5 * m.m[1].i + 0.5 * m.m[3].i};
    // t1 = (0,1): -i/2, (1,0): +i/2  ->  -i/2 M10 + i/2 M01
    out[1] = {0.5 * m.m[3].i - 0.5 * m.m[1].i, -0.5 * m.m[3].r + 0.5 * m.m[1].r};
    out[2] = {0.5 * m.m[0].r - 0.5 * m.m[4].r, 0.5 * m.m[0].i - 0.5 * m.m[4].i};
    out[3] = {0.5 * m.m[2].r + 0.5 * m.m[6].r, 0.5 * m.m[2].i + 0.5 * m.m[6].i};
    out[4] = {0.5 * m.m[6].i - 0.5 * m.m[2].i, -0.5 * m.m[6].r + 0.5 * m.m[2].r};
    out[5] = {0.5 * m.m[5].r + 0.5 * m.m[7].r, 0.5 * m.m[5].i + 0.5 * m.m[7].i};
    out[6] = {0.5 * m.m[7].i - 0.5 * m.m[5].i, -0.5 * m.m[7].r + 0.5 * m.m[5].r};
    out[7] = {c8 * m.m[0].r + c8 * m.m[4].r - s3 * m.m[8].r,
              c8 * m.m[0].i + c8 * m.m[4].i - s3 * m.m[8].i};
}

// t^a M (left multiplication by a generator)
__device__ __forceinline__ M3<double> ta_mul(int a, const M3<double> &m) {
    M3<double> r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = {0., 0.};
    const double c8 = IPG_C8, s3 = IPG_INV_SQRT3;
    // row i of t^a M = sum_j t^a[i][j] M[j][:]
    auto axpy_row = [&](int dst, C<double> c, int src) {
#pragma unroll
        for (int s = 0; s < 3; s++) {
            C<double> t = cmul(c, m.m[3 * src + s]);
            r.m[3 * dst + s].r += t.r;
            r.m[3 * dst + s].i += t.i;
        }
    };
    switch (a) {
        case 0: axpy_row(0, {0.5, 0}, 1); axpy_row(1, {0.5, 0}, 0); break;
        case 1: axpy_row(0, {0, -0.5}, 1); axpy_row(1, {0, 0.5}, 0); break;
        case 2: axpy_row(0, {0.5, 0}, 0); axpy_row(1, {-0.5, 0}, 1); break;
        case 3: axpy_row(0, {0.5, 0}, 2); axpy_row(2, {0.5, 0}, 0); break;
        case 4: axpy_row(0, {0, -0.5}, 2); axpy_row(2, {0, 0.5}, 0); break;
        case 5: axpy_row(1, {0.5, 0}, 2); axpy_row(2, {0.5, 0}, 1); break;
        case 6: axpy_row(1, {0, -0.5}, 2); axpy_row(2, {0, 0.5}, 1); break;
        default:
            axpy_row(0, {c8, 0}, 0);
            axpy_row(1, {c8, 0}, 1);
            axpy_row(2, {-s3, 0}, 2);
            break;
    }
    return r;
}

}  // namespace ipg
