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

// Product of two Hermitian matrices that commute (both polynomials in one
// Hermitian matrix), which is Hermitian: only the real diagonal and the
// upper triangle are formed.
template <typename T>
__device__ __forceinline__ H3<T> hmul_commuting(const H3<T> &a, const H3<T> &b) {
    const M3<T> A = from_h(a), B = from_h(b);
    auto e = [&](int i, int j) {
        C<T> s = cmul(A.m[3 * i], B.m[j]);
        const C<T> s1 = cmul(A.m[3 * i + 1], B.m[3 + j]), s2 = cmul(A.m[3 * i + 2], B.m[6 + j]);
        return C<T>{s.r + s1.r + s2.r, s.i + s1.i + s2.i};
    };
    H3<T> r;
    r.d0 = e(0, 0).r;
    r.d1 = e(1, 1).r;
    r.d2 = e(2, 2).r;
    r.o01 = e(0, 1);
    r.o02 = e(0, 2);
    r.o12 = e(1, 2);
    return r;
}

// s h + c 1
template <typename T>
__device__ __forceinline__ H3<T> h_affine(const H3<T> &h, T s, T c) {
    return {s * h.d0 + c, s * h.d1 + c, s * h.d2 + c, {s * h.o01.r, s * h.o01.i},
            {s * h.o02.r, s * h.o02.i}, {s * h.o12.r, s * h.o12.i}};
}

// exp(i q.t) in FP32 for the FP32 form's Wilson-line factors: scaling and
// squaring with a Taylor series (Moler & Van Loan, "Nineteen dubious ways to
// compute the exponential of a matrix", SIAM Review 45 (2003), method 3).
// H = q.t is scaled by 2^-s until |H|_F = sqrt(sum q^2 / 2) <= 1/2; then
// exp(iH) = C + iS with the even and odd parts
//   C = 1 - H^2/2! + H^4/4! - H^6/6! + H^8/8!,  S = H - H^3/3! + H^5/5! - H^7/7!,
// both Hermitian polynomials in H^2 (Horner, products of commuting Hermitian
// matrices); the remainder is below 0.5^9/9! = 5.4e-9, under FP32 rounding.
// The s squarings are full complex products. Unlike the closed form, this
// stays accurate where eigenvalues of H nearly coincide (weak fields).
__device__ __forceinline__ M3<float> exp_i_taylor_f32(const float q_in[8]) {
    float nrm2 = 0.f;
#pragma unroll
    for (int a = 0; a < 8; a++) nrm2 += q_in[a] * q_in[a];
    nrm2 *= 0.5f;
    int s = 0;
    while (nrm2 > 0.25f && s < 64) {
        nrm2 *= 0.25f;
        s++;
    }
    float q[8];
#pragma unroll
    for (int a = 0; a < 8; a++) q[a] = ldexpf(q_in[a], -s);
    // H = sum_a q_a t^a in the generator convention of exp_from_coeff
    const float c8 = (float)IPG_C8;
    H3<float> h;
    h.d0 = 0.5f * q[2] + c8 * q[7];
    h.d1 = -0.5f * q[2] + c8 * q[7];
    h.d2 = -2.f * c8 * q[7];
    h.o01 = {0.5f * q[0], -0.5f * q[1]};
    h.o02 = {0.5f * q[3], -0.5f * q[4]};
    h.o12 = {0.5f * q[5], -0.5f * q[6]};
    const H3<float> h2 = hmul_commuting(h, h);
    // C = 1 + H2 (-1/2 + H2 (1/24 + H2 (-1/720 + H2 / 40320)))
    H3<float> c = h_affine(h2, 1.f / 40320.f, -1.f / 720.f);
    c = h_affine(hmul_commuting(h2, c), 1.f, 1.f / 24.f);
    c = h_affine(hmul_commuting(h2, c), 1.f, -0.5f);
    c = h_affine(hmul_commuting(h2, c), 1.f, 1.f);
    // S = H (1 + H2 (-1/6 + H2 (1/120 - H2 / 5040)))
    H3<float> r = h_affine(h2, -1.f / 5040.f, 1.f / 120.f);
    r = h_affine(hmul_commuting(h2, r), 1.f, -1.f / 6.f);
    r = h_affine(hmul_commuting(h2, r), 1.f, 1.f);
    const H3<float> sd = hmul_commuting(h, r);
    // E = C + i S entry by entry (C_ji = conj C_ij, S_ji = conj S_ij)
    const M3<float> C = from_h(c), S = from_h(sd);
    M3<float> e;
#pragma unroll
    for (int k = 0; k < 9; k++) e.m[k] = {C.m[k].r - S.m[k].i, C.m[k].i + S.m[k].r};
    for (int k = 0; k < s; k++) e = mul(e, e);
    return e;
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
