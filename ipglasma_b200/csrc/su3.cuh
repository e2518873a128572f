// SU(3) / su(3) algebra on 3x3 complex matrices for the lattice kernels.
//
// Semantics follow the reference's Matrix class (Matrix.cpp:100-289,579-604):
// row-major 3x3 complex, conjg() = Hermitian conjugate, prodABconj = A*B^dag,
// prodAconjB = A^dag*B. Everything is templated on the real type so the FP64
// plain form and the FP32 bulk form share one source.
#pragma once

#include <cuda_runtime.h>

namespace ipg {

template <typename T>
struct C {
    T r, i;
};

template <typename T>
struct M3 {
    C<T> m[9];  // row-major
};

// Hermitian 3x3 stored as its 3 real diagonal entries and the upper triangle.
template <typename T>
struct H3 {
    T d0, d1, d2;
    C<T> o01, o02, o12;
};

template <typename T>
__host__ __device__ __forceinline__ C<T> cmul(C<T> a, C<T> b) {
    return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
}
// a * conj(b)
template <typename T>
__host__ __device__ __forceinline__ C<T> cmulc(C<T> a, C<T> b) {
    return {a.r * b.r + a.i * b.i, a.i * b.r - a.r * b.i};
}

template <typename T>
__host__ __device__ __forceinline__ void set_identity(M3<T> &a) {
#pragma unroll
    for (int k = 0; k < 9; k++) a.m[k] = {T(0), T(0)};
    a.m[0].r = a.m[4].r = a.m[8].r = T(1);
}

// Entry (r, k) of A (DAG = false) or of A^dag (DAG = true).
template <bool DAG, typename T>
__host__ __device__ __forceinline__ C<T> entry(const M3<T> &a, int r, int k) {
    if constexpr (DAG)
        return {a.m[3 * k + r].r, -a.m[3 * k + r].i};
    else
        return a.m[3 * r + k];
}

// Z + op(A) op(B), each entry one chain of 12 fused multiply-adds that starts
// from the accumulator, so every real product is one FMA (the negations fold
// into the FMA operands).
template <bool DA, bool DB, typename T>
__host__ __device__ __forceinline__ M3<T> mul_acc(const M3<T> &a, const M3<T> &b,
                                                  const M3<T> &z) {
    M3<T> c;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int s = 0; s < 3; s++) {
            T re = z.m[3 * r + s].r, im = z.m[3 * r + s].i;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const C<T> x = entry<DA>(a, r, k), y = entry<DB>(b, k, s);
                re += x.r * y.r;
                re -= x.i * y.i;
                im += x.r * y.i;
                im += x.i * y.r;
            }
            c.m[3 * r + s] = {re, im};
        }
    return c;
}

// op(A) op(B). RA (RB): the diagonal of A (B) is known to be real (a
// Hermitian operand made by from_h), so the products with its zero imaginary
// parts are left out; the remaining terms keep their order. (Where a zero
// term is dropped the compiler may fuse a different product of the next sum,
// which moves FP64 results at the level of the last bit; the packed FP32
// form fuses explicitly and is unchanged.)
template <bool DA, bool DB, bool RA = false, bool RB = false, typename T>
__host__ __device__ __forceinline__ M3<T> mul_g(const M3<T> &a, const M3<T> &b) {
    M3<T> c;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int s = 0; s < 3; s++) {
            const C<T> x0 = entry<DA>(a, r, 0), y0 = entry<DB>(b, 0, s);
            const bool xr0 = RA && r == 0, yr0 = RB && s == 0;
            T re = x0.r * y0.r, im;
            if (!xr0 && !yr0) re -= x0.i * y0.i;
            if (!yr0) {
                im = x0.r * y0.i;
                if (!xr0) im += x0.i * y0.r;
            } else if (!xr0) {
                im = x0.i * y0.r;
            } else {
                im = T(0);
            }
#pragma unroll
            for (int k = 1; k < 3; k++) {
                const C<T> x = entry<DA>(a, r, k), y = entry<DB>(b, k, s);
                const bool xr = RA && r == k, yr = RB && k == s;
                re += x.r * y.r;
                if (!xr && !yr) re -= x.i * y.i;
                if (!yr) im += x.r * y.i;
                if (!xr) im += x.i * y.r;
            }
            c.m[3 * r + s] = {re, im};
        }
    return c;
}

// C = A * B
template <typename T>
__host__ __device__ __forceinline__ M3<T> mul(const M3<T> &a, const M3<T> &b) {
    return mul_g<false, false>(a, b);
}

// C = A * B^dag
template <typename T>
__host__ __device__ __forceinline__ M3<T> mul_nd(const M3<T> &a,
                                                 const M3<T> &b) {
    return mul_g<false, true>(a, b);
}

// C = A^dag * B
template <typename T>
__host__ __device__ __forceinline__ M3<T> mul_dn(const M3<T> &a,
                                                 const M3<T> &b) {
    return mul_g<true, false>(a, b);
}

template <typename T>
__host__ __device__ __forceinline__ M3<T> dagger(const M3<T> &a) {
    M3<T> c;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int s = 0; s < 3; s++)
            c.m[3 * r + s] = {a.m[3 * s + r].r, -a.m[3 * s + r].i};
    return c;
}

template <typename T>
__host__ __device__ __forceinline__ C<T> trace(const M3<T> &a) {
    return {a.m[0].r + a.m[4].r + a.m[8].r, a.m[0].i + a.m[4].i + a.m[8].i};
}

// Re tr(A B)
template <typename T>
__host__ __device__ __forceinline__ T re_trace_mul(const M3<T> &a,
                                                   const M3<T> &b) {
    T s = T(0);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s += a.m[3 * r + k].r * b.m[3 * k + r].r;
            s -= a.m[3 * r + k].i * b.m[3 * k + r].i;
        }
    return s;
}

// Im tr(A B)
template <typename T>
__host__ __device__ __forceinline__ T im_trace_mul(const M3<T> &a,
                                                   const M3<T> &b) {
    T s = T(0);
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s += a.m[3 * r + k].r * b.m[3 * k + r].i;
            s += a.m[3 * r + k].i * b.m[3 * k + r].r;
        }
    return s;
}

template <typename T>
__host__ __device__ __forceinline__ void add_to(M3<T> &a, const M3<T> &b) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        a.m[k].r += b.m[k].r;
        a.m[k].i += b.m[k].i;
    }
}

template <typename T>
__host__ __device__ __forceinline__ void sub_from(M3<T> &a, const M3<T> &b) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        a.m[k].r -= b.m[k].r;
        a.m[k].i -= b.m[k].i;
    }
}

template <typename T>
__host__ __device__ __forceinline__ M3<T> minus(const M3<T> &a,
                                                const M3<T> &b) {
    M3<T> c;
#pragma unroll
    for (int k = 0; k < 9; k++) c.m[k] = {a.m[k].r - b.m[k].r, a.m[k].i - b.m[k].i};
    return c;
}

template <typename T>
__host__ __device__ __forceinline__ M3<T> scaled(const M3<T> &a, T s) {
    M3<T> c;
#pragma unroll
    for (int k = 0; k < 9; k++) c.m[k] = {a.m[k].r * s, a.m[k].i * s};
    return c;
}

// ---------------------------------------------------------------------------
// Hermitian helpers
// ---------------------------------------------------------------------------

template <typename T>
__host__ __device__ __forceinline__ M3<T> from_h(const H3<T> &h) {
    M3<T> a;
    a.m[0] = {h.d0, T(0)};
    a.m[4] = {h.d1, T(0)};
    a.m[8] = {h.d2, T(0)};
    a.m[1] = h.o01;
    a.m[2] = h.o02;
    a.m[5] = h.o12;
    a.m[3] = {h.o01.r, -h.o01.i};
    a.m[6] = {h.o02.r, -h.o02.i};
    a.m[7] = {h.o12.r, -h.o12.i};
    return a;
}

// Hermitian part read off the diagonal and upper triangle; the caller knows
// the matrix is Hermitian up to rounding.
template <typename T>
__host__ __device__ __forceinline__ H3<T> to_h(const M3<T> &a) {
    H3<T> h;
    h.d0 = a.m[0].r;
    h.d1 = a.m[4].r;
    h.d2 = a.m[8].r;
    h.o01 = a.m[1];
    h.o02 = a.m[2];
    h.o12 = a.m[5];
    return h;
}

// U * H * U^dag for Hermitian H: the result is Hermitian, so only the
// diagonal and the upper triangle are formed.
template <typename T>
__host__ __device__ __forceinline__ H3<T> conj_h(const M3<T> &u,
                                                 const H3<T> &h) {
    M3<T> hm = from_h(h);
    M3<T> w = mul_g<false, false, false, true>(u, hm);  // W = U H
    // (W U^dag)[r][s] = sum_k W[r][k] conj(U[s][k])
    H3<T> out;
    T dr[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        T re = T(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re += w.m[3 * r + k].r * u.m[3 * r + k].r;
            re += w.m[3 * r + k].i * u.m[3 * r + k].i;
        }
        dr[r] = re;
    }
    out.d0 = dr[0];
    out.d1 = dr[1];
    out.d2 = dr[2];
    C<T> o[3];
    const int rs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int r = rs[q][0], s = rs[q][1];
        T re = T(0), im = T(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re += w.m[3 * r + k].r * u.m[3 * s + k].r;
            re += w.m[3 * r + k].i * u.m[3 * s + k].i;
            im += w.m[3 * r + k].i * u.m[3 * s + k].r;
            im -= w.m[3 * r + k].r * u.m[3 * s + k].i;
        }
        o[q] = {re, im};
    }
    out.o01 = o[0];
    out.o02 = o[1];
    out.o12 = o[2];
    return out;
}

// U^dag * H * U
template <typename T>
__host__ __device__ __forceinline__ H3<T> conj_h_dag(const M3<T> &u,
                                                     const H3<T> &h) {
    M3<T> hm = from_h(h);
    M3<T> w = mul_g<false, false, true, false>(hm, u);  // W = H U
    // (U^dag W)[r][s] = sum_k conj(U[k][r]) W[k][s]
    H3<T> out;
    T dr[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        T re = T(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re += u.m[3 * k + r].r * w.m[3 * k + r].r;
            re += u.m[3 * k + r].i * w.m[3 * k + r].i;
        }
        dr[r] = re;
    }
    out.d0 = dr[0];
    out.d1 = dr[1];
    out.d2 = dr[2];
    C<T> o[3];
    const int rs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int r = rs[q][0], s = rs[q][1];
        T re = T(0), im = T(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re += u.m[3 * k + r].r * w.m[3 * k + s].r;
            re += u.m[3 * k + r].i * w.m[3 * k + s].i;
            im += u.m[3 * k + r].r * w.m[3 * k + s].i;
            im -= u.m[3 * k + r].i * w.m[3 * k + s].r;
        }
        o[q] = {re, im};
    }
    out.o01 = o[0];
    out.o02 = o[1];
    out.o12 = o[2];
    return out;
}

template <typename T>
__host__ __device__ __forceinline__ void h_add(H3<T> &a, const H3<T> &b) {
    a.d0 += b.d0;
    a.d1 += b.d1;
    a.d2 += b.d2;
    a.o01.r += b.o01.r;
    a.o01.i += b.o01.i;
    a.o02.r += b.o02.r;
    a.o02.i += b.o02.i;
    a.o12.r += b.o12.r;
    a.o12.i += b.o12.i;
}

// a += s * b
template <typename T>
__host__ __device__ __forceinline__ void h_axpy(H3<T> &a, T s, const H3<T> &b) {
    a.d0 += s * b.d0;
    a.d1 += s * b.d1;
    a.d2 += s * b.d2;
    a.o01.r += s * b.o01.r;
    a.o01.i += s * b.o01.i;
    a.o02.r += s * b.o02.r;
    a.o02.i += s * b.o02.i;
    a.o12.r += s * b.o12.r;
    a.o12.i += s * b.o12.i;
}

// i * [A, B] for Hermitian A, B: Hermitian and traceless.
template <typename T>
__host__ __device__ __forceinline__ H3<T> i_commutator(const H3<T> &a,
                                                       const H3<T> &b) {
    M3<T> am = from_h(a), bm = from_h(b);
    M3<T> ab = mul_g<false, false, true, true>(am, bm);
    // [A,B] = AB - (AB)^dag ; i*[A,B] entries: i*(x - conj(y))
    H3<T> out;
    // diagonal: AB_rr - conj(AB_rr) = 2 i Im(AB_rr); times i -> -2 Im
    out.d0 = -T(2) * ab.m[0].i;
    out.d1 = -T(2) * ab.m[4].i;
    out.d2 = -T(2) * ab.m[8].i;
    // upper (r,s): AB_rs - conj(AB_sr); times i
    const int rs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    C<T> o[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int r = rs[q][0], s = rs[q][1];
        T xr = ab.m[3 * r + s].r - ab.m[3 * s + r].r;
        T xi = ab.m[3 * r + s].i + ab.m[3 * s + r].i;
        o[q] = {-xi, xr};
    }
    out.o01 = o[0];
    out.o02 = o[1];
    out.o12 = o[2];
    return out;
}

// i * (X - X^dag) for a general X: Hermitian.
template <typename T>
__host__ __device__ __forceinline__ H3<T> i_antiherm(const M3<T> &x) {
    H3<T> out;
    out.d0 = -T(2) * x.m[0].i;
    out.d1 = -T(2) * x.m[4].i;
    out.d2 = -T(2) * x.m[8].i;
    const int rs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    C<T> o[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const int r = rs[q][0], s = rs[q][1];
        T xr = x.m[3 * r + s].r - x.m[3 * s + r].r;
        T xi = x.m[3 * r + s].i + x.m[3 * s + r].i;
        o[q] = {-xi, xr};
    }
    out.o01 = o[0];
    out.o02 = o[1];
    out.o12 = o[2];
    return out;
}

template <typename T>
__host__ __device__ __forceinline__ void h_traceless(H3<T> &h) {
    T t = (h.d0 + h.d1 + h.d2) / T(3);
    h.d0 -= t;
    h.d1 -= t;
    h.d2 -= t;
}

template <typename T>
__device__ __forceinline__ void reunitarize(M3<T> &u) {
    // Gram-Schmidt on the first two rows, third row = conj(row0 x row1),
    // the SU(3) completion used by the reference's Matrix::reu (Matrix.h:67-109).
    T n0 = u.m[0].r * u.m[0].r + u.m[0].i * u.m[0].i + u.m[1].r * u.m[1].r +
           u.m[1].i * u.m[1].i + u.m[2].r * u.m[2].r + u.m[2].i * u.m[2].i;
    T inv0 = rsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        u.m[k].r *= inv0;
        u.m[k].i *= inv0;
    }
    // proj = <row0, row1> = sum conj(row0_k) row1_k
    C<T> pr = {T(0), T(0)};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        pr.r += u.m[k].r * u.m[3 + k].r + u.m[k].i * u.m[3 + k].i;
        pr.i += u.m[k].r * u.m[3 + k].i - u.m[k].i * u.m[3 + k].r;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        C<T> t = cmul(pr, u.m[k]);
        u.m[3 + k].r -= t.r;
        u.m[3 + k].i -= t.i;
    }
    T n1 = u.m[3].r * u.m[3].r + u.m[3].i * u.m[3].i + u.m[4].r * u.m[4].r +
           u.m[4].i * u.m[4].i + u.m[5].r * u.m[5].r + u.m[5].i * u.m[5].i;
    T inv1 = rsqrt(n1);
#pragma unroll
    for (int k = 3; k < 6; k++) {
        u.m[k].r *= inv1;
        u.m[k].i *= inv1;
    }
    // row2 = conj(row0 x row1)
    C<T> a0 = u.m[0], a1 = u.m[1], a2 = u.m[2], b0 = u.m[3], b1 = u.m[4],
         b2 = u.m[5];
    C<T> c0 = cmul(a1, b2), c0b = cmul(a2, b1);
    C<T> c1 = cmul(a2, b0), c1b = cmul(a0, b2);
    C<T> c2 = cmul(a0, b1), c2b = cmul(a1, b0);
    u.m[6] = {c0.r - c0b.r, -(c0.i - c0b.i)};
    u.m[7] = {c1.r - c1b.r, -(c1.i - c1b.i)};
    u.m[8] = {c2.r - c2b.r, -(c2.i - c2b.i)};
}

}  // namespace ipg
