// Device layout of the lattice fields (structure of arrays, component-major).
//
// The reference keeps every site as a heap Cell of eight 3x3 matrices with
// aliased slots (Cell.h:155-174). Here each field is a set of planes of n = N*N
// values, so a warp reading one component of 32 neighbouring sites issues one
// coalesced 256-byte (FP64) or 128-byte (FP32) transaction:
//   links Ux, Uy       9 complex planes each (full 3x3; the FP64 plain form
//                      does not reunitarise, so no compression is possible)
//   E1, E2             8 real planes each (traceless Hermitian: d0, d1, then
//                      the upper triangle o01, o02, o12 as re/im pairs)
//   phi, pi            9 real planes each (Hermitian with trace: d0, d1, d2,
//                      then the upper triangle)
// Site index pos = ix * N + iy, as in Lattice.cpp:15-28.
#pragma once

#include "su3.cuh"

namespace ipg {

template <typename T>
struct Links {
    C<T> *x;  // [9][n]
    C<T> *y;  // [9][n]
};

template <typename T>
struct State {
    C<T> *ux, *uy;  // [9][n]
    T *e1, *e2;     // [8][n]
    T *phi, *pi;    // [9][n]
};

template <typename T>
__device__ __forceinline__ M3<T> ld_m3(const C<T> *__restrict__ p, size_t pos,
                                       size_t n) {
    M3<T> a;
#pragma unroll
    for (int k = 0; k < 9; k++) a.m[k] = p[k * n + pos];
    return a;
}

template <typename T>
__device__ __forceinline__ void st_m3(C<T> *__restrict__ p, size_t pos,
                                      size_t n, const M3<T> &a) {
#pragma unroll
    for (int k = 0; k < 9; k++) p[k * n + pos] = a.m[k];
}

template <typename T>
__device__ __forceinline__ H3<T> ld_h(const T *__restrict__ p, size_t pos,
                                      size_t n) {
    H3<T> h;
    h.d0 = p[0 * n + pos];
    h.d1 = p[1 * n + pos];
    h.d2 = p[2 * n + pos];
    h.o01 = {p[3 * n + pos], p[4 * n + pos]};
    h.o02 = {p[5 * n + pos], p[6 * n + pos]};
    h.o12 = {p[7 * n + pos], p[8 * n + pos]};
    return h;
}

template <typename T>
__device__ __forceinline__ void st_h(T *__restrict__ p, size_t pos, size_t n,
                                     const H3<T> &h) {
    p[0 * n + pos] = h.d0;
    p[1 * n + pos] = h.d1;
    p[2 * n + pos] = h.d2;
    p[3 * n + pos] = h.o01.r;
    p[4 * n + pos] = h.o01.i;
    p[5 * n + pos] = h.o02.r;
    p[6 * n + pos] = h.o02.i;
    p[7 * n + pos] = h.o12.r;
    p[8 * n + pos] = h.o12.i;
}

// traceless Hermitian: d2 = -(d0 + d1)
template <typename T>
__device__ __forceinline__ H3<T> ld_h8(const T *__restrict__ p, size_t pos,
                                       size_t n) {
    H3<T> h;
    h.d0 = p[0 * n + pos];
    h.d1 = p[1 * n + pos];
    h.d2 = -(h.d0 + h.d1);
    h.o01 = {p[2 * n + pos], p[3 * n + pos]};
    h.o02 = {p[4 * n + pos], p[5 * n + pos]};
    h.o12 = {p[6 * n + pos], p[7 * n + pos]};
    return h;
}

template <typename T>
__device__ __forceinline__ void st_h8(T *__restrict__ p, size_t pos, size_t n,
                                      const H3<T> &h) {
    p[0 * n + pos] = h.d0;
    p[1 * n + pos] = h.d1;
    p[2 * n + pos] = h.o01.r;
    p[3 * n + pos] = h.o01.i;
    p[4 * n + pos] = h.o02.r;
    p[5 * n + pos] = h.o02.i;
    p[6 * n + pos] = h.o12.r;
    p[7 * n + pos] = h.o12.i;
}

// FP64 views of either form's stored state, for the observables and checks:
// fields widened on load, and links as stored (FP64 form) or formed as
// 1 + W in FP64 from the FP32 form's deviation storage W = U - 1 (the values
// an FP64 copy of the state holds)
__device__ __forceinline__ H3<double> widen_h(const H3<float> &h) {
    return {h.d0, h.d1, h.d2, {h.o01.r, h.o01.i}, {h.o02.r, h.o02.i}, {h.o12.r, h.o12.i}};
}
__device__ __forceinline__ H3<double> h64(const double *p, size_t pos, size_t n) {
    return ld_h(p, pos, n);
}
__device__ __forceinline__ H3<double> h64(const float *p, size_t pos, size_t n) {
    return widen_h(ld_h(p, pos, n));
}
__device__ __forceinline__ H3<double> h8_64(const double *p, size_t pos, size_t n) {
    return ld_h8(p, pos, n);
}
__device__ __forceinline__ H3<double> h8_64(const float *p, size_t pos, size_t n) {
    return widen_h(ld_h8(p, pos, n));
}
__device__ __forceinline__ M3<double> link64(const C<double> *p, size_t pos, size_t n) {
    return ld_m3(p, pos, n);
}
__device__ __forceinline__ M3<double> link64(const C<float> *p, size_t pos, size_t n) {
    const M3<float> w = ld_m3(p, pos, n);
    M3<double> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double shift = (k == 0 || k == 4 || k == 8) ? 1.0 : 0.0;
        u.m[k] = {(double)w.m[k].r + shift, (double)w.m[k].i};
    }
    return u;
}

}  // namespace ipg
