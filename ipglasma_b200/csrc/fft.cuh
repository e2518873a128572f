// Block-level Stockham FFT in shared memory with register butterflies.
//
// Length N = 2^LOGN (8 <= N <= 2048), N/8 threads per sequence, each thread
// holding 8 points in registers per pass. Passes are radix 8 while at least
// three factors of two remain, then one radix-4 or radix-2 pass, so N = 512
// takes 3 shared-memory passes instead of 9 radix-2 passes. The autosort
// (Stockham) indexing keeps input and output in natural order:
//   pass with radix R, sub-length Ns:  for butterfly j < N/R,
//     v[r] = x[j + r N/R] * w^(r (j mod Ns) N/(Ns R)),  v = DFT_R(v),
//     y[(j - j mod Ns) R + j mod Ns + r Ns] = v[r]
// (Govindaraju et al., "High Performance Discrete Fourier Transforms on
// Graphics Processors", SC'08). Twiddles come from a table w^m = exp(-2 pi i
// m/N), m < N, evaluated on the host in double precision. Forward is
// exp(-i...) (FFTW_FORWARD); inverse uses conjugate twiddles; unnormalised.
#pragma once

#include "su3.cuh"

namespace ipg {

template <typename T>
__device__ __forceinline__ C<T> cadd(C<T> a, C<T> b) {
    return {a.r + b.r, a.i + b.i};
}
template <typename T>
__device__ __forceinline__ C<T> csub(C<T> a, C<T> b) {
    return {a.r - b.r, a.i - b.i};
}
// multiply by -i (forward) or +i (inverse)
template <typename T, bool INV>
__device__ __forceinline__ C<T> rot90(C<T> a) {
    return INV ? C<T>{-a.i, a.r} : C<T>{a.i, -a.r};
}

template <typename T, bool INV>
__device__ __forceinline__ void dft2(C<T> &a, C<T> &b) {
    const C<T> t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft4(C<T> &x0, C<T> &x1, C<T> &x2, C<T> &x3) {
    const C<T> a = cadd(x0, x2), b = csub(x0, x2);
    const C<T> c = cadd(x1, x3), d = rot90<T, INV>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft8(C<T> *v) {
    C<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<T, INV>(e0, e1, e2, e3);
    dft4<T, INV>(o0, o1, o2, o3);
    const T h = T(0.70710678118654752440);
    // w8^1 = (1 -+ i)/sqrt2, w8^2 = -+i, w8^3 = (-1 -+ i)/sqrt2
    const C<T> t1 = INV ? C<T>{h * (o1.r - o1.i), h * (o1.r + o1.i)}
                        : C<T>{h * (o1.r + o1.i), h * (o1.i - o1.r)};
    const C<T> t2 = rot90<T, INV>(o2);
    const C<T> t3 = INV ? C<T>{-h * (o3.r + o3.i), h * (o3.r - o3.i)}
                        : C<T>{h * (o3.i - o3.r), -h * (o3.r + o3.i)};
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
}

template <int R, typename T, bool INV>
__device__ __forceinline__ void dft_r(C<T> *v) {
    if constexpr (R == 8) {
        dft8<T, INV>(v);
    } else if constexpr (R == 4) {
        dft4<T, INV>(v[0], v[1], v[2], v[3]);
    } else {
        dft2<T, INV>(v[0], v[1]);
    }
}

// Shared-memory layout of a sequence: point p lives at pad(p) = p + p/8, and
// consecutive sequences are seq_stride(N) = N + N/8 + 1 apart. The padding
// breaks the power-of-two strides of the Stockham stores (8j + r in the
// first pass) and of column tiles, which would otherwise put a whole warp on
// the same shared-memory banks.
__host__ __device__ constexpr int fft_pad(int p) { return p + (p >> 3); }
__host__ __device__ constexpr int fft_seq_stride(int N) { return N + (N >> 3) + 1; }

// One Stockham pass on the sequence in `buf`; t = thread index within the
// sequence (0 .. N/8-1). Caller brackets with __syncthreads().
template <int LOGN, int R, typename T, bool INV>
__device__ __forceinline__ void stockham_pass(C<T> *buf, int t, int Ns,
                                              const C<T> *__restrict__ tw) {
    constexpr int N = 1 << LOGN;
    constexpr int NB = 8 / R;  // butterflies per thread
    C<T> v[8];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * (N / 8);
#pragma unroll
        for (int r = 0; r < R; r++) v[b * R + r] = buf[fft_pad(j + r * (N / R))];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * (N / 8);
        const int k = j & (Ns - 1);
        const int step = k * (N / (Ns * R));
#pragma unroll
        for (int r = 1; r < R; r++) {
            C<T> w = tw[r * step];
            if (INV) w.i = -w.i;
            v[b * R + r] = cmul(v[b * R + r], w);
        }
        dft_r<R, T, INV>(v + b * R);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) buf[fft_pad(base + r * Ns)] = v[b * R + r];
    }
    __syncthreads();
}

// Full transform of the N points in buf (natural order in and out, padded
// layout fft_pad). All threads of the block must call it (it synchronises
// the block).
template <int LOGN, typename T, bool INV>
__device__ __forceinline__ void block_fft(C<T> *buf, int t,
                                          const C<T> *__restrict__ tw) {
    int Ns = 1;
    constexpr int P8 = LOGN / 3, REM = LOGN % 3;
#pragma unroll
    for (int p = 0; p < P8; p++) {
        stockham_pass<LOGN, 8, T, INV>(buf, t, Ns, tw);
        Ns *= 8;
    }
    if constexpr (REM == 2) stockham_pass<LOGN, 4, T, INV>(buf, t, Ns, tw);
    if constexpr (REM == 1) stockham_pass<LOGN, 2, T, INV>(buf, t, Ns, tw);
}

}  // namespace ipg
