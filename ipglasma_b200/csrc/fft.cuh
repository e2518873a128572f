// Block-level Stockham FFT in shared memory with register butterflies.
//
// Length N = 2^LOGN (8 <= N <= 2048), N/8 threads per sequence, each thread
// holding 8 points in registers per pass. Passes are radix 8 while at least
// three factors of two remain, then one radix-4 or radix-2 pass, so N = 512
// takes 3 passes instead of 9 radix-2 passes, and only the data exchange
// between consecutive passes goes through shared memory. The autosort
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

// Pass schedule of a length-2^LOGN transform: LOGN/3 radix-8 passes, then
// one radix-4 or radix-2 pass for the remaining factors. Every pass before
// pass p is radix 8, so its sub-length is Ns = 8^p.
template <int LOGN>
struct FftPlan {
    static constexpr int N = 1 << LOGN;
    static constexpr int P8 = LOGN / 3, REM = LOGN % 3;
    static constexpr int PASSES = P8 + (REM ? 1 : 0);
    static constexpr int radix(int p) { return p < P8 ? 8 : (REM == 2 ? 4 : 2); }
    static constexpr int ns(int p) { return 1 << (3 * p); }
};

// The eight points of thread t (0 .. N/8-1) in pass p: butterfly b < 8/R
// works on j = t + b N/8 and reads points j + r N/R into v[b R + r].
template <int LOGN, int PASS, typename T>
__device__ __forceinline__ void pass_load(const C<T> *buf, int t, C<T> v[8]) {
    constexpr int N = 1 << LOGN, R = FftPlan<LOGN>::radix(PASS), NB = 8 / R;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * (N / 8);
#pragma unroll
        for (int r = 0; r < R; r++) v[b * R + r] = buf[fft_pad(j + r * (N / R))];
    }
}

// Twiddle factors of pass p for thread t (none in pass 0, where Ns = 1).
template <int LOGN, int PASS, typename T, bool INV>
__device__ __forceinline__ void pass_twiddles(int t, const C<T> *__restrict__ tw,
                                              C<T> w[8]) {
    constexpr int N = 1 << LOGN, R = FftPlan<LOGN>::radix(PASS), NB = 8 / R;
    constexpr int NS = FftPlan<LOGN>::ns(PASS);
    if constexpr (NS > 1) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int j = t + b * (N / 8);
            const int step = (j & (NS - 1)) * (N / (NS * R));
            if constexpr (R == 8) {
                // one table read, the other six powers by products: the
                // twiddle loads were most of the loads of the row and column
                // kernels, which are load-latency bound (the products are
                // within 1e-15 of the table values, a few ulp)
                C<T> w1 = tw[step];
                if (INV) w1.i = -w1.i;
                const C<T> w2 = cmul(w1, w1), w4 = cmul(w2, w2);
                const C<T> w3 = cmul(w2, w1);
                w[b * R + 1] = w1;
                w[b * R + 2] = w2;
                w[b * R + 3] = w3;
                w[b * R + 4] = w4;
                w[b * R + 5] = cmul(w4, w1);
                w[b * R + 6] = cmul(w4, w2);
                w[b * R + 7] = cmul(w4, w3);
            } else {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C<T> x = tw[r * step];
                    if (INV) x.i = -x.i;
                    w[b * R + r] = x;
                }
            }
        }
    }
}

template <int LOGN, int PASS, typename T, bool INV>
__device__ __forceinline__ void pass_butterflies(C<T> v[8], const C<T> w[8]) {
    constexpr int R = FftPlan<LOGN>::radix(PASS), NB = 8 / R;
    constexpr int NS = FftPlan<LOGN>::ns(PASS);
#pragma unroll
    for (int b = 0; b < NB; b++) {
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) v[b * R + r] = cmul(v[b * R + r], w[b * R + r]);
        }
        dft_r<R, T, INV>(v + b * R);
    }
}

// Stockham output positions: butterfly output r goes to (j - k) R + k + r Ns
// with k = j mod Ns.
template <int LOGN, int PASS, typename T>
__device__ __forceinline__ void pass_store(C<T> *buf, int t, const C<T> v[8]) {
    constexpr int N = 1 << LOGN, R = FftPlan<LOGN>::radix(PASS), NB = 8 / R;
    constexpr int NS = FftPlan<LOGN>::ns(PASS);
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * (N / 8);
        const int k = j & (NS - 1);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) buf[fft_pad(base + r * NS)] = v[b * R + r];
    }
}

template <int LOGN, int PASS, typename T, bool INV>
__device__ __forceinline__ void middle_passes(C<T> *buf, int t,
                                              const C<T> *__restrict__ tw) {
    if constexpr (PASS < FftPlan<LOGN>::PASSES - 1) {
        C<T> v[8], w[8];
        pass_twiddles<LOGN, PASS, T, INV>(t, tw, w);
        pass_load<LOGN, PASS, T>(buf, t, v);
        __syncthreads();
        pass_butterflies<LOGN, PASS, T, INV>(v, w);
        pass_store<LOGN, PASS, T>(buf, t, v);
        __syncthreads();
        middle_passes<LOGN, PASS + 1, T, INV>(buf, t, tw);
    }
}

// Transform of one length-N sequence spread over N/8 threads, with input and
// output in registers: on entry x[m] is point t + m N/8 of the sequence, on
// return x[m] is the transform at frequency t + m N/8. The first pass works on
// x directly (its input points are exactly these) and the last pass leaves
// its outputs in the same slots, so shared memory (buf, padded layout
// fft_pad) carries only the passes in between. All threads of the block call
// it together; buf may be overwritten as soon as it returns.
template <int LOGN, typename T, bool INV>
__device__ __forceinline__ void fft_regs(C<T> x[8], C<T> *buf, int t,
                                         const C<T> *__restrict__ tw) {
    using P = FftPlan<LOGN>;
    constexpr int LAST = P::PASSES - 1;
    // pass 0: radix 8, Ns = 1, v[r] = point t + r N/8 = x[r]
    dft8<T, INV>(x);
    if constexpr (LAST > 0) {
        pass_store<LOGN, 0, T>(buf, t, x);
        __syncthreads();
        middle_passes<LOGN, 1, T, INV>(buf, t, tw);
        C<T> v[8], w[8];
        pass_twiddles<LOGN, LAST, T, INV>(t, tw, w);
        pass_load<LOGN, LAST, T>(buf, t, v);
        __syncthreads();
        pass_butterflies<LOGN, LAST, T, INV>(v, w);
        // in the last pass j < Ns, so output r of butterfly b is frequency
        // j + r N/R = t + (b + r NB) N/8
        constexpr int R = P::radix(LAST), NB = 8 / R;
#pragma unroll
        for (int b = 0; b < NB; b++)
#pragma unroll
            for (int r = 0; r < R; r++) x[b + r * NB] = v[b * R + r];
    }
}

}  // namespace ipg
