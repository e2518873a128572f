// Per-event reductions with FP64 accumulation: Gauss-law violation
// (Evolution::checkGaussLaw, Evolution.cpp:295-364), link unitarity,
// total energy and the eccentricities epsilon_n, Psi_n
// (Evolution::eccentricity, Evolution.cpp:1280-1810, cutoff 0, constant
// coupling), Newton statistics and cell flags.
//
// Every reduction runs on a fixed grid of RG blocks with a grid-stride loop,
// each block writes one partial, and a single thread folds the RG partials in
// order, so results are deterministic (bit-identical run to run).
#include <cstdint>

#include "fields.cuh"
#include "ipg_internal.h"

namespace ipg {

namespace {

constexpr int RB = 256;  // threads per reduction block
constexpr int RG = 296;  // reduction blocks (2 per SM)

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *out) {
    __shared__ double sh[K][RB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.;
        for (int w = 0; w < RB / 32; w++) s += sh[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

__device__ __forceinline__ void block_max(double v, double *out) {
    __shared__ double sh[RB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.;
        for (int w = 0; w < RB / 32; w++) m = fmax(m, sh[w]);
        *out = m;
    }
}

// fold RG partial rows of K values into out[K]; slots in max_mask take the max
template <int K>
__global__ void k_fold(const double *partial, double *out, unsigned max_mask) {
    const int k = threadIdx.x;
    if (k >= K) return;
    const bool mx = (max_mask >> k) & 1u;
    double s = 0.;
    for (int b = 0; b < RG; b++) {
        const double v = partial[(size_t)b * K + k];
        s = mx ? fmax(s, v) : s + v;
    }
    out[k] = s;
}

#define GRID_STRIDE(i, n) \
    for (size_t i = (size_t)blockIdx.x * RB + threadIdx.x; i < (n); i += (size_t)RG * RB)

}  // namespace

// --------------------------------------------------------------------------
// Gauss law: G = UxXm1^dag E1(x-1) UxXm1 - E1 + UyYm1^dag E2(y-1) UyYm1 - E2
//               - i (phi pi - pi phi);  max over sites of |G|^2 / 2
// --------------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(RB) k_gauss(int N, State<S> s, double *partial) {
    const size_t n = (size_t)N * N;
    double val = 0.;
    GRID_STRIDE(pos, n) {
        const int ix = (int)(pos / N), iy = (int)(pos % N);
        const size_t mX = (size_t)max(0, ix - 1) * N + iy;
        const size_t mY = (size_t)ix * N + max(0, iy - 1);
        M3<double> G = mul(mul_dn(link64(s.ux, mX, n), from_h(h8_64(s.e1, mX, n))),
                           link64(s.ux, mX, n));
        sub_from(G, from_h(h8_64(s.e1, pos, n)));
        add_to(G, mul(mul_dn(link64(s.uy, mY, n), from_h(h8_64(s.e2, mY, n))),
                      link64(s.uy, mY, n)));
        sub_from(G, from_h(h8_64(s.e2, pos, n)));
        const M3<double> ph = from_h(h64(s.phi, pos, n)), pi = from_h(h64(s.pi, pos, n));
        const M3<double> c = minus(mul(ph, pi), mul(pi, ph));
#pragma unroll
        for (int k = 0; k < 9; k++) {  // - i c
            G.m[k].r += c.m[k].i;
            G.m[k].i -= c.m[k].r;
        }
        double sq = 0.;
#pragma unroll
        for (int k = 0; k < 9; k++) sq += G.m[k].r * G.m[k].r + G.m[k].i * G.m[k].i;
        val = fmax(val, 0.5 * sq);
    }
    block_max(val, partial + blockIdx.x);
}

template <typename S>
void launch_gauss_law(int N, const State<S> &s, double *d_partial, double *d_out,
                      cudaStream_t st) {
    k_gauss<S><<<RG, RB, 0, st>>>(N, s, d_partial);
    k_fold<1><<<1, 32, 0, st>>>(d_partial, d_out, 1u);
}
template void launch_gauss_law<double>(int, const State<double> &, double *, double *,
                                       cudaStream_t);
template void launch_gauss_law<float>(int, const State<float> &, double *, double *,
                                      cudaStream_t);

// --------------------------------------------------------------------------
// max over links of the largest |(U^dag U - 1)_ij|
// --------------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(RB) k_unitarity(int N, const C<S> *ux, const C<S> *uy,
                                                  double *partial) {
    const size_t n = (size_t)N * N;
    double val = 0.;
    GRID_STRIDE(pos, n) {
        for (int d = 0; d < 2; d++) {
            const M3<double> u = link64(d ? uy : ux, pos, n);
            M3<double> p = mul_dn(u, u);
            p.m[0].r -= 1.;
            p.m[4].r -= 1.;
            p.m[8].r -= 1.;
#pragma unroll
            for (int k = 0; k < 9; k++)
                val = fmax(val, sqrt(p.m[k].r * p.m[k].r + p.m[k].i * p.m[k].i));
        }
    }
    block_max(val, partial + blockIdx.x);
}

template <typename S>
void launch_unitarity(int N, const C<S> *ux, const C<S> *uy, double *d_partial,
                      double *d_out, cudaStream_t st) {
    k_unitarity<S><<<RG, RB, 0, st>>>(N, ux, uy, d_partial);
    k_fold<1><<<1, 32, 0, st>>>(d_partial, d_out, 1u);
}
template void launch_unitarity<double>(int, const C<double> *, const C<double> *, double *,
                                       double *, cudaStream_t);
template void launch_unitarity<float>(int, const C<float> *, const C<float> *, double *,
                                      double *, cudaStream_t);

// --------------------------------------------------------------------------
// eccentricities
// --------------------------------------------------------------------------
// pass 1: sum x w, y w, w, T^tautau, eps   (w = eps u^tau where eps >= 0)
__global__ void __launch_bounds__(RB) k_ecc1(int N, double L, double a, const double *eps,
                                             const double *utau, const double *Ttt,
                                             double *partial) {
    const size_t n = (size_t)N * N;
    double v[5] = {0., 0., 0., 0., 0.};
    GRID_STRIDE(pos, n) {
        const int ix = (int)(pos / N), iy = (int)(pos % N);
        const double x = -L / 2. + a * ix, y = -L / 2. + a * iy;
        const double e = eps[pos];
        const double w = (e < 0.) ? 0. : e * utau[pos];
        v[0] += x * w;
        v[1] += y * w;
        v[2] += w;
        v[3] += Ttt[pos];
        v[4] += e;
    }
    block_sum<5>(v, partial + (size_t)blockIdx.x * 5);
}

// pass 2 over [2, N-2)^2 about the centroid: r^n, r^n cos(n phi), r^n sin(n phi)
// in the reference's choice of powers (avr1 and the n = 1 moments use r^3)
__global__ void __launch_bounds__(RB) k_ecc2(int N, double L, double a, const double *eps,
                                             const double *utau, const double *cent,
                                             double *partial) {
    const size_t n = (size_t)N * N;
    double v[18];
#pragma unroll
    for (int k = 0; k < 18; k++) v[k] = 0.;
    const double avx = cent[0] / cent[2], avy = cent[1] / cent[2];
    GRID_STRIDE(pos, n) {
        const int ix = (int)(pos / N), iy = (int)(pos % N);
        if (ix < 2 || ix >= N - 2 || iy < 2 || iy >= N - 2) continue;
        const double x = -L / 2. + a * ix - avx, y = -L / 2. + a * iy - avy;
        double phiA;
        if (x >= 0) {
            phiA = atan(y / x);
            if (x == 0) phiA = (y >= 0) ? M_PI / 2. : 3. * M_PI / 2.;
        } else {
            phiA = atan(y / x) + M_PI;
        }
        const double e = eps[pos];
        const double w = (e < 0.) ? 0. : e * utau[pos];
        const double r = sqrt(x * x + y * y);
        const double r2 = r * r, r3 = r * r * r, r4 = r * r * r * r;
        const double r5 = r * r * r * r * r, r6 = r * r * r * r * r * r;
        // 0..5: avr1 avrSq avr3 avr4 avr5 avr6
        v[0] += r3 * w;
        v[1] += r2 * w;
        v[2] += r3 * w;
        v[3] += r4 * w;
        v[4] += r5 * w;
        v[5] += r6 * w;
        // 6..17: cos/sin moments for n = 1..6
        v[6] += r3 * cos(phiA) * w;
        v[7] += r3 * sin(phiA) * w;
        v[8] += r2 * cos(2. * phiA) * w;
        v[9] += r2 * sin(2. * phiA) * w;
        v[10] += r3 * cos(3. * phiA) * w;
        v[11] += r3 * sin(3. * phiA) * w;
        v[12] += r4 * cos(4. * phiA) * w;
        v[13] += r4 * sin(4. * phiA) * w;
        v[14] += r5 * cos(5. * phiA) * w;
        v[15] += r5 * sin(5. * phiA) * w;
        v[16] += r6 * cos(6. * phiA) * w;
        v[17] += r6 * sin(6. * phiA) * w;
    }
    block_sum<18>(v, partial + (size_t)blockIdx.x * 18);
}

// pass 3 (Evolution.cpp:1346-1368 and 1669-1790 with cutoff 0): over all
// cells about the all-cell centroid, sum x^2 w, y^2 w, w; over the cells
// with eps >= 0, their count, sum eps and sum g2mu2A g2mu2B; over
// [2, N-2)^2, the largest ix + 1 with w > 0 on the row iy = N/2 + yshift and
// the largest iy + 1 on the column ix = N/2 + xshift (the reference keeps
// the last such cell of its loop, Evolution.cpp:1631-1636)
__global__ void __launch_bounds__(RB) k_ecc3(int N, double L, double a, const double *eps,
                                             const double *utau, const double *g2A,
                                             const double *g2B, const double *cent,
                                             double *partial) {
    const size_t n = (size_t)N * N;
    double v[6] = {0., 0., 0., 0., 0., 0.};
    double row_ix = 0., col_iy = 0.;
    const double avx = cent[0] / cent[2], avy = cent[1] / cent[2];
    const int xshift = (int)floor(avx / a + 0.00000000001);
    const int yshift = (int)floor(avy / a + 0.00000000001);
    GRID_STRIDE(pos, n) {
        const int ix = (int)(pos / N), iy = (int)(pos % N);
        const double x = -L / 2. + a * ix - avx, y = -L / 2. + a * iy - avy;
        const double e = eps[pos];
        const double w = (e < 0.) ? 0. : e * utau[pos];
        v[0] += x * x * w;
        v[1] += y * y * w;
        v[2] += w;
        if (!(e < 0.)) {
            v[3] += 1.;
            v[4] += e;
            v[5] += g2A[pos] * g2B[pos];
        }
        if (ix >= 2 && ix < N - 2 && iy >= 2 && iy < N - 2 && w > 0.) {
            if (iy == N / 2 + yshift) row_ix = fmax(row_ix, ix + 1.);
            if (ix == N / 2 + xshift) col_iy = fmax(col_iy, iy + 1.);
        }
    }
    block_sum<6>(v, partial + (size_t)blockIdx.x * 8);
    block_max(row_ix, partial + (size_t)blockIdx.x * 8 + 6);
    __syncthreads();  // block_max's shared slots are reused by the next call
    block_max(col_iy, partial + (size_t)blockIdx.x * 8 + 7);
}

void launch_eccentricity_extras(int N, double L, double a, const double *eps,
                                const double *utau, const double *g2A, const double *g2B,
                                const double *d_sums1, double *d_partial, double *d_out,
                                cudaStream_t st) {
    k_ecc3<<<RG, RB, 0, st>>>(N, L, a, eps, utau, g2A, g2B, d_sums1, d_partial);
    k_fold<8><<<1, 32, 0, st>>>(d_partial, d_out, (1u << 6) | (1u << 7));
}

void launch_eccentricity(int N, double L, double a, const double *eps,
                         const double *utau, const double *Ttt,
                         double *d_partial, double *d_sums1,
                         double *d_sums2, cudaStream_t st) {
    k_ecc1<<<RG, RB, 0, st>>>(N, L, a, eps, utau, Ttt, d_partial);
    k_fold<5><<<1, 32, 0, st>>>(d_partial, d_sums1, 0u);
    k_ecc2<<<RG, RB, 0, st>>>(N, L, a, eps, utau, d_sums1, d_partial);
    k_fold<18><<<1, 32, 0, st>>>(d_partial, d_sums2, 0u);
}

// --------------------------------------------------------------------------
// Newton statistics: out = {max iterations, sum of iterations, links that
// restarted, links that failed}
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(RB) k_newton_stats(size_t links, const int *iters,
                                                     const int *status, double *partial) {
    double mx = 0.;
    double v[3] = {0., 0., 0.};
    GRID_STRIDE(k, links) {
        mx = fmax(mx, (double)iters[k]);
        v[0] += iters[k];
        v[1] += status[k] >= 1;
        v[2] += status[k] == 2;
    }
    block_max(mx, partial + (size_t)blockIdx.x * 4);
    block_sum<3>(v, partial + (size_t)blockIdx.x * 4 + 1);
}

void launch_newton_stats(size_t links, const int *iters, const int *status,
                         double *d_partial, double *d_out, cudaStream_t st) {
    k_newton_stats<<<RG, RB, 0, st>>>(links, iters, status, d_partial);
    k_fold<4><<<1, 32, 0, st>>>(d_partial, d_out, 1u);
}

// cells with found == 0 and cells with non-finite e
__global__ void __launch_bounds__(RB) k_cell_flags(size_t n, const int *found,
                                                   const double *eps, double *partial) {
    double v[2] = {0., 0.};
    GRID_STRIDE(k, n) {
        v[0] += found[k] == 0;
        v[1] += !isfinite(eps[k]);
    }
    block_sum<2>(v, partial + (size_t)blockIdx.x * 2);
}

void launch_cell_flags(size_t n, const int *found, const double *eps,
                       double *d_partial, double *d_out, cudaStream_t st) {
    k_cell_flags<<<RG, RB, 0, st>>>(n, found, eps, d_partial);
    k_fold<2><<<1, 32, 0, st>>>(d_partial, d_out, 0u);
}

// --------------------------------------------------------------------------
// FP32 <-> FP64 state conversion
// --------------------------------------------------------------------------
// The FP32 form stores links as their deviation from the identity, W = U - 1
// (see k_leapfrog_dev): down-conversion forms U - 1 in FP64 before rounding,
// up-conversion adds the identity back in FP64 (exact).
template <typename S, typename D>
__global__ void k_convert(size_t n, State<S> src, State<D> dst) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const bool down = sizeof(D) < sizeof(S);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const bool diag = (k == 0 || k == 4 || k == 8);
        const double shift = diag ? (down ? -1.0 : 1.0) : 0.0;
        dst.ux[k * n + pos] = {(D)((double)src.ux[k * n + pos].r + shift),
                               (D)src.ux[k * n + pos].i};
        dst.uy[k * n + pos] = {(D)((double)src.uy[k * n + pos].r + shift),
                               (D)src.uy[k * n + pos].i};
        dst.phi[k * n + pos] = (D)src.phi[k * n + pos];
        dst.pi[k * n + pos] = (D)src.pi[k * n + pos];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
        dst.e1[k * n + pos] = (D)src.e1[k * n + pos];
        dst.e2[k * n + pos] = (D)src.e2[k * n + pos];
    }
}

template <typename T>
void launch_convert_state(size_t n, const State<T> &src, State<double> &dst,
                          cudaStream_t st) {
    k_convert<T, double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, src, dst);
}

template <typename T>
void launch_convert_state_down(size_t n, const State<double> &src,
                               State<T> &dst, cudaStream_t st) {
    k_convert<double, T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, src, dst);
}

template void launch_convert_state<float>(size_t, const State<float> &,
                                          State<double> &, cudaStream_t);
template void launch_convert_state_down<float>(size_t, const State<double> &,
                                               State<float> &, cudaStream_t);

}  // namespace ipg
