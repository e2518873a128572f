// Colour-charge density maps g^2 mu^2(x) of both nuclei from nucleon
// positions, on the device.
//
// The reference builds g^2 mu^2 in Init::setColorChargeDensity
// (Init.cpp:753-1676) from the summed nucleon thicknesses
// T(x) = sum_k exp(-|x - x_k|^2 / (2 B)) / (2 pi B) (Init.cpp:1052-1062, no
// nucleon substructure) and an IP-Sat Q_s(T) table. The table is outside this
// library; the map here is the Q_s ~ sqrt(T) form
//   Q_s^2 = QsMax^2 T / max T,   g^2 mu^2 = Q_s^2 / QsmuRatio^2 a^2 / hbarc^2 / g^2
// in lattice units (the conversion of Init.cpp:1403-1408).
//
// The Gaussian is separable, so T on the N x N grid is a rank-A product:
// per nucleus, tables gx[k][i] = exp(-(x_i - x_k)^2/2B) and gy[k][j] are
// formed once (A N exponentials instead of A N^2), then every site sums A
// products. The maximum is reduced on a fixed grid of blocks (deterministic).
#include <cstdint>

#include "ipg_internal.h"

namespace ipg {

namespace {
constexpr double kHbarcN = 0.1973269718;  // GeV fm
constexpr int kRB = 256, kRG = 296;
}  // namespace

__global__ void k_nucleon_tables(int N, double L, double B, int A, const double *xyz,
                                 double shift, double *gx, double *gy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A * N) return;
    const int k = t / N, i = t - k * N;
    const double a = L / N;
    const double x = -L / 2. + a * i;
    const double dx = x - xyz[3 * k] - shift, dy = x - xyz[3 * k + 1];
    gx[t] = exp(-dx * dx / (2. * B));
    gy[t] = exp(-dy * dy / (2. * B));
}

// T(i, j) = sum_k gx[k][i] gy[k][j] / (2 pi B); per-block maximum into partial
__global__ void __launch_bounds__(kRB) k_thickness(int N, double B, int A, const double *gx,
                                                   const double *gy, double *T, double *partial) {
    const size_t n = (size_t)N * N;
    double m = 0.;
    for (size_t p = (size_t)blockIdx.x * kRB + threadIdx.x; p < n; p += (size_t)kRG * kRB) {
        const int i = (int)(p / N), j = (int)(p % N);
        double s = 0.;
        for (int k = 0; k < A; k++) s += gx[(size_t)k * N + i] * gy[(size_t)k * N + j];
        const double t = s / (2. * M_PI * B);
        T[p] = t;
        m = fmax(m, t);
    }
    __shared__ double sh[kRB / 32];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int w = 0; w < kRB / 32; w++) r = fmax(r, sh[w]);
        partial[blockIdx.x] = r;
    }
}

// every block folds the partial maxima (same order everywhere) and scales
__global__ void __launch_bounds__(kRB) k_g2mu_scale(int N, double factor, const double *partial,
                                                    double *T) {
    __shared__ double tmax;
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int b = 0; b < kRG; b++) r = fmax(r, partial[b]);
        tmax = r;
    }
    __syncthreads();
    const size_t n = (size_t)N * N;
    for (size_t p = (size_t)blockIdx.x * kRB + threadIdx.x; p < n; p += (size_t)kRG * kRB) {
        const double rel = tmax > 0. ? T[p] / tmax : 0.;
        T[p] = factor * rel;
    }
}

void launch_g2mu_from_nucleons(const NucleiArgs &a, cudaStream_t st) {
    const double B = a.BG * kHbarcN * kHbarcN;  // fm^2
    const double lat = a.L / a.N;
    // QsMax^2 / QsmuRatio^2 a^2 / hbarc^2 / g^2 times T / max T
    const double factor = a.QsMax * a.QsMax / (a.QsmuRatio * a.QsmuRatio) * lat * lat /
                          (kHbarcN * kHbarcN) / (a.g * a.g);
    const int t = a.A * a.N;
    k_nucleon_tables<<<(t + 255) / 256, 256, 0, st>>>(a.N, a.L, B, a.A, a.xyz, a.shift, a.gx,
                                                       a.gy);
    k_thickness<<<kRG, kRB, 0, st>>>(a.N, B, a.A, a.gx, a.gy, a.out, a.partial);
    k_g2mu_scale<<<kRG, kRB, 0, st>>>(a.N, factor, a.partial, a.out);
}

}  // namespace ipg
