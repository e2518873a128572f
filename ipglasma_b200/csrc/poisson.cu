// Colour charges -> Poisson solve -> Wilson lines (Init::setV,
// Init.cpp:1678-1849).
//
// The reference transforms each of the 8 colours of a sheet separately with
// FFTW after an fftshift, multiplies by the lattice Green function on the
// centred k-grid and transforms back (FFT.cpp:492-605, Init.cpp:1707-1747).
// For an even N the fftshifts on both sides cancel (cyclic convolution
// commutes with a shift by N/2), so here the multiplier is applied on the
// plain DFT grid with the centred index (p + N/2) mod N, which gives the same
// k~ values. Two real colours are packed into one complex transform (colour
// 2c in the real part, 2c+1 in the imaginary part): the Green function is real
// and even, so the two results separate into the real and imaginary parts of
// the inverse transform.
//
// Kernels per batch of sheets (the work buffer of a batch is sized to stay in
// the 126 MB L2):
//   k_rows_fwd  rho = g sqrt(g2mu2/Ny) xi (read, or Philox in-kernel), row FFTs
//   k_cols      column FFT, Green multiply, inverse column FFT
//   k_rows_inv  inverse row FFTs, 1/N^2
//   k_wilson    per site: V <- exp(-i A_k.t) V over the batch, sheets in order
//               (new * old, Init.cpp:1750-1768)
// The FFTs are the block-level Stockham transforms of fft.cuh.
#include <cstdint>

#include "expm.cuh"
#include "fft.cuh"
#include "fields.cuh"
#include "ipg_internal.h"
#include "philox.cuh"

namespace ipg {

// Green function of the lattice Laplacian on the DFT grid (Init.cpp:1712-1742)
__global__ void k_green(int N, double m_lat, double uvdamp_lat, double *green) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N * N) return;
    const int pi = p / N, pj = p % N;
    const int i = (pi + N / 2) % N, j = (pj + N / 2) % N;  // centred index
    const double kx = 2. * M_PI * (-0.5 + (double)i / (double)N);
    const double ky = 2. * M_PI * (-0.5 + (double)j / (double)N);
    const double kt2 = 4. * (sin(kx / 2.) * sin(kx / 2.) + sin(ky / 2.) * sin(ky / 2.));
    double gk;
    if (m_lat == 0) {
        gk = (kt2 != 0) ? 1. / kt2 : 0.;
    } else {
        gk = (1. / (kt2 + m_lat * m_lat)) * exp(-sqrt(kt2) * uvdamp_lat);
    }
    green[p] = gk;
}

void launch_green(int N, double m_lat, double uvdamp_lat, double *green,
                  cudaStream_t st) {
    const int n = N * N;
    k_green<<<(n + 255) / 256, 256, 0, st>>>(N, m_lat, uvdamp_lat, green);
}

namespace {

// rows of one CTA in the row kernels: a CTA is RPB rows x 4 channels x N/8
template <int LOGN>
constexpr int rows_per_block() {
    return (1 << LOGN) >= 512 ? 1 : ((512 >> LOGN) < (1 << LOGN) ? (512 >> LOGN) : (1 << LOGN));
}
// columns of one CTA in the column kernel
template <int LOGN>
constexpr int cols_per_block() {
    return (1 << LOGN) >= 512 ? 4096 >> LOGN : ((1 << LOGN) < 16 ? (1 << LOGN) : 16);
}

// eight unit normals of one (nucleus, sheet, site) from the counter stream
__device__ __forceinline__ void philox_normals8(uint64_t key, uint32_t nucleus,
                                                uint32_t k, uint32_t pos,
                                                double z[8]) {
    normal4({pos, k, (nucleus << 1) | 0u, 0u}, key, z);
    normal4({pos, k, (nucleus << 1) | 1u, 0u}, key, z + 4);
}

}  // namespace

template <int LOGN>
__global__ void __launch_bounds__(LOGN >= 11 ? 1024 : 512) k_rows_fwd(WilsonArgs w, int k0) {
    constexpr int N = 1 << LOGN, TPS = N / 8, RPB = rows_per_block<LOGN>();
    constexpr int S = fft_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<double> *sm = reinterpret_cast<C<double> *>(smraw);
    const size_t n = (size_t)N * N;
    const int ix0 = blockIdx.x * RPB;
    const int s = blockIdx.y, k = k0 + s;
    const double Nyd = (double)w.Ny;
    const C<double> *tw = reinterpret_cast<const C<double> *>(w.twiddle);
    for (int idx = threadIdx.x; idx < RPB * N; idx += blockDim.x) {
        const int rl = idx / N, j = idx - rl * N;
        const size_t pos = (size_t)(ix0 + rl) * N + j;
        const double amp = w.g * sqrt(w.g2mu2[pos] / Nyd);
        double z[8];
        if (w.xi) {
            const double *src = w.xi + ((size_t)k * n + pos) * 8;
#pragma unroll
            for (int a = 0; a < 8; a++) z[a] = src[a];
        } else {
            philox_normals8(w.philox_key, w.nucleus, (uint32_t)k, (uint32_t)pos, z);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) sm[(rl * 4 + c) * S + fft_pad(j)] = {amp * z[2 * c], amp * z[2 * c + 1]};
    }
    __syncthreads();
    const int seq = threadIdx.x / TPS, t = threadIdx.x - seq * TPS;
    block_fft<LOGN, double, false>(sm + seq * S, t, tw);
    for (int idx = threadIdx.x; idx < RPB * 4 * N; idx += blockDim.x) {
        const int q = idx / N, j = idx - q * N;
        const int rl = q >> 2, c = q & 3;
        const C<double> v = sm[q * S + fft_pad(j)];
        w.work[((size_t)s * 4 + c) * n + (size_t)(ix0 + rl) * N + j] = make_double2(v.r, v.i);
    }
}

template <int LOGN>
__global__ void __launch_bounds__(512) k_cols(WilsonArgs w) {
    constexpr int N = 1 << LOGN, TPS = N / 8, JB = cols_per_block<LOGN>();
    constexpr int S = fft_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<double> *sm = reinterpret_cast<C<double> *>(smraw);
    const size_t n = (size_t)N * N;
    const int jb = blockIdx.x * JB;
    const int c = blockIdx.y, s = blockIdx.z;
    double2 *base = w.work + ((size_t)s * 4 + c) * n;
    const C<double> *tw = reinterpret_cast<const C<double> *>(w.twiddle);
    for (int idx = threadIdx.x; idx < N * JB; idx += blockDim.x) {
        const int i = idx / JB, q = idx - i * JB;
        const double2 v = base[(size_t)i * N + jb + q];
        sm[q * S + fft_pad(i)] = {v.x, v.y};
    }
    __syncthreads();
    const int seq = threadIdx.x / TPS, t = threadIdx.x - seq * TPS;
    block_fft<LOGN, double, false>(sm + seq * S, t, tw);
    for (int idx = threadIdx.x; idx < N * JB; idx += blockDim.x) {
        const int q = idx / N, i = idx - q * N;
        const double gk = w.green[(size_t)i * N + jb + q];
        sm[q * S + fft_pad(i)] = {sm[q * S + fft_pad(i)].r * gk, sm[q * S + fft_pad(i)].i * gk};
    }
    __syncthreads();
    block_fft<LOGN, double, true>(sm + seq * S, t, tw);
    for (int idx = threadIdx.x; idx < N * JB; idx += blockDim.x) {
        const int i = idx / JB, q = idx - i * JB;
        const C<double> v = sm[q * S + fft_pad(i)];
        base[(size_t)i * N + jb + q] = make_double2(v.r, v.i);
    }
}

template <int LOGN>
__global__ void __launch_bounds__(LOGN >= 11 ? 1024 : 512) k_rows_inv(WilsonArgs w) {
    constexpr int N = 1 << LOGN, TPS = N / 8, RPB = rows_per_block<LOGN>();
    constexpr int S = fft_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<double> *sm = reinterpret_cast<C<double> *>(smraw);
    const size_t n = (size_t)N * N;
    const int ix0 = blockIdx.x * RPB;
    const int s = blockIdx.y;
    const C<double> *tw = reinterpret_cast<const C<double> *>(w.twiddle);
    for (int idx = threadIdx.x; idx < RPB * 4 * N; idx += blockDim.x) {
        const int q = idx / N, j = idx - q * N;
        const int rl = q >> 2, c = q & 3;
        const double2 v = w.work[((size_t)s * 4 + c) * n + (size_t)(ix0 + rl) * N + j];
        sm[q * S + fft_pad(j)] = {v.x, v.y};
    }
    __syncthreads();
    const int seq = threadIdx.x / TPS, t = threadIdx.x - seq * TPS;
    block_fft<LOGN, double, true>(sm + seq * S, t, tw);
    const double ntot = (double)n;
    for (int idx = threadIdx.x; idx < RPB * 4 * N; idx += blockDim.x) {
        const int q = idx / N, j = idx - q * N;
        const int rl = q >> 2, c = q & 3;
        const C<double> v = sm[q * S + fft_pad(j)];
        w.work[((size_t)s * 4 + c) * n + (size_t)(ix0 + rl) * N + j] =
            make_double2(v.r / ntot, v.i / ntot);
    }
}

// V <- exp(-i A_k.t) V for the sheets of the batch, in ascending k
__global__ void __launch_bounds__(128) k_wilson(WilsonArgs w, int ns) {
    const size_t n = (size_t)w.N * w.N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    M3<double> V = ld_m3(w.V, pos, n);
    for (int s = 0; s < ns; s++) {
        double in[8];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const double2 v = w.work[((size_t)s * 4 + c) * n + pos];
            in[2 * c] = -v.x;
            in[2 * c + 1] = -v.y;
        }
        const M3<double> e = exp_from_coeff(in);
        V = mul(e, V);
    }
    st_m3(w.V, pos, n, V);
}

template <int LOGN>
static void launch_sheets(const WilsonArgs &w, int k0, int ns, cudaStream_t st) {
    constexpr int N = 1 << LOGN, TPS = N / 8;
    constexpr int RPB = rows_per_block<LOGN>(), JB = cols_per_block<LOGN>();
    const size_t row_smem = sizeof(double2) * RPB * 4 * fft_seq_stride(N);
    const size_t col_smem = sizeof(double2) * JB * fft_seq_stride(N);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_rows_fwd<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)row_smem);
        cudaFuncSetAttribute(k_rows_inv<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)row_smem);
        cudaFuncSetAttribute(k_cols<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)col_smem);
        attr = true;
    }
    k_rows_fwd<LOGN><<<dim3(N / RPB, ns), RPB * 4 * TPS, row_smem, st>>>(w, k0);
    k_cols<LOGN><<<dim3(N / JB, 4, ns), JB * TPS, col_smem, st>>>(w);
    k_rows_inv<LOGN><<<dim3(N / RPB, ns), RPB * 4 * TPS, row_smem, st>>>(w);
    const size_t n = (size_t)N * N;
    k_wilson<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(w, ns);
}

void launch_wilson_sheets(const WilsonArgs &w, int k0, int ns, cudaStream_t st) {
    switch (w.logN) {
        case 3: launch_sheets<3>(w, k0, ns, st); break;
        case 4: launch_sheets<4>(w, k0, ns, st); break;
        case 5: launch_sheets<5>(w, k0, ns, st); break;
        case 6: launch_sheets<6>(w, k0, ns, st); break;
        case 7: launch_sheets<7>(w, k0, ns, st); break;
        case 8: launch_sheets<8>(w, k0, ns, st); break;
        case 9: launch_sheets<9>(w, k0, ns, st); break;
        case 10: launch_sheets<10>(w, k0, ns, st); break;
        case 11: launch_sheets<11>(w, k0, ns, st); break;
        default: break;
    }
}

}  // namespace ipg
