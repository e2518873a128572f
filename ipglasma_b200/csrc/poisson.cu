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
// Kernels per batch of sheets (a work buffer of up to 128 MB per batch: large
// batches give each launch more parallelism):
//   k_rows_fwd  rho = g sqrt(g2mu2/Ny) xi (read, or Philox in-kernel), row FFTs
//   k_cols      column FFT, Green multiply, inverse column FFT
//   k_rows_inv  inverse row FFTs, 1/N^2
//   k_wilson    per site: V <- exp(-i A_k.t) V over the batch, sheets in order
//               (new * old, Init.cpp:1750-1768)
// The FFTs are the block-level Stockham transforms of fft.cuh with input and
// output in registers: thread t of a sequence loads points t + m N/8
// (m = 0..7) straight from global memory, which is the first pass's operand
// order, and the last pass leaves frequencies t + m N/8 in the same slots, so
// they are stored straight back (and, in k_cols, multiplied by the Green
// function on the way from the forward to the inverse transform). For
// fixed m, consecutive t (rows) or consecutive columns (k_cols) are
// consecutive addresses.
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

// rho = amp xi with amp = g sqrt(g2mu2 / Ny) (Init.cpp:1695-1705), evaluated
// once per nucleus instead of once per sheet and colour channel
__global__ void k_amp(int n, double g, double Nyd, const double *g2mu2, double *amp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) amp[p] = g * sqrt(g2mu2[p] / Nyd);
}

// The unit normals k_rows_fwd draws in registers when no noise is given,
// written out as xi[s][pos][a] for sheets k0 .. k0+ns-1: the same counter
// (pos, k, 2 nucleus + a/4, 0), the same words (x, y) for colours a % 4 < 2
// and (z, w) otherwise, the same Box-Muller. One thread per (site, counter
// half), so colours 4h .. 4h+3 of a site come from one thread.
__global__ void k_draw_noise(int N, int k0, int ns, uint64_t key, uint32_t nucleus,
                             double *out) {
    const size_t n = (size_t)N * N;
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 2 * n * (size_t)ns) return;
    const int hc = (int)(gid & 1);
    const size_t rest = gid >> 1;
    const size_t pos = rest % n;
    const int s = (int)(rest / n);
    const U4 r = philox4x32_10({(uint32_t)pos, (uint32_t)(k0 + s), (nucleus << 1) | (uint32_t)hc, 0u},
                               (uint32_t)key, (uint32_t)(key >> 32));
    double z0[2], z1[2];
    box_muller(r.x, r.y, z0);  // channel 2 hc: colours 4 hc, 4 hc + 1
    box_muller(r.z, r.w, z1);  // channel 2 hc + 1: colours 4 hc + 2, 4 hc + 3
    double *o = out + ((size_t)s * n + pos) * 8 + 4 * hc;
    o[0] = z0[0];
    o[1] = z0[1];
    o[2] = z1[0];
    o[3] = z1[1];
}

void launch_draw_noise(int N, int k0, int ns, uint64_t key, uint32_t nucleus, double *out,
                       cudaStream_t st) {
    const size_t threads = 2 * (size_t)N * N * ns;
    k_draw_noise<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(N, k0, ns, key, nucleus,
                                                                     out);
}

__global__ void k_round_to_float(size_t n, const double *in, float *out) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) out[p] = (float)in[p];
}

void launch_round_to_float(size_t n, const double *in, float *out, cudaStream_t st) {
    k_round_to_float<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, in, out);
}

void launch_wilson_amp(const WilsonArgs &w, cudaStream_t st) {
    const int n = w.N * w.N;
    k_amp<<<(n + 255) / 256, 256, 0, st>>>(n, w.g, (double)w.Ny, w.g2mu2, w.amp);
}

namespace {

// packed complex storage of the work buffer: double2 (FP64 transforms) or
// float2 (the FP32 form's transforms, WilsonArgs::fp32)
template <typename R>
struct Store2;
template <>
struct Store2<double> {
    using type = double2;
};
template <>
struct Store2<float> {
    using type = float2;
};
template <typename R>
using store2_t = typename Store2<R>::type;

template <typename R>
__device__ __forceinline__ store2_t<R> *work_of(const WilsonArgs &w) {
    return reinterpret_cast<store2_t<R> *>(w.work);
}
template <typename R>
__device__ __forceinline__ const C<R> *twiddles_of(const WilsonArgs &w) {
    if constexpr (sizeof(R) == 8)
        return reinterpret_cast<const C<R> *>(w.twiddle);
    else
        return reinterpret_cast<const C<R> *>(w.twiddle32);
}

// rows of one CTA in the row kernels: a CTA is RPB rows x 4 channels x N/8
// threads, sequence seq = 4 rl + c
template <int LOGN>
constexpr int rows_per_block() {
    return (1 << LOGN) >= 512 ? 1 : ((512 >> LOGN) < (1 << LOGN) ? (512 >> LOGN) : (1 << LOGN));
}
// columns of one CTA in the column kernel: JB columns x N/8 threads, column
// fastest in the thread index
template <int LOGN>
constexpr int cols_per_block() {
    return (1 << LOGN) >= 512 ? 4096 >> LOGN : ((1 << LOGN) < 16 ? (1 << LOGN) : 16);
}
template <int LOGN>
constexpr int row_threads() {
    return rows_per_block<LOGN>() * 4 * ((1 << LOGN) / 8);
}
template <int LOGN>
constexpr int col_threads() {
    return cols_per_block<LOGN>() * ((1 << LOGN) / 8);
}
// sequence stride of the forward row kernel: there lanes 2i and 2i+1 hold the
// same points of neighbouring sequences (channels 2h, 2h+1), so the stride is
// made 4 mod 8 (in 16-byte units) to put the pair half a bank cycle apart;
// with fft_seq_stride (1 mod 8) lane 2i+1 met lane 2i+2 on the same banks
constexpr int fwd_seq_stride(int N) {
    return fft_seq_stride(N) + ((12 - fft_seq_stride(N) % 8) % 8);
}

}  // namespace

template <int LOGN, typename R>
__global__ void __launch_bounds__(row_threads<LOGN>()) k_rows_fwd(WilsonArgs w, int k0) {
    if (w.skip && *w.skip) return;
    constexpr int N = 1 << LOGN, TPS = N / 8, RPB = rows_per_block<LOGN>();
    constexpr int S = fwd_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<R> *sm = reinterpret_cast<C<R> *>(smraw);
    const size_t n = (size_t)N * N;
    // lanes 2i and 2i+1 hold channels 2h and 2h+1 of the same points (they
    // share one Philox counter); TPS >= 1 sequences of N/8 threads each
    const int half = threadIdx.x & 1, rest = threadIdx.x >> 1;
    const int t = rest % TPS, pair = rest / TPS;  // pair = 2 rl + h
    const int rl = pair >> 1, c = ((pair & 1) << 1) | half;
    const int seq = 4 * rl + c;
    const int s = blockIdx.y, k = k0 + s;
    const size_t row = (size_t)(blockIdx.x * RPB + rl) * N;
    const C<R> *tw = twiddles_of<R>(w);
    C<R> x[8];
    if (w.rho_in) {
        const double2 *in = w.rho_in + ((size_t)s * 4 + c) * n + row + t;
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const double2 v = in[m * TPS];
            x[m] = {(R)v.x, (R)v.y};
        }
    } else {
        double amp[8], z[8][2];
#pragma unroll
        for (int m = 0; m < 8; m++) amp[m] = w.amp[row + t + m * TPS];
        if (w.xi) {
#pragma unroll
            for (int m = 0; m < 8; m++) {
                // colours 2c, 2c+1 of the site
                const size_t pos = row + t + m * TPS;
                const double2 v =
                    *reinterpret_cast<const double2 *>(w.xi + ((size_t)k * n + pos) * 8 + 2 * c);
                z[m][0] = v.x;
                z[m][1] = v.y;
            }
        } else {
            // colours 0-3 come from counter half 0, 4-7 from half 1; channel 2h
            // uses words (x, y) of the counter, channel 2h+1 words (z, w). Each
            // lane of the pair draws the counters of four points and hands the
            // partner's words over
            const uint32_t hc = (uint32_t)(c >> 1);
            uint32_t keep[8][2], give[4][2];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int m = 4 * half + j;
                const U4 r = philox4x32_10(
                    {(uint32_t)(row + t + m * TPS), (uint32_t)k, (w.nucleus << 1) | hc, 0u},
                    (uint32_t)w.philox_key, (uint32_t)(w.philox_key >> 32));
                keep[m][0] = half ? r.z : r.x;
                keep[m][1] = half ? r.w : r.y;
                give[j][0] = half ? r.x : r.z;
                give[j][1] = half ? r.y : r.w;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int m = 4 * (1 - half) + j;
                keep[m][0] = __shfl_xor_sync(0xffffffffu, give[j][0], 1);
                keep[m][1] = __shfl_xor_sync(0xffffffffu, give[j][1], 1);
            }
#pragma unroll
            for (int m = 0; m < 8; m++) box_muller(keep[m][0], keep[m][1], z[m]);
        }
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = {(R)(amp[m] * z[m][0]), (R)(amp[m] * z[m][1])};
    }
    fft_regs<LOGN, R, false>(x, sm + seq * S, t, tw);
    store2_t<R> *out = work_of<R>(w) + ((size_t)s * 4 + c) * n + row + t;
#pragma unroll
    for (int m = 0; m < 8; m++) out[m * TPS] = {x[m].r, x[m].i};
}

// CONV: forward transform, Green multiply, inverse transform; otherwise the
// forward transform only
template <int LOGN, bool CONV = true, typename R = double>
__global__ void __launch_bounds__(col_threads<LOGN>(), 2) k_cols(WilsonArgs w) {
    if (w.skip && *w.skip) return;
    constexpr int N = 1 << LOGN, TPS = N / 8, JB = cols_per_block<LOGN>();
    constexpr int S = fft_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<R> *sm = reinterpret_cast<C<R> *>(smraw);
    const size_t n = (size_t)N * N;
    const int q = threadIdx.x & (JB - 1), t = threadIdx.x / JB;
    const int col = blockIdx.x * JB + q;
    const int c = blockIdx.y, s = blockIdx.z;
    store2_t<R> *base = work_of<R>(w) + ((size_t)s * 4 + c) * n + col;
    const C<R> *tw = twiddles_of<R>(w);
    C<R> x[8];
    R gk[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const store2_t<R> v = base[(size_t)(t + m * TPS) * N];
        x[m] = {v.x, v.y};
    }
    fft_regs<LOGN, R, false>(x, sm + q * S, t, tw);
    if constexpr (CONV) {
        // the Green factors are loaded after the forward transform: that
        // keeps the kernel within 64 registers, two 512-thread blocks per SM
        const R *green = sizeof(R) == 8 ? reinterpret_cast<const R *>(w.green)
                                        : reinterpret_cast<const R *>(w.green32);
#pragma unroll
        for (int m = 0; m < 8; m++) gk[m] = green[(size_t)(t + m * TPS) * N + col];
#pragma unroll
        for (int m = 0; m < 8; m++) x[m] = {x[m].r * gk[m], x[m].i * gk[m]};
        fft_regs<LOGN, R, true>(x, sm + q * S, t, tw);
    }
#pragma unroll
    for (int m = 0; m < 8; m++) base[(size_t)(t + m * TPS) * N] = {x[m].r, x[m].i};
}

template <int LOGN, typename R>
__global__ void __launch_bounds__(row_threads<LOGN>()) k_rows_inv(WilsonArgs w) {
    if (w.skip && *w.skip) return;
    constexpr int N = 1 << LOGN, TPS = N / 8, RPB = rows_per_block<LOGN>();
    constexpr int S = fft_seq_stride(N);
    extern __shared__ __align__(16) unsigned char smraw[];
    C<R> *sm = reinterpret_cast<C<R> *>(smraw);
    const size_t n = (size_t)N * N;
    const int seq = threadIdx.x / TPS, t = threadIdx.x - seq * TPS;
    const int rl = seq >> 2, c = seq & 3;
    const int s = blockIdx.y;
    store2_t<R> *p = work_of<R>(w) + ((size_t)s * 4 + c) * n + (size_t)(blockIdx.x * RPB + rl) * N + t;
    const C<R> *tw = twiddles_of<R>(w);
    C<R> x[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const store2_t<R> v = p[m * TPS];
        x[m] = {v.x, v.y};
    }
    fft_regs<LOGN, R, true>(x, sm + seq * S, t, tw);
    // n = N^2 is a power of two, so multiplying by 1/n is exact and gives
    // the same bits as the reference's division by n
    const R inv_n = R(1) / (R)n;
#pragma unroll
    for (int m = 0; m < 8; m++) p[m * TPS] = {x[m].r * inv_n, x[m].i * inv_n};
}

// V <- exp(-i A_k.t) V for the sheets of the batch, in ascending k. FP64
// transforms (R = double): the reference's closed-form exponential in FP64.
// The FP32 form (R = float): the exponential of the FP32 A in FP32 by
// scaling and squaring (exp_i_taylor_f32), the product accumulated in FP64
// and V reunitarised in FP64 at the end of the batch (the FP32 factors are
// unitary to FP32 rounding).
template <typename R>
__global__ void __launch_bounds__(128) k_wilson(WilsonArgs w, int ns) {
    const size_t n = (size_t)w.N * w.N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const store2_t<R> *work = work_of<R>(w);
    M3<double> V = ld_m3(w.V, pos, n);
    for (int s = 0; s < ns; s++) {
        R in[8];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const store2_t<R> v = work[((size_t)s * 4 + c) * n + pos];
            in[2 * c] = -v.x;
            in[2 * c + 1] = -v.y;
        }
        if constexpr (sizeof(R) == 8) {
            V = mul(exp_from_coeff(in), V);
        } else {
            const M3<float> e32 = exp_i_taylor_f32(in);
            M3<double> e;
#pragma unroll
            for (int k = 0; k < 9; k++) e.m[k] = {(double)e32.m[k].r, (double)e32.m[k].i};
            V = mul(e, V);
        }
    }
    if constexpr (sizeof(R) == 4) reunitarize(V);
    st_m3(w.V, pos, n, V);
}

template <int LOGN, typename R>
static void launch_sheets_t(const WilsonArgs &w, int k0, int ns, cudaStream_t st) {
    constexpr int N = 1 << LOGN;
    constexpr int RPB = rows_per_block<LOGN>(), JB = cols_per_block<LOGN>();
    const size_t row_smem = sizeof(C<R>) * RPB * 4 * fft_seq_stride(N);
    const size_t fwd_smem = sizeof(C<R>) * RPB * 4 * fwd_seq_stride(N);
    const size_t col_smem = sizeof(C<R>) * JB * fft_seq_stride(N);
    // the attribute is per device: set it on every launch (a host-side call
    // without a device round trip)
    cudaFuncSetAttribute(k_rows_fwd<LOGN, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fwd_smem);
    cudaFuncSetAttribute(k_rows_inv<LOGN, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)row_smem);
    cudaFuncSetAttribute(k_cols<LOGN, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)col_smem);
    k_rows_fwd<LOGN, R><<<dim3(N / RPB, ns), row_threads<LOGN>(), fwd_smem, st>>>(w, k0);
    k_cols<LOGN, true, R><<<dim3(N / JB, 4, ns), col_threads<LOGN>(), col_smem, st>>>(w);
    k_rows_inv<LOGN, R><<<dim3(N / RPB, ns), row_threads<LOGN>(), row_smem, st>>>(w);
    const size_t n = (size_t)N * N;
    if (!w.rho_in && !w.no_product)
        k_wilson<R><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(w, ns);
}

template <int LOGN>
static void launch_sheets(const WilsonArgs &w, int k0, int ns, cudaStream_t st) {
    if (w.fp32)
        launch_sheets_t<LOGN, float>(w, k0, ns, st);
    else
        launch_sheets_t<LOGN, double>(w, k0, ns, st);
}

template <int LOGN>
static void launch_forward(const WilsonArgs &w, int ns, cudaStream_t st) {
    constexpr int N = 1 << LOGN;
    constexpr int RPB = rows_per_block<LOGN>(), JB = cols_per_block<LOGN>();
    const size_t fwd_smem = sizeof(double2) * RPB * 4 * fwd_seq_stride(N);
    const size_t col_smem = sizeof(double2) * JB * fft_seq_stride(N);
    cudaFuncSetAttribute(k_rows_fwd<LOGN, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fwd_smem);
    cudaFuncSetAttribute(k_cols<LOGN, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)col_smem);
    k_rows_fwd<LOGN, double><<<dim3(N / RPB, ns), row_threads<LOGN>(), fwd_smem, st>>>(w, 0);
    k_cols<LOGN, false><<<dim3(N / JB, 4, ns), col_threads<LOGN>(), col_smem, st>>>(w);
}

void launch_fft2_forward(const WilsonArgs &w, int ns, cudaStream_t st) {
    switch (w.logN) {
        case 3: launch_forward<3>(w, ns, st); break;
        case 4: launch_forward<4>(w, ns, st); break;
        case 5: launch_forward<5>(w, ns, st); break;
        case 6: launch_forward<6>(w, ns, st); break;
        case 7: launch_forward<7>(w, ns, st); break;
        case 8: launch_forward<8>(w, ns, st); break;
        case 9: launch_forward<9>(w, ns, st); break;
        case 10: launch_forward<10>(w, ns, st); break;
        case 11: launch_forward<11>(w, ns, st); break;
        default: break;
    }
}

// the Wilson-line product of a batch whose A is already in w.work
void launch_wilson_product(const WilsonArgs &w, int ns, cudaStream_t st) {
    const size_t n = (size_t)w.N * w.N;
    if (w.fp32)
        k_wilson<float><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(w, ns);
    else
        k_wilson<double><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(w, ns);
}

void launch_poisson_sheets(const WilsonArgs &w, int ns, cudaStream_t st) {
    // launch_sheets skips the Wilson-line product when rho_in is set
    launch_wilson_sheets(w, 0, ns, st);
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
