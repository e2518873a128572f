// Allocation-free Wilson lines: ipg_wilson_lines_noalloc.
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory pool or allocator hooks, real-time or embedded hosts
// that forbid allocation after start-up, and callers that must not trigger
// the implicit synchronisation a cudaMalloc/cudaFree can cause. The regular
// API (ipg_create) allocates every buffer of an event once; this entry point
// instead uses one fixed, file-scope device array for all of its scratch
// (the FFT work buffer of one sheet, the Green function, the twiddle table
// and the Wilson-line planes) and the caller's own input and output buffers.
//
// Limits and rules of use:
//   - lattices up to IPG_NOALLOC_MAX_N = 256 sites per side (the scratch array
//     is sized for that, about 14 MB, held by every GPU that loads the
//     library until the process exits); larger sizes are rejected;
//   - the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress, with that device current; make that first call
//     before any stream capture;
//   - all calls share the one array and it keeps the last call's contents,
//     so every buffer that must start from a known value is rewritten by the
//     call itself; two calls whose work overlaps on the GPU (different
//     streams, or different host threads on the same device) race on the
//     array and give wrong results: serialise them.
//   - the looked-up address is cached per device index for the life of the
//     process; it assumes the device's primary context is not reset
//     (cudaDeviceReset) between calls.
// The sheets are processed with the same kernels as ipg_init_fields (one
// sheet per batch). The twiddle table is built here on the device with
// sincospi, where ipg_create builds it on the host with cos/sin of 2 pi k/N,
// so the two paths agree to about 1e-12 on the Wilson lines, not bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/ipglasma_b200.h"
#include "ipg_internal.h"

using namespace ipg;

namespace {

constexpr int kMaxN = 256;
constexpr size_t kMaxSites = (size_t)kMaxN * kMaxN;
constexpr int kMaxDevices = 64;
constexpr double kHbarcNoAlloc = 0.1973269718;  // GeV fm

struct NoAllocScratch {
    double2 work[4 * kMaxSites];  // one sheet, 4 packed colour channels
    double2 V[9 * kMaxSites];     // Wilson line, 9 complex planes
    double green[kMaxSites];      // Poisson multiplier
    double amp[kMaxSites];        // charge amplitude g sqrt(g2mu2 / Ny)
    double2 twiddle[kMaxN];       // exp(-2 pi i k / N)
};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices];

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(NoAllocScratch **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<NoAllocScratch *>(g_scratch_addr[dev]);
    return cudaSuccess;
}

__global__ void k_na_twiddle(int N, double2 *tw) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    double s, c;
    sincospi(2.0 * (double)k / (double)N, &s, &c);
    tw[k] = make_double2(c, -s);
}

__global__ void k_na_identity(size_t n, C<double> *V) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
#pragma unroll
    for (int k = 0; k < 9; k++) V[k * n + pos] = {(k == 0 || k == 4 || k == 8) ? 1. : 0., 0.};
}

// planes [9][n] -> per-site 18 doubles (the ABI's matrix layout)
__global__ void k_na_to_sites(size_t n, const C<double> *V, double *out) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C<double> v = V[k * n + pos];
        out[18 * pos + 2 * k] = v.r;
        out[18 * pos + 2 * k + 1] = v.i;
    }
}

}  // namespace

extern "C" ipg_status ipg_wilson_lines_noalloc(int N, int Ny, double L, double g,
                                               double m, double UVdamp,
                                               const double *d_g2mu2,
                                               const double *d_xi, double *d_V,
                                               void *stream) {
    if (N < 8 || N > kMaxN || (N & (N - 1)) != 0) {
        fprintf(stderr,
                "ipg_wilson_lines_noalloc: size %d rejected: it must be a power of two "
                "between 8 and %d (the fixed scratch array holds at most %d x %d sites)\n",
                N, kMaxN, kMaxN, kMaxN);
        return IPG_ERR_BAD_CONFIG;
    }
    if (Ny < 1 || !(L > 0) || !(g > 0) || m < 0 || UVdamp < 0 || !d_g2mu2 || !d_xi || !d_V) {
        fprintf(stderr, "ipg_wilson_lines_noalloc: invalid argument\n");
        return IPG_ERR_BAD_CONFIG;
    }
    if ((uintptr_t)d_xi & 15) {
        // colour pairs are read as 16-byte vectors
        fprintf(stderr, "ipg_wilson_lines_noalloc: d_xi must be 16-byte aligned\n");
        return IPG_ERR_BAD_CONFIG;
    }
    NoAllocScratch *S = nullptr;
    cudaError_t e = scratch_address(&S);
    if (e != cudaSuccess) {
        fprintf(stderr, "ipg_wilson_lines_noalloc: scratch set-up failed: %s\n",
                cudaGetErrorString(e));
        return IPG_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)N * N;
    const double a = L / N;
    int logN = 0;
    while ((1 << logN) < N) logN++;

    k_na_twiddle<<<(N + 127) / 128, 128, 0, st>>>(N, S->twiddle);
    launch_green(N, m * a / kHbarcNoAlloc, UVdamp / a * kHbarcNoAlloc, S->green, st);
    C<double> *V = reinterpret_cast<C<double> *>(S->V);
    k_na_identity<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, V);

    WilsonArgs w;
    w.N = N;
    w.logN = logN;
    w.Ny = Ny;
    w.g = g;
    w.g2mu2 = d_g2mu2;
    w.xi = d_xi;
    w.philox_key = 0;
    w.nucleus = 0;
    w.twiddle = S->twiddle;
    w.green = S->green;
    w.amp = S->amp;
    w.work = S->work;
    w.V = V;
    launch_wilson_amp(w, st);
    for (int k = 0; k < Ny; k++) launch_wilson_sheets(w, k, 1, st);
    k_na_to_sites<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, V, d_V);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "ipg_wilson_lines_noalloc: launch failed: %s\n", cudaGetErrorString(e));
        return IPG_ERR_CUDA;
    }
    return IPG_OK;
}
