// C ABI (include/ipglasma_b200.h): context, buffers, schedule.
//
// One context is one event of one lattice size. Device memory per event is
// allocated once at ipg_create and reused by every call; nothing on the hot
// path allocates.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <map>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ipglasma_b200.h"
#include "ipg_internal.h"
#include "writers.h"

using namespace ipg;

namespace {
constexpr double kHbarc = 0.1973269718;  // GeV fm (Phys_consts.h)
}

struct ipg_ctx {
    ipg_config cfg{};
    int N = 0, logN = 0;
    size_t n = 0;
    double a = 0, dtau = 0, m_lat = 0, uv_lat = 0;
    int itmax = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Wilson-line stage: the exponential products of a sheet batch run on
    // stream_v while the next batch's Poisson transforms run on stream, into
    // the other of two work buffers (work, work2)
    cudaStream_t stream_v = nullptr;
    cudaEvent_t ev_fft[2] = {nullptr, nullptr}, ev_prod[2] = {nullptr, nullptr};
    cudaEvent_t ev_nuc_fork = nullptr, ev_nuc_join = nullptr;  // input adjoint, two nuclei
    // ipg_get_observables_async: the copies run on stream_copy after
    // ev_obs_ready; the next observables stage waits for ev_obs_copied
    cudaStream_t stream_copy = nullptr;
    cudaEvent_t ev_obs_ready = nullptr, ev_obs_copied = nullptr;
    bool obs_copy_pending = false;
    std::string err;
    long long launches = 0;

    // inputs
    double *g2mu2A = nullptr, *g2mu2B = nullptr;
    double *xiA_own = nullptr, *xiB_own = nullptr;
    const double *xiA = nullptr, *xiB = nullptr;
    bool have_g2mu = false, have_noise = false, device_noise = false;

    // initial-condition scratch
    double2 *twiddle = nullptr;
    double *green = nullptr;
    // FP32 contexts: the Poisson transforms' twiddles and Green function in
    // FP32 (the transforms of the FP32 form run in FP32)
    float2 *twiddle32 = nullptr;
    float *green32 = nullptr;
    double *amp = nullptr;
    double2 *work = nullptr, *work2 = nullptr;
    double *nuc_xyz = nullptr, *nuc_gx = nullptr, *nuc_gy = nullptr;  // ipg_set_nuclei
    struct {  // ipg_set_nuclei_ipsat (allocated by its first call)
        double *TA = nullptr, *TB = nullptr, *yB = nullptr;
        int *inside = nullptr, *prev = nullptr, *row_last = nullptr, *flags = nullptr;
        double *nuc = nullptr, *col = nullptr;  // nucleons of A then B
        int nuc_cap = 0;
        double *table = nullptr;
        size_t table_cap = 0;
        bool have_T = false;
    } ips;
    int nuc_cap = 0;
    int work_sheets = 0;
    C<double> *VA = nullptr, *VB = nullptr;
    C<double> *u1x = nullptr, *u2x = nullptr, *u1y = nullptr, *u2y = nullptr;
    int *newton_iters = nullptr, *newton_status = nullptr;
    double *newton_alpha = nullptr;  // [8][2n] exponents of the tau = 0 links

    // fields: FP64 state (+ second U/phi buffer), FP32 state (+ second buffer)
    State<double> s64{};
    C<double> *ux64b = nullptr, *uy64b = nullptr;
    double *phi64b = nullptr;
    State<float> s32{};
    C<float> *ux32b = nullptr, *uy32b = nullptr;
    float *phi32b = nullptr;

    // observables
    double *T10 = nullptr, *eps = nullptr, *u4 = nullptr, *pi10 = nullptr;
    double *carry = nullptr;
    int *wrote = nullptr, *found = nullptr;
    double *partial = nullptr, *scal = nullptr;
    double *h_scal = nullptr;  // pinned host copy of scal
    EventGeom *d_ev = nullptr;

    bool initialized = false, half_done = false, finished = false;
    cudaEvent_t ie[4] = {nullptr, nullptr, nullptr, nullptr};  // init stage timing
    bool init_from_wilson = false;                              // of the pending init
    int it = 0;  // completed full steps
    double last_leapfrog_ms = 0;
    int last_leapfrog_launches = 0;

    // adjoint workspace (allocated by the first ipg_forward)
    struct {
        int k = 0, steps = 0;
        std::vector<State<double>> cp;  // state before step j k
        State<double> w[3]{};           // working states
        AdjState adj{};
        double *tbar = nullptr;
        State<double> fin{};            // state after the last step
        bool ready = false;
        double sums[6] = {0};            // W, X, Y, Sxx, Syy, Sxy of the weight
        double sum_ttt = 0, ET = 0, eps2 = 0;
        double ms_forward = 0, ms_backward = 0;  // device time of the last pair
        double *sites = nullptr;                 // [n][18] staging for the host copy
        bool from_inputs = false;  // the tau = 0 state came from g2mu + noise
        // initial-condition adjoint: U1/U2 adjoints, V adjoints, a V copy
        C<double> *b1x = nullptr, *b2x = nullptr, *b1y = nullptr, *b2y = nullptr;
        C<double> *vbA = nullptr, *vbB = nullptr, *vcur = nullptr, *vcur2 = nullptr;
        double *amp2 = nullptr;  // nucleus B's rho amplitude in the input adjoint
        double *g2mu_bar = nullptr;
        double *rho_all = nullptr;  // [2][Ny][n][8] rho adjoint, kept on the device
        // FP32 adjoint (contexts of the FP32 form): the bulk form's own states
        // (deviation storage) and adjoints in FP32; the tau = 0 adjoint is
        // widened into adj at the end
        bool fp32 = false;
        std::vector<State<float>> cp32;   // checkpoints (every state when k = 1)
        std::vector<State<float>> seg32;  // a segment's states, recomputed
        State<float> w32[3]{};
        State<float> fin32{};
        AdjStateT<float> adj32{};
        float *tbar32 = nullptr;
    } aw;

    double *ecc3 = nullptr;  // [8] ipg_eccentricity_report sums (first call)

    // gauge fixing and multiplicity (allocated by the first call)
    struct {
        double2 *planes = nullptr;   // [16][n]: chi [4][n] and G [9][n] while gauge
                                     // fixing, the spectrum's planes after
        double *green = nullptr;     // [n] gauge-fixing multiplier
        double *sin_half = nullptr;  // [N]
        double *partial = nullptr;   // [kGaugeBlocks][kMultRow]
        double *out = nullptr;       // [kMultRow]
        GaugeFixCtl *ctl = nullptr;
        GaugeFixCtl *h_ctl = nullptr;  // pinned
        double *h_out = nullptr;       // pinned [kMultRow]
    } gf;

    // output files formatted on the GPU (ipg_write_outputs); freed by ipg_destroy
    struct {
        long long cap_lines = 0;
        char *chunks = nullptr, *text = nullptr;
        int *chunk_len = nullptr, *bad = nullptr;
        long long *chunk_off = nullptr;
        double *term = nullptr;
        char *h_text = nullptr;     // pinned image of the file body
        double *h_term = nullptr;   // pinned Etot terms
        long long *h_small = nullptr;  // pinned: total bytes, bad flag
    } out;
    bool init_from_inputs = false;

    std::vector<void *> allocs;
};

namespace {

ipg_status fail(ipg_ctx *c, ipg_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return st;
}

ipg_status cuda_check(ipg_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return IPG_OK;
    return fail(c, IPG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define IPG_CUDA(c, expr)                                        \
    do {                                                         \
        ipg_status _s = cuda_check((c), (expr), #expr);          \
        if (_s != IPG_OK) return _s;                             \
    } while (0)

#define IPG_LAUNCHED(c, k)                                                 \
    do {                                                                   \
        (c)->launches += (k);                                              \
        ipg_status _s = cuda_check((c), cudaGetLastError(), "kernel launch"); \
        if (_s != IPG_OK) return _s;                                       \
    } while (0)

template <typename P>
ipg_status dalloc(ipg_ctx *c, P **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(P));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, IPG_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s",
                    count * sizeof(P), cudaGetErrorString(e));
    }
    c->allocs.push_back(q);
    *p = reinterpret_cast<P *>(q);
    return IPG_OK;
}

#define IPG_TRY(expr)                    \
    do {                                 \
        ipg_status _s = (expr);          \
        if (_s != IPG_OK) return _s;     \
    } while (0)

__global__ void k_identity(size_t n, C<double> *V) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
#pragma unroll
    for (int k = 0; k < 9; k++)
        V[k * n + pos] = {(k == 0 || k == 4 || k == 8) ? 1. : 0., 0.};
}

int ilog2(int v) {
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

ipg_status alloc_state64(ipg_ctx *c, State<double> &s) {
    const size_t n = c->n;
    IPG_TRY(dalloc(c, &s.ux, 9 * n));
    IPG_TRY(dalloc(c, &s.uy, 9 * n));
    IPG_TRY(dalloc(c, &s.e1, 8 * n));
    IPG_TRY(dalloc(c, &s.e2, 8 * n));
    IPG_TRY(dalloc(c, &s.phi, 9 * n));
    IPG_TRY(dalloc(c, &s.pi, 9 * n));
    return IPG_OK;
}

ipg_status alloc_state32(ipg_ctx *c, State<float> &s) {
    const size_t n = c->n;
    IPG_TRY(dalloc(c, &s.ux, 9 * n));
    IPG_TRY(dalloc(c, &s.uy, 9 * n));
    IPG_TRY(dalloc(c, &s.e1, 8 * n));
    IPG_TRY(dalloc(c, &s.e2, 8 * n));
    IPG_TRY(dalloc(c, &s.phi, 9 * n));
    IPG_TRY(dalloc(c, &s.pi, 9 * n));
    return IPG_OK;
}

bool is_fp32(const ipg_ctx *c) { return c->cfg.precision == IPG_FP32; }

// one leapfrog launch on the active precision, then swap the U/phi buffers
template <typename T>
ipg_status step_impl(ipg_ctx *c, State<T> &s, C<T> *&uxb, C<T> *&uyb,
                     T *&phib, double tau, double dt_pe, double dt_pu,
                     int do_pe, int do_pu, bool reunit) {
    StepCoef<T> cf;
    cf.tau = (T)tau;
    cf.dt_pe = (T)dt_pe;
    cf.dt_pu = (T)dt_pu;
    cf.g = (T)c->cfg.g;
    cf.do_pe = do_pe;
    cf.do_pu = do_pu;
    set_derived(cf);
    launch_leapfrog<T>(c->d_ev, c->N, s, uxb, uyb, phib, cf, reunit, c->stream, c->scal + 38);
    IPG_LAUNCHED(c, 1);
    if (do_pu) {
        std::swap(s.ux, uxb);
        std::swap(s.uy, uyb);
        std::swap(s.phi, phib);
    }
    return IPG_OK;
}

ipg_status step(ipg_ctx *c, double tau, double dt_pe, double dt_pu, int do_pe,
                int do_pu) {
    if (is_fp32(c))
        return step_impl<float>(c, c->s32, c->ux32b, c->uy32b, c->phi32b, tau,
                                dt_pe, dt_pu, do_pe, do_pu, true);
    return step_impl<double>(c, c->s64, c->ux64b, c->uy64b, c->phi64b, tau,
                             dt_pe, dt_pu, do_pe, do_pu, false);
}

ipg_status sync(ipg_ctx *c) {
    IPG_CUDA(c, cudaStreamSynchronize(c->stream));
    return IPG_OK;
}

float elapsed(ipg_ctx *c) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    return ms;
}

// host layout helpers: per-site 3x3 (18 doubles) <-> device planes
void planes_to_sites_m3(const std::vector<double> &pl, size_t n, double *out) {
    // pl: [9][n] complex = 18 n doubles, interleaved per component
    for (size_t p = 0; p < n; p++)
        for (int k = 0; k < 9; k++) {
            out[18 * p + 2 * k] = pl[2 * (k * n + p)];
            out[18 * p + 2 * k + 1] = pl[2 * (k * n + p) + 1];
        }
}

void herm_to_sites(const std::vector<double> &pl, size_t n, bool traceless,
                   double *out) {
    for (size_t p = 0; p < n; p++) {
        double d0, d1, d2, o[6];
        if (traceless) {
            d0 = pl[0 * n + p];
            d1 = pl[1 * n + p];
            d2 = -(d0 + d1);
            for (int q = 0; q < 6; q++) o[q] = pl[(2 + q) * n + p];
        } else {
            d0 = pl[0 * n + p];
            d1 = pl[1 * n + p];
            d2 = pl[2 * n + p];
            for (int q = 0; q < 6; q++) o[q] = pl[(3 + q) * n + p];
        }
        double *m = out + 18 * p;
        const double v[18] = {d0,   0.,    o[0], o[1],  o[2], o[3],
                              o[0], -o[1], d1,   0.,    o[4], o[5],
                              o[2], -o[3], o[4], -o[5], d2,   0.};
        std::memcpy(m, v, sizeof(v));
    }
}

void sites_to_herm(const double *in, size_t n, bool traceless,
                   std::vector<double> &pl) {
    pl.assign((traceless ? 8 : 9) * n, 0.);
    for (size_t p = 0; p < n; p++) {
        const double *m = in + 18 * p;
        const double d0 = m[0], d1 = m[8], d2 = m[16];
        const double o[6] = {m[2], m[3], m[4], m[5], m[10], m[11]};
        if (traceless) {
            const double t = (d0 + d1 + d2) / 3.;
            pl[0 * n + p] = d0 - t;
            pl[1 * n + p] = d1 - t;
            for (int q = 0; q < 6; q++) pl[(2 + q) * n + p] = o[q];
        } else {
            pl[0 * n + p] = d0;
            pl[1 * n + p] = d1;
            pl[2 * n + p] = d2;
            for (int q = 0; q < 6; q++) pl[(3 + q) * n + p] = o[q];
        }
    }
}

ipg_status to_fp32_if_needed(ipg_ctx *c) {
    if (!is_fp32(c)) return IPG_OK;
    launch_convert_state_down<float>(c->n, c->s64, c->s32, c->stream);
    IPG_LAUNCHED(c, 1);
    return IPG_OK;
}

// make c->s64 hold the current state (converts from FP32 when needed)
ipg_status state64(ipg_ctx *c) {
    if (!is_fp32(c)) return IPG_OK;
    launch_convert_state<float>(c->n, c->s32, c->s64, c->stream);
    IPG_LAUNCHED(c, 1);
    return IPG_OK;
}

ipg_status copy_state(ipg_ctx *c, const State<double> &dst, const State<double> &src) {
    const size_t n = c->n;
    auto cp = [&](void *d, const void *s_, size_t bytes) {
        return cudaMemcpyAsync(d, s_, bytes, cudaMemcpyDeviceToDevice, c->stream);
    };
    IPG_CUDA(c, cp(dst.ux, src.ux, 9 * n * sizeof(C<double>)));
    IPG_CUDA(c, cp(dst.uy, src.uy, 9 * n * sizeof(C<double>)));
    IPG_CUDA(c, cp(dst.e1, src.e1, 8 * n * sizeof(double)));
    IPG_CUDA(c, cp(dst.e2, src.e2, 8 * n * sizeof(double)));
    IPG_CUDA(c, cp(dst.phi, src.phi, 9 * n * sizeof(double)));
    IPG_CUDA(c, cp(dst.pi, src.pi, 9 * n * sizeof(double)));
    return IPG_OK;
}

ipg_status copy_state32(ipg_ctx *c, const State<float> &dst, const State<float> &src) {
    const size_t n = c->n;
    auto cp = [&](void *d, const void *s_, size_t bytes) {
        return cudaMemcpyAsync(d, s_, bytes, cudaMemcpyDeviceToDevice, c->stream);
    };
    IPG_CUDA(c, cp(dst.ux, src.ux, 9 * n * sizeof(C<float>)));
    IPG_CUDA(c, cp(dst.uy, src.uy, 9 * n * sizeof(C<float>)));
    IPG_CUDA(c, cp(dst.e1, src.e1, 8 * n * sizeof(float)));
    IPG_CUDA(c, cp(dst.e2, src.e2, 8 * n * sizeof(float)));
    IPG_CUDA(c, cp(dst.phi, src.phi, 9 * n * sizeof(float)));
    IPG_CUDA(c, cp(dst.pi, src.pi, 9 * n * sizeof(float)));
    return IPG_OK;
}

// One step of the FP32 bulk form from `in` into `out`: E and pi are copied
// to `out` first (unless they are the same buffers) and updated there, the
// new U and phi are written to `out`, whose U/phi buffers differ from `in`'s.
ipg_status step32_into(ipg_ctx *c, const State<float> &in, const State<float> &out,
                       const StepCoef<double> &cfd) {
    const size_t n = c->n;
    if (out.e1 != in.e1) {
        IPG_CUDA(c, cudaMemcpyAsync(out.e1, in.e1, 8 * n * sizeof(float),
                                    cudaMemcpyDeviceToDevice, c->stream));
        IPG_CUDA(c, cudaMemcpyAsync(out.e2, in.e2, 8 * n * sizeof(float),
                                    cudaMemcpyDeviceToDevice, c->stream));
        IPG_CUDA(c, cudaMemcpyAsync(out.pi, in.pi, 9 * n * sizeof(float),
                                    cudaMemcpyDeviceToDevice, c->stream));
    }
    State<float> s = in;
    s.e1 = out.e1;
    s.e2 = out.e2;
    s.pi = out.pi;
    StepCoef<float> cf;
    cf.tau = (float)cfd.tau;
    cf.dt_pe = (float)cfd.dt_pe;
    cf.dt_pu = (float)cfd.dt_pu;
    cf.g = (float)cfd.g;
    cf.do_pe = cfd.do_pe;
    cf.do_pu = cfd.do_pu;
    set_derived(cf);
    launch_leapfrog<float>(c->d_ev, c->N, s, out.ux, out.uy, out.phi, cf, true, c->stream,
                           c->scal + 38);
    IPG_LAUNCHED(c, 1);
    return IPG_OK;
}

// coefficients of launch s of run_evolution (0: tau = 0 half step)
StepCoef<double> evolution_coef(const ipg_ctx *c, int s) {
    StepCoef<double> cf;
    cf.tau = s * c->dtau;
    cf.dt_pe = c->dtau;
    cf.dt_pu = c->dtau;
    cf.g = c->cfg.g;
    cf.do_pe = s > 0;
    cf.do_pu = 1;
    set_derived(cf);
    return cf;
}

// T^tautau-weighted eccentricity over the cells [2, N-2)^2 (the cells the
// reference's eccentricity sums over) with the weighted centroid as origin (a
// smooth weight: a clamp such as max(T^tautau, 0) would put a kink where
// vacuum cells sit at T^tautau = 0):
// eps2 = |sum w (x~ + i y~)^2| / sum w (x~^2 + y~^2), from the weight sums
// W, X = sum w x, Y, Sxx = sum w x^2, Syy, Sxy; d[6] receives d eps2 / d sums.
double eps2_from_sums(const double *S, double *d) {
    const double W = S[0], X = S[1], Y = S[2], Sxx = S[3], Syy = S[4], Sxy = S[5];
    const double cxx = Sxx - X * X / W, cyy = Syy - Y * Y / W, cxy = Sxy - X * Y / W;
    const double re = cxx - cyy, im = 2. * cxy, den = cxx + cyy;
    const double mag = std::sqrt(re * re + im * im);
    const double e = mag / den;
    if (d) {
        // d e / d (cxx, cyy, cxy)
        const double dre = mag > 0 ? re / mag : 0., dim = mag > 0 ? im / mag : 0.;
        const double gxx = (dre) / den - e / den;
        const double gyy = (-dre) / den - e / den;
        const double gxy = 2. * dim / den;
        // cxx = Sxx - X^2/W, cyy = Syy - Y^2/W, cxy = Sxy - XY/W
        d[0] = gxx * (X * X / (W * W)) + gyy * (Y * Y / (W * W)) + gxy * (X * Y / (W * W));
        d[1] = gxx * (-2. * X / W) + gxy * (-Y / W);
        d[2] = gyy * (-2. * Y / W) + gxy * (-X / W);
        d[3] = gxx;
        d[4] = gyy;
        d[5] = gxy;
    }
    return e;
}

bool in_ecc_window(int N, int i, int j) { return i >= 2 && i < N - 2 && j >= 2 && j < N - 2; }

// The leapfrog schedule of Evolution::run up to it = itmax - 1: the tau = 0
// half step of phi and U (Evolution.cpp:393-394), then full steps
// it = 1 .. itmax-1 (416-421).
ipg_status run_evolution(ipg_ctx *c) {
    const int itmax = c->itmax;
    const double dtau = c->dtau;
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    IPG_TRY(step(c, 0., dtau, dtau, 0, 1));
    c->half_done = true;
    for (int it = 1; it < itmax; it++) {
        IPG_TRY(step(c, it * dtau, dtau, dtau, 1, 1));
        c->it = it;
    }
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    IPG_TRY(sync(c));
    c->last_leapfrog_ms = elapsed(c);
    c->last_leapfrog_launches = itmax;
    return IPG_OK;
}

// Observables at it = itmax before the last half step (Evolution.cpp:406-410),
// the last half step of pi and E (426-431), the Gauss law (633-635) and the
// checks, all enqueued on the context's stream; the scalars are copied to
// pinned host memory. observables_finish waits and fills the result.
// Every path that rewrites the observable arrays (eps, u4, pi10, T10) calls
// this first: an asynchronous copy of the previous contents
// (ipg_get_observables_async) must have read them before the context's
// stream overwrites them.
ipg_status wait_observable_copies(ipg_ctx *c) {
    if (c->obs_copy_pending) IPG_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_obs_copied, 0));
    return IPG_OK;
}

ipg_status observables_enqueue(ipg_ctx *c) {
    const int itmax = c->itmax;
    const double dtau = c->dtau;
    const size_t n = c->n;
    const int N = c->N;
    IPG_TRY(wait_observable_copies(c));
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    TmunuArgs ta;
    ta.N = N;
    ta.g = c->cfg.g;
    ta.tau = itmax * dtau;
    ta.a = c->a;
    ta.s = c->s64;
    ta.T10 = c->T10;
    // FP32 contexts: T^munu reads the FP32 state directly
    ta.from32 = is_fp32(c) ? 1 : 0;
    ta.s32 = c->s32;
    launch_tmunu(ta, c->stream);
    IPG_LAUNCHED(c, 7);
    LandauArgs la;
    la.N = N;
    la.tau_fm = itmax * dtau * c->a;
    la.tau2_fm = c->a * itmax * dtau * c->a * itmax * dtau;
    la.tau_fm_parts[0] = itmax;
    la.tau_fm_parts[1] = dtau;
    la.tau_fm_parts[2] = c->a;
    la.T10 = c->T10;
    la.eps = c->eps;
    la.u4 = c->u4;
    la.pi10 = c->pi10;
    la.found = c->found;
    launch_landau(la, c->carry, c->wrote, c->stream);
    IPG_LAUNCHED(c, 2);
    double *scal = c->scal;
    launch_eccentricity(N, c->cfg.L, c->a, c->eps, c->u4, c->T10, c->partial,
                        scal + 0, scal + 8, c->stream);
    IPG_LAUNCHED(c, 4);

    IPG_TRY(step(c, itmax * dtau, dtau / 2., dtau, 1, 0));
    c->it = itmax;
    // the checks read the live state; on FP32 contexts the FP64 copy is made
    // only where a caller asks for FP64 fields (ipg_get_field, the gauge
    // fixing and the spectrum)
    if (is_fp32(c)) {
        launch_gauss_law(N, c->s32, c->partial, scal + 32, c->stream);
        launch_unitarity(N, c->s32.ux, c->s32.uy, c->partial, scal + 33, c->stream);
    } else {
        launch_gauss_law(N, c->s64, c->partial, scal + 32, c->stream);
        launch_unitarity(N, c->s64.ux, c->s64.uy, c->partial, scal + 33, c->stream);
    }
    IPG_LAUNCHED(c, 4);
    launch_cell_flags(n, c->found, c->eps, c->partial, scal + 36, c->stream);
    IPG_LAUNCHED(c, 2);
    IPG_CUDA(c, cudaMemcpyAsync(c->h_scal, scal, sizeof(double) * 39,
                                cudaMemcpyDeviceToHost, c->stream));
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    return IPG_OK;
}

ipg_status observables_finish(ipg_ctx *c, ipg_result *res) {
    IPG_TRY(sync(c));
    const double ms_obs = elapsed(c);
    c->finished = true;
    const int itmax = c->itmax;
    const double dtau = c->dtau;
    const double *h = c->h_scal;
    const int nan_count = (int)h[37];
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->itmax = itmax;
        res->dtau = dtau;
        res->tau_final = itmax * dtau * c->a;
        res->gauss_violation = h[32];
        res->unitarity_max = h[33];
        res->sum_Ttautau = h[3];
        res->sum_eps = h[4];
        res->E_T = res->tau_final * c->a * c->a * kHbarc * h[3];
        // radial moments: [0..5] avr1 avrSq avr3 avr4 avr5 avr6,
        // [6 + 2(n-1)], [7 + 2(n-1)] cos/sin moments for n = 1..6
        const double *m = h + 8;
        const double avr[6] = {m[0], m[1], m[2], m[3], m[4], m[5]};
        for (int k = 0; k < 6; k++) {
            const double cs = m[6 + 2 * k], sn = m[7 + 2 * k];
            res->eccentricity[k] = std::sqrt(cs * cs + sn * sn) / avr[k];
            res->psi[k] = (std::atan(sn / cs) + M_PI) / (k + 1);
        }
        res->cells_without_u = (int)h[36];
        res->ms_evolution = c->last_leapfrog_ms;
        res->ms_observables = ms_obs;
    }
    if (h[38] != 0.)
        return fail(c, IPG_ERR_TIMEOUT, "a leapfrog step gave up waiting for its tile loads");
    if (nan_count) return fail(c, IPG_ERR_NAN, "%d cells with non-finite e", nan_count);
    return IPG_OK;
}

// ---- gauge fixing and multiplicity ----------------------------------------

ipg_status gf_alloc(ipg_ctx *c) {
    auto &g = c->gf;
    if (g.planes) return IPG_OK;
    const size_t n = c->n;
    const int N = c->N;
    IPG_TRY(dalloc(c, &g.planes, 16 * n));
    IPG_TRY(dalloc(c, &g.green, n));
    IPG_TRY(dalloc(c, &g.sin_half, (size_t)N));
    IPG_TRY(dalloc(c, &g.partial, (size_t)kGaugeBlocks * kMultRow));
    IPG_TRY(dalloc(c, &g.out, (size_t)kMultRow));
    IPG_TRY(dalloc(c, &g.ctl, 1));
    IPG_CUDA(c, cudaMallocHost(&g.h_ctl, sizeof(GaugeFixCtl)));
    IPG_CUDA(c, cudaMallocHost(&g.h_out, sizeof(double) * kMultRow));
    // sin(kx / 2) with kx = 2 pi (-0.5 + i / N), the expression of
    // Evolution.cpp:2507-2513 (and GaugeFix.cpp:120-125), on the host
    std::vector<double> sh(N);
    for (int i = 0; i < N; i++) {
        const double kx = 2. * M_PI * (-0.5 + static_cast<double>(i) / static_cast<double>(N));
        sh[i] = std::sin(kx / 2.);
    }
    IPG_CUDA(c, cudaMemcpyAsync(g.sin_half, sh.data(), sizeof(double) * N,
                                cudaMemcpyHostToDevice, c->stream));
    launch_gauge_green(N, g.sin_half, g.green, c->stream);
    IPG_LAUNCHED(c, 1);
    return sync(c);
}

// the FP64 fields the gauge fixing and the spectrum work on: the live state
// of an FP64 context, a widened copy of an FP32 one
ipg_status fields64(ipg_ctx *c) { return state64(c); }

ipg_status gauge_fix_run(ipg_ctx *c, int max_iter, ipg_gauge_report *rep) {
    IPG_TRY(gf_alloc(c));
    auto &g = c->gf;
    const size_t n = c->n;
    GaugeFixCtl *h = g.h_ctl;
    std::memset(h, 0, sizeof(GaugeFixCtl));
    h->prev = 10000.;  // GaugeFix.cpp:34
    h->last = std::nan("");
    for (int k = 0; k < kGaugeHistory; k++) h->hist[k] = std::nan("");
    IPG_CUDA(c, cudaMemcpyAsync(g.ctl, h, sizeof(GaugeFixCtl), cudaMemcpyHostToDevice,
                                c->stream));
    GaugeFixArgs a;
    a.s = c->s64;
    a.N = c->N;
    a.chi = g.planes;
    a.G = reinterpret_cast<C<double> *>(g.planes + 4 * n);
    a.partial = g.partial;
    a.ctl = g.ctl;
    WilsonArgs w{};
    w.N = c->N;
    w.logN = c->logN;
    w.twiddle = c->twiddle;
    w.green = g.green;
    w.work = g.planes;
    w.rho_in = g.planes;
    w.no_product = 1;
    w.skip = &g.ctl->done;
    a.fft = w;
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    // iterations are enqueued in chunks; after a stopping rule every kernel
    // of the remaining iterations returns at once, and the host stops
    // enqueueing at the next chunk boundary
    constexpr int kChunk = 16;
    int launched = 0;
    while (launched < max_iter) {
        const int k = std::min(kChunk, max_iter - launched);
        for (int i = 0; i < k; i++) launch_gauge_fix_iteration(a, c->stream);
        IPG_LAUNCHED(c, 6 * k);
        launched += k;
        IPG_CUDA(c, cudaMemcpyAsync(h, g.ctl, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        IPG_TRY(sync(c));
        if (h->done) break;
    }
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    // the reference transforms the live fields; later steps of an FP32
    // context continue from the transformed fields rounded back to FP32
    IPG_TRY(to_fp32_if_needed(c));
    IPG_CUDA(c, cudaMemcpyAsync(h, g.ctl, sizeof(GaugeFixCtl), cudaMemcpyDeviceToHost,
                                c->stream));
    IPG_TRY(sync(c));
    if (rep) {
        rep->iterations = h->iter;
        rep->residual_checks = h->checks;
        rep->nan_sites = h->nan_sites;
        rep->residual = h->last;
        std::memcpy(rep->residual_every10, h->hist, sizeof(double) * kGaugeHistory);
        rep->ms = elapsed(c);
    }
    return IPG_OK;
}

ipg_status multiplicity_run(ipg_ctx *c, const ipg_multiplicity_params *p,
                            ipg_multiplicity_result *out) {
    ipg_multiplicity_params prm{};
    if (p) prm = *p;
    if (prm.max_gauge_iterations <= 0) prm.max_gauge_iterations = 4000;
    if (!c->initialized) return fail(c, IPG_ERR_STATE, "no fields: call ipg_init_fields first");
    const int it = c->it;
    if (it < 1)
        return fail(c, IPG_ERR_STATE, "the spectrum needs the fields after a step (it >= 1)");
    IPG_TRY(fields64(c));
    ipg_multiplicity_result m;
    std::memset(&m, 0, sizeof(m));
    IPG_TRY(gauge_fix_run(c, prm.max_gauge_iterations, &m.gauge));
    auto &g = c->gf;
    MultArgs ma;
    ma.N = c->N;
    ma.it = it;
    ma.dtau = c->dtau;
    ma.g = c->cfg.g;
    ma.a = c->a;
    ma.sin_half = g.sin_half;
    WilsonArgs w{};
    w.N = c->N;
    w.logN = c->logN;
    w.twiddle = c->twiddle;
    w.work = g.planes;
    w.rho_in = g.planes;
    w.no_product = 1;
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    launch_multiplicity(c->s64, ma, g.planes, w, g.partial, g.out, c->stream);
    IPG_LAUNCHED(c, 5);
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(g.h_out, g.out, sizeof(double) * kMultRow,
                                cudaMemcpyDeviceToHost, c->stream));
    IPG_TRY(sync(c));
    const double *o = g.h_out;
    int cnt[kKtBins];
    for (int b = 0; b < kKtBins; b++) cnt[b] = (int)o[2 + 2 * kKtBins + b];
    const ipg_status st =
        ipg_multiplicity_finish(o[0], o[1], o + 2, o + 2 + kKtBins, cnt, c->a, &prm, &m);
    if (st != IPG_OK) return fail(c, st, "bad multiplicity parameters");
    m.it = it;
    m.ms_spectrum = elapsed(c);
    if (out) *out = m;
    return IPG_OK;
}

}  // namespace

extern "C" {

const char *ipg_last_error(const ipg_ctx *ctx) {
    return ctx ? ctx->err.c_str() : "null context";
}

ipg_status ipg_create(const ipg_config *cfg, ipg_ctx **out) {
    if (!cfg || !out) return IPG_ERR_BAD_CONFIG;
    *out = nullptr;
    ipg_ctx *c = new (std::nothrow) ipg_ctx();
    if (!c) return IPG_ERR_NOMEM;
    c->cfg = *cfg;
    const int N = cfg->size;
    auto bad = [&](const char *msg) {
        c->err = msg;
        *out = c;  // caller can read the message, then destroy
        return IPG_ERR_BAD_CONFIG;
    };
    if (N < 8 || N > 2048 || (N & (N - 1)) != 0)
        return bad("size must be a power of two in [8, 2048]");
    if (cfg->Nc != 3) return bad("only SU(3) (Nc = 3) is supported");
    if (cfg->Ny < 1) return bad("Ny must be >= 1");
    if (!(cfg->L > 0) || !(cfg->g > 0) || !(cfg->maxtime > 0) || cfg->m < 0 ||
        cfg->UVdamp < 0)
        return bad("L, g, maxtime must be > 0 and m, UVdamp >= 0");
    if (cfg->precision != IPG_FP64 && cfg->precision != IPG_FP32)
        return bad("precision must be IPG_FP64 or IPG_FP32");
    if (cfg->newton_mode != 0 && cfg->newton_mode != 1)
        return bad("newton_mode must be 0 (the reference's iteration) or 1 (Newton on the group)");
    if (c->cfg.newton_max_iterations <= 0) c->cfg.newton_max_iterations = 2000;
    if (c->cfg.newton_max_restarts <= 0) c->cfg.newton_max_restarts = 200;
    if (!(c->cfg.newton_tolerance > 0)) c->cfg.newton_tolerance = 1e-6;
    c->N = N;
    c->logN = ilog2(N);
    c->n = (size_t)N * N;
    c->a = cfg->L / N;
    if (cfg->dtau > 0) {
        c->dtau = cfg->dtau;
    } else {
        const int steps = static_cast<int>(10 * cfg->maxtime / c->a) + 1;
        c->dtau = cfg->maxtime / (steps * c->a);
    }
    c->itmax = static_cast<int>(cfg->maxtime / (c->a * c->dtau) + 0.1);
    if (c->itmax < 1) return bad("maxtime shorter than one time step");
    c->m_lat = cfg->m * c->a / kHbarc;
    c->uv_lat = cfg->UVdamp / c->a * kHbarc;
    *out = c;

    IPG_CUDA(c, cudaSetDevice(cfg->device));
    IPG_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    IPG_CUDA(c, cudaStreamCreateWithFlags(&c->stream_v, cudaStreamNonBlocking));
    IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_nuc_fork, cudaEventDisableTiming));
    IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_nuc_join, cudaEventDisableTiming));
    IPG_CUDA(c, cudaStreamCreateWithFlags(&c->stream_copy, cudaStreamNonBlocking));
    IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_obs_ready, cudaEventDisableTiming));
    IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_obs_copied, cudaEventDisableTiming));
    for (int i = 0; i < 2; i++) {
        IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_fft[i], cudaEventDisableTiming));
        IPG_CUDA(c, cudaEventCreateWithFlags(&c->ev_prod[i], cudaEventDisableTiming));
    }
    IPG_CUDA(c, cudaEventCreate(&c->ev0));
    IPG_CUDA(c, cudaEventCreate(&c->ev1));
    for (cudaEvent_t &x : c->ie) IPG_CUDA(c, cudaEventCreate(&x));

    const size_t n = c->n;
    IPG_TRY(dalloc(c, &c->g2mu2A, n));
    IPG_TRY(dalloc(c, &c->g2mu2B, n));
    // an event made from Wilson lines has no g2mu maps: zero, as the
    // reference's cells keep them
    IPG_CUDA(c, cudaMemset(c->g2mu2A, 0, sizeof(double) * n));
    IPG_CUDA(c, cudaMemset(c->g2mu2B, 0, sizeof(double) * n));
    IPG_TRY(dalloc(c, &c->twiddle, (size_t)N));
    IPG_TRY(dalloc(c, &c->green, n));
    IPG_TRY(dalloc(c, &c->amp, n));
    // work buffer of a sheet batch: up to 128 MB (8 sheets at 512^2, 32 at
    // 256^2). Larger batches give each transform launch more parallelism:
    // the 512^2 Wilson-line stage takes 3.59 ms at 128 MB, 3.68 ms at 64 MB,
    // 4.08 ms at 32 MB
    const size_t per_sheet = 4 * n * sizeof(double2);
    c->work_sheets = (int)std::max<size_t>(1, (128ull << 20) / per_sheet);
    c->work_sheets = std::min(c->work_sheets, cfg->Ny);
    IPG_TRY(dalloc(c, &c->work, (size_t)c->work_sheets * 4 * n));
    IPG_TRY(dalloc(c, &c->work2, (size_t)c->work_sheets * 4 * n));
    IPG_TRY(dalloc(c, &c->VA, 9 * n));
    IPG_TRY(dalloc(c, &c->VB, 9 * n));
    IPG_TRY(dalloc(c, &c->u1x, 9 * n));
    IPG_TRY(dalloc(c, &c->u2x, 9 * n));
    IPG_TRY(dalloc(c, &c->u1y, 9 * n));
    IPG_TRY(dalloc(c, &c->u2y, 9 * n));
    IPG_TRY(dalloc(c, &c->newton_iters, 2 * n));
    IPG_TRY(dalloc(c, &c->newton_status, 2 * n));
    IPG_TRY(dalloc(c, &c->newton_alpha, 16 * n));
    IPG_TRY(alloc_state64(c, c->s64));
    IPG_TRY(dalloc(c, &c->ux64b, 9 * n));
    IPG_TRY(dalloc(c, &c->uy64b, 9 * n));
    IPG_TRY(dalloc(c, &c->phi64b, 9 * n));
    if (is_fp32(c)) {
        IPG_TRY(alloc_state32(c, c->s32));
        IPG_TRY(dalloc(c, &c->ux32b, 9 * n));
        IPG_TRY(dalloc(c, &c->uy32b, 9 * n));
        IPG_TRY(dalloc(c, &c->phi32b, 9 * n));
    }
    IPG_TRY(dalloc(c, &c->T10, 10 * n));
    IPG_TRY(dalloc(c, &c->eps, n));
    IPG_TRY(dalloc(c, &c->u4, 4 * n));
    IPG_TRY(dalloc(c, &c->pi10, 10 * n));
    IPG_TRY(dalloc(c, &c->carry, 5 * n));
    IPG_TRY(dalloc(c, &c->wrote, n));
    IPG_TRY(dalloc(c, &c->found, n));
    IPG_TRY(dalloc(c, &c->partial, 8192));  // 296 reduction blocks x <= 18 slots
    IPG_TRY(dalloc(c, &c->scal, 64));
    IPG_CUDA(c, cudaMallocHost(&c->h_scal, 64 * sizeof(double)));
    IPG_TRY(dalloc(c, &c->d_ev, 1));

    // twiddles exp(-2 pi i k/N), evaluated on the host in double precision
    std::vector<double2> tw(N);
    for (int k = 0; k < N; k++) {
        const double ang = 2.0 * M_PI * (double)k / (double)N;
        tw[k] = make_double2(std::cos(ang), -std::sin(ang));
    }
    IPG_CUDA(c, cudaMemcpyAsync(c->twiddle, tw.data(), sizeof(double2) * tw.size(),
                                cudaMemcpyHostToDevice, c->stream));
    EventGeom geom{N, cfg->Ny, c->a, cfg->g, c->m_lat, c->uv_lat};
    IPG_CUDA(c, cudaMemcpyAsync(c->d_ev, &geom, sizeof(geom),
                                cudaMemcpyHostToDevice, c->stream));
    launch_green(N, c->m_lat, c->uv_lat, c->green, c->stream);
    IPG_LAUNCHED(c, 1);
    if (is_fp32(c)) {
        std::vector<float2> tw32(N);
        for (int k = 0; k < N; k++) tw32[k] = make_float2((float)tw[k].x, (float)tw[k].y);
        IPG_TRY(dalloc(c, &c->twiddle32, (size_t)N));
        IPG_TRY(dalloc(c, &c->green32, n));
        IPG_CUDA(c, cudaMemcpyAsync(c->twiddle32, tw32.data(), sizeof(float2) * N,
                                    cudaMemcpyHostToDevice, c->stream));
        launch_round_to_float(n, c->green, c->green32, c->stream);
        IPG_LAUNCHED(c, 1);
        IPG_TRY(sync(c));
    }
    IPG_TRY(sync(c));
    c->err.clear();
    return IPG_OK;
}

ipg_status ipg_destroy(ipg_ctx *ctx) {
    if (!ctx) return IPG_OK;
    if (ctx->stream) {
        cudaSetDevice(ctx->cfg.device);
        cudaStreamSynchronize(ctx->stream);
    }
    // an observables copy may still be writing the caller's host arrays
    if (ctx->stream_copy) cudaStreamSynchronize(ctx->stream_copy);
    for (void *p : ctx->allocs) cudaFree(p);
    if (ctx->h_scal) cudaFreeHost(ctx->h_scal);
    if (ctx->gf.h_ctl) cudaFreeHost(ctx->gf.h_ctl);
    if (ctx->gf.h_out) cudaFreeHost(ctx->gf.h_out);
    {
        auto &o = ctx->out;
        for (void *p : {(void *)o.chunks, (void *)o.text, (void *)o.chunk_len, (void *)o.bad,
                        (void *)o.chunk_off, (void *)o.term})
            if (p) cudaFree(p);
        for (void *p : {(void *)o.h_text, (void *)o.h_term, (void *)o.h_small})
            if (p) cudaFreeHost(p);
    }
    for (cudaEvent_t x : ctx->ie)
        if (x) cudaEventDestroy(x);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream_copy) {
        cudaStreamSynchronize(ctx->stream_copy);
        cudaStreamDestroy(ctx->stream_copy);
    }
    if (ctx->ev_obs_ready) cudaEventDestroy(ctx->ev_obs_ready);
    if (ctx->ev_obs_copied) cudaEventDestroy(ctx->ev_obs_copied);
    if (ctx->ev_nuc_fork) cudaEventDestroy(ctx->ev_nuc_fork);
    if (ctx->ev_nuc_join) cudaEventDestroy(ctx->ev_nuc_join);
    if (ctx->stream_v) {
        cudaStreamSynchronize(ctx->stream_v);
        cudaStreamDestroy(ctx->stream_v);
    }
    for (int i = 0; i < 2; i++) {
        if (ctx->ev_fft[i]) cudaEventDestroy(ctx->ev_fft[i]);
        if (ctx->ev_prod[i]) cudaEventDestroy(ctx->ev_prod[i]);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return IPG_OK;
}

ipg_status ipg_reseed(ipg_ctx *ctx, uint64_t seed) {
    if (!ctx) return IPG_ERR_BAD_CONFIG;
    ctx->cfg.seed = seed;
    return IPG_OK;
}

ipg_status ipg_time_grid(const ipg_ctx *ctx, double *dtau, int *itmax) {
    if (!ctx) return IPG_ERR_BAD_CONFIG;
    if (dtau) *dtau = ctx->dtau;
    if (itmax) *itmax = ctx->itmax;
    return IPG_OK;
}

ipg_status ipg_set_g2mu(ipg_ctx *c, const double *A, const double *B) {
    if (!c || !A || !B) return fail(c, IPG_ERR_BAD_CONFIG, "null argument");
    IPG_CUDA(c, cudaMemcpyAsync(c->g2mu2A, A, sizeof(double) * c->n,
                                cudaMemcpyHostToDevice, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(c->g2mu2B, B, sizeof(double) * c->n,
                                cudaMemcpyHostToDevice, c->stream));
    c->have_g2mu = true;
    return IPG_OK;
}

ipg_status ipg_set_g2mu_device(ipg_ctx *c, const double *A, const double *B) {
    if (!c || !A || !B) return fail(c, IPG_ERR_BAD_CONFIG, "null argument");
    IPG_CUDA(c, cudaMemcpyAsync(c->g2mu2A, A, sizeof(double) * c->n,
                                cudaMemcpyDeviceToDevice, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(c->g2mu2B, B, sizeof(double) * c->n,
                                cudaMemcpyDeviceToDevice, c->stream));
    c->have_g2mu = true;
    return IPG_OK;
}

ipg_status ipg_set_nuclei(ipg_ctx *c, const double *xyzA, int nA, const double *xyzB, int nB,
                          double b, double BG, double QsMax, double QsmuRatio) {
    if (!c || !xyzA || !xyzB || nA < 1 || nB < 1) return IPG_ERR_BAD_CONFIG;
    if (!(BG > 0) || !(QsMax > 0) || !(QsmuRatio > 0))
        return fail(c, IPG_ERR_BAD_CONFIG, "BG, QsMax and QsmuRatio must be > 0");
    const int amax = std::max(nA, nB);
    if (amax > c->nuc_cap) {
        IPG_TRY(dalloc(c, &c->nuc_xyz, 3 * (size_t)amax));
        IPG_TRY(dalloc(c, &c->nuc_gx, (size_t)amax * c->N));
        IPG_TRY(dalloc(c, &c->nuc_gy, (size_t)amax * c->N));
        c->nuc_cap = amax;
    }
    for (int nuc = 0; nuc < 2; nuc++) {
        IPG_CUDA(c, cudaMemcpyAsync(c->nuc_xyz, nuc ? xyzB : xyzA, 3 * sizeof(double) * (nuc ? nB : nA),
                                    cudaMemcpyHostToDevice, c->stream));
        NucleiArgs na;
        na.N = c->N;
        na.L = c->cfg.L;
        na.BG = BG;
        na.QsMax = QsMax;
        na.QsmuRatio = QsmuRatio;
        na.g = c->cfg.g;
        na.A = nuc ? nB : nA;
        na.xyz = c->nuc_xyz;
        na.shift = nuc ? b / 2. : -b / 2.;
        na.gx = c->nuc_gx;
        na.gy = c->nuc_gy;
        na.partial = c->partial;
        na.out = nuc ? c->g2mu2B : c->g2mu2A;
        launch_g2mu_from_nucleons(na, c->stream);
        IPG_LAUNCHED(c, 3);
    }
    IPG_TRY(sync(c));  // the positions buffer is reused for the second nucleus
    c->have_g2mu = true;
    return IPG_OK;
}

ipg_status ipg_set_nuclei_ipsat(ipg_ctx *c, const double *xyzA, int nA, const double *xyzB,
                                int nB, const double *phiA, const double *phiB,
                                const double *normA, const double *normB, double b,
                                const ipg_ipsat_params *p, const double *Tlist,
                                const double *qs2, int nT, int ny, double dy,
                                ipg_ipsat_report *rep) {
    if (!c || !xyzA || !xyzB || nA < 1 || nB < 1 || !p || !Tlist || !qs2)
        return IPG_ERR_BAD_CONFIG;
    if (nT < 2 || ny < 2 || !(dy > 0) || !(p->BG > 0) || !(p->QsmuRatio > 0) ||
        !(p->QsmuRatioB > 0) || !(p->roots > 0) || p->average_over_nuclei < 1)
        return fail(c, IPG_ERR_BAD_CONFIG, "IP-Sat parameters or table shape out of range");
    for (int i = 0; i + 1 < nT; i++)
        if (!(Tlist[i] < Tlist[i + 1]))
            return fail(c, IPG_ERR_BAD_CONFIG, "the T column of the table must increase");
    const size_t n = c->n;
    auto &S = c->ips;
    if (!S.TA) {
        IPG_TRY(dalloc(c, &S.TA, n));
        IPG_TRY(dalloc(c, &S.TB, n));
        IPG_TRY(dalloc(c, &S.yB, n));
        IPG_TRY(dalloc(c, &S.inside, n));
        IPG_TRY(dalloc(c, &S.prev, n));
        IPG_TRY(dalloc(c, &S.row_last, (size_t)c->N));
        IPG_TRY(dalloc(c, &S.flags, 1));
    }
    if (nA + nB > S.nuc_cap) {
        IPG_TRY(dalloc(c, &S.nuc, 4 * (size_t)(nA + nB)));
        IPG_TRY(dalloc(c, &S.col, 3 * (size_t)(nA + nB)));
        S.nuc_cap = nA + nB;
    }
    const size_t tsz = (size_t)nT + (size_t)nT * ny;
    if (tsz > S.table_cap) {
        IPG_TRY(dalloc(c, &S.table, tsz));
        S.table_cap = tsz;
    }
    // nucleon positions shifted by -+ b/2 along x (Init.cpp:855-864, reaction
    // plane not rotated); wounding with d^2 < sigma_NN / (10 pi) fm^2
    // (Init.cpp:1125-1141, 1196-1200)
    std::vector<double> nuc(4 * (size_t)(nA + nB)), col(3 * (size_t)(nA + nB));
    std::vector<int> hit(nA + nB, 0);
    for (int k = 0; k < nA + nB; k++) {
        const bool isB = k >= nA;
        const int i = isB ? k - nA : k;
        const double *xyz = isB ? xyzB : xyzA;
        nuc[4 * k] = isB ? xyz[3 * i] + b / 2. : xyz[3 * i] - b / 2.;
        nuc[4 * k + 1] = xyz[3 * i + 1];
        nuc[4 * k + 2] = isB ? (phiB ? phiB[i] : 0.) : (phiA ? phiA[i] : 0.);
        nuc[4 * k + 3] = isB ? (normB ? normB[i] : 1.) : (normA ? normA[i] : 1.);
    }
    const double d2 = p->sigmaNN / (M_PI * 10.);
    int Ncoll = 0;
    for (int i = 0; i < nA; i++)
        for (int j = 0; j < nB; j++) {
            const double dx = nuc[4 * (nA + j)] - nuc[4 * i];
            const double dyy = nuc[4 * (nA + j) + 1] - nuc[4 * i + 1];
            if (dx * dx + dyy * dyy < d2) {
                Ncoll++;
                hit[i] = hit[nA + j] = 1;
            }
        }
    if (nA == 1 && nB == 1) hit[0] = hit[1] = 1;  // p+p: collided in any case
    int Npart = 0;
    for (int k = 0; k < nA + nB; k++) {
        Npart += hit[k];
        col[3 * k] = nuc[4 * k];
        col[3 * k + 1] = nuc[4 * k + 1];
        col[3 * k + 2] = hit[k];
    }
    IPG_CUDA(c, cudaMemcpyAsync(S.nuc, nuc.data(), sizeof(double) * nuc.size(),
                                cudaMemcpyHostToDevice, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(S.col, col.data(), sizeof(double) * col.size(),
                                cudaMemcpyHostToDevice, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(S.table, Tlist, sizeof(double) * nT, cudaMemcpyHostToDevice,
                                c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(S.table + nT, qs2, sizeof(double) * nT * ny,
                                cudaMemcpyHostToDevice, c->stream));
    IPG_CUDA(c, cudaMemsetAsync(S.flags, 0, sizeof(int), c->stream));
    IpsatArgs a;
    a.N = c->N;
    a.L = c->cfg.L;
    a.a = c->a;
    a.g = c->cfg.g;
    a.BG = p->BG;
    a.xi = p->proton_anisotropy;
    a.nuclei_in_average = (double)p->average_over_nuclei;
    a.ratioA = p->QsmuRatio;
    a.ratioB = p->QsmuRatioB;
    a.rapidity = p->rapidity;
    a.roots = p->roots;
    a.xfactor = p->x_factor;
    a.rmax = p->rmax;
    a.fluct_x = p->use_fluctuating_x;
    a.nA = nA;
    a.nB = nB;
    a.nucA = S.nuc;
    a.nucB = S.nuc + 4 * (size_t)nA;
    a.nT = nT;
    a.ny = ny;
    a.dy = dy;
    a.Tlist = S.table;
    a.qs2 = S.table + nT;
    a.TA = S.TA;
    a.TB = S.TB;
    a.g2A = c->g2mu2A;
    a.g2B = c->g2mu2B;
    a.yB = S.yB;
    a.inside = S.inside;
    a.prev = S.prev;
    a.row_last = S.row_last;
    a.flags = S.flags;
    launch_ipsat(a, false, c->stream);
    IPG_LAUNCHED(c, a.fluct_x ? 5 : 2);
    int flags = 0;
    IPG_CUDA(c, cudaMemcpyAsync(&flags, S.flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    IPG_TRY(sync(c));
    if (flags & 8) {
        // a fixed point started from a negative rapidity, where the reference
        // carries Q_s from the previous cell: redo both in the sequential order
        launch_ipsat(a, true, c->stream);
        IPG_LAUNCHED(c, 1);
        IPG_CUDA(c, cudaMemcpyAsync(&flags, S.flags, sizeof(int), cudaMemcpyDeviceToHost,
                                    c->stream));
        IPG_TRY(sync(c));
    }
    S.have_T = true;
    c->have_g2mu = true;
    if (rep) {
        launch_ipsat_averages(a, S.col, S.col + 3 * (size_t)nA,
                              std::sqrt(0.1 * p->sigmaNN / M_PI), c->partial, c->stream);
        IPG_LAUNCHED(c, 1);
        std::vector<double> part(296 * 8);
        IPG_CUDA(c, cudaMemcpyAsync(part.data(), c->partial, sizeof(double) * part.size(),
                                    cudaMemcpyDeviceToHost, c->stream));
        IPG_TRY(sync(c));
        double sum[8] = {0};
        for (int blk = 0; blk < 296; blk++)
            for (int k = 0; k < 8; k++) sum[k] += part[8 * blk + k];
        const double cnt = sum[4];
        std::memset(rep, 0, sizeof(*rep));
        rep->Npart = Npart;
        rep->Ncoll = Ncoll;
        rep->Tpp = sum[6];
        rep->average_Qs = cnt > 0 ? std::sqrt(sum[1] / cnt) : 0.;
        rep->average_Qs_avg = cnt > 0 ? std::sqrt(sum[3] / cnt) : 0.;
        rep->average_Qs_min = cnt > 0 ? std::sqrt(sum[2] / cnt) : 0.;
        rep->Qs2min_ST = sum[5] * c->a * c->a / kHbarc / kHbarc;
        rep->overlap_cells = (int)cnt;
        rep->flags = flags;
    }
    return IPG_OK;
}

ipg_status ipg_get_thickness(ipg_ctx *c, double *TA, double *TB) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->ips.have_T) return fail(c, IPG_ERR_STATE, "no IP-Sat maps set");
    if (TA)
        IPG_CUDA(c, cudaMemcpyAsync(TA, c->ips.TA, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                    c->stream));
    if (TB)
        IPG_CUDA(c, cudaMemcpyAsync(TB, c->ips.TB, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                                    c->stream));
    return sync(c);
}

ipg_status ipg_get_g2mu(ipg_ctx *c, double *g2mu2A, double *g2mu2B) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->have_g2mu) return fail(c, IPG_ERR_STATE, "no g2mu maps set");
    if (g2mu2A)
        IPG_CUDA(c, cudaMemcpy(g2mu2A, c->g2mu2A, c->n * sizeof(double), cudaMemcpyDeviceToHost));
    if (g2mu2B)
        IPG_CUDA(c, cudaMemcpy(g2mu2B, c->g2mu2B, c->n * sizeof(double), cudaMemcpyDeviceToHost));
    return IPG_OK;
}

ipg_status ipg_set_noise(ipg_ctx *c, const double *A, const double *B) {
    if (!c || !A || !B) return fail(c, IPG_ERR_BAD_CONFIG, "null argument");
    const size_t cnt = (size_t)c->cfg.Ny * c->n * 8;
    if (!c->xiA_own) {
        IPG_TRY(dalloc(c, &c->xiA_own, cnt));
        IPG_TRY(dalloc(c, &c->xiB_own, cnt));
    }
    IPG_CUDA(c, cudaMemcpyAsync(c->xiA_own, A, sizeof(double) * cnt,
                                cudaMemcpyHostToDevice, c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(c->xiB_own, B, sizeof(double) * cnt,
                                cudaMemcpyHostToDevice, c->stream));
    c->xiA = c->xiA_own;
    c->xiB = c->xiB_own;
    c->have_noise = true;
    c->device_noise = false;
    return IPG_OK;
}

ipg_status ipg_set_noise_device(ipg_ctx *c, const double *A, const double *B) {
    if (!c || !A || !B) return fail(c, IPG_ERR_BAD_CONFIG, "null argument");
    // colour pairs are read as 16-byte vectors
    if (((uintptr_t)A | (uintptr_t)B) & 15)
        return fail(c, IPG_ERR_BAD_CONFIG, "noise arrays must be 16-byte aligned");
    c->xiA = A;
    c->xiB = B;
    c->have_noise = true;
    c->device_noise = false;
    return IPG_OK;
}

ipg_status ipg_use_device_noise(ipg_ctx *c) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    c->xiA = c->xiB = nullptr;
    c->have_noise = true;
    c->device_noise = true;
    return IPG_OK;
}

ipg_status ipg_draw_device_noise(ipg_ctx *c, int nucleus, int sheet_first, int sheet_count,
                                 double *xi) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!xi || nucleus < 0 || nucleus > 1 || sheet_first < 0 || sheet_count < 0 ||
        sheet_first + sheet_count > c->cfg.Ny)
        return fail(c, IPG_ERR_BAD_CONFIG, "noise draw: nucleus %d, sheets [%d, %d) of %d",
                    nucleus, sheet_first, sheet_first + sheet_count, c->cfg.Ny);
    // staged through the initial-condition work buffer: work_sheets sheets of
    // 4 complex channels are 8 doubles a site and sheet
    double *stage = reinterpret_cast<double *>(c->work);
    const size_t per_sheet = 8 * c->n;
    for (int k0 = 0; k0 < sheet_count; k0 += c->work_sheets) {
        const int ns = std::min(c->work_sheets, sheet_count - k0);
        launch_draw_noise(c->N, sheet_first + k0, ns, c->cfg.seed, (uint32_t)nucleus, stage,
                          c->stream);
        IPG_LAUNCHED(c, 1);
        IPG_CUDA(c, cudaMemcpyAsync(xi + (size_t)k0 * per_sheet, stage,
                                    sizeof(double) * per_sheet * ns, cudaMemcpyDeviceToHost,
                                    c->stream));
    }
    return sync(c);
}

// The initial conditions on the context's stream, without waiting for them
// (init_finish waits); from_wilson: V_A and V_B were loaded with
// ipg_set_field, skip setV
static ipg_status init_enqueue(ipg_ctx *c, bool from_wilson) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!from_wilson && (!c->have_g2mu || !c->have_noise))
        return fail(c, IPG_ERR_STATE, "set g2mu and noise before ipg_init_fields");
    const size_t n = c->n;
    const int N = c->N;
    cudaEvent_t *e = c->ie;
    c->init_from_wilson = from_wilson;
    IPG_CUDA(c, cudaEventRecord(e[0], c->stream));
    // scal[38]: set by a step kernel whose bounded wait gave up
    IPG_CUDA(c, cudaMemsetAsync(c->scal + 38, 0, sizeof(double), c->stream));

    // Wilson lines, nucleus A then B (Init.cpp:1688-1847)
    int batch = 0;
    for (int nuc = 0; nuc < (from_wilson ? 0 : 2); nuc++) {
        C<double> *V = nuc ? c->VB : c->VA;
        k_identity<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, V);
        IPG_LAUNCHED(c, 1);
        WilsonArgs w;
        w.N = N;
        w.logN = c->logN;
        w.Ny = c->cfg.Ny;
        w.g = c->cfg.g;
        w.g2mu2 = nuc ? c->g2mu2B : c->g2mu2A;
        w.xi = nuc ? c->xiB : c->xiA;
        w.philox_key = c->cfg.seed;
        w.nucleus = (uint32_t)nuc;
        w.twiddle = c->twiddle;
        w.green = c->green;
        w.amp = c->amp;
        w.work = c->work;
        w.V = V;
        // the FP32 form transforms in FP32: twice the sheets fit a work buffer
        w.fp32 = is_fp32(c) ? 1 : 0;
        w.twiddle32 = c->twiddle32;
        w.green32 = c->green32;
        const int sheets = w.fp32 ? 2 * c->work_sheets : c->work_sheets;
        launch_wilson_amp(w, c->stream);
        IPG_LAUNCHED(c, 1);
        for (int k0 = 0; k0 < c->cfg.Ny; k0 += sheets, batch++) {
            const int ns = std::min(sheets, c->cfg.Ny - k0);
            const int i = batch & 1;
            w.work = i ? c->work2 : c->work;
            // the buffer is free once the product of two batches ago has read it
            if (batch >= 2) IPG_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_prod[i], 0));
            w.no_product = 1;
            launch_wilson_sheets(w, k0, ns, c->stream);
            IPG_CUDA(c, cudaEventRecord(c->ev_fft[i], c->stream));
            IPG_CUDA(c, cudaStreamWaitEvent(c->stream_v, c->ev_fft[i], 0));
            w.no_product = 0;
            launch_wilson_product(w, ns, c->stream_v);
            IPG_CUDA(c, cudaEventRecord(c->ev_prod[i], c->stream_v));
            IPG_LAUNCHED(c, 4);
        }
    }
    if (batch > 0) {
        // V_A, V_B complete before anything else on the context stream
        IPG_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_prod[(batch - 1) & 1], 0));
    }
    IPG_CUDA(c, cudaEventRecord(e[1], c->stream));

    // tau = 0 links (Init.cpp:2462-2517)
    launch_link_products(N, c->VA, c->VB, c->u1x, c->u2x, c->u1y, c->u2y, c->stream);
    IPG_LAUNCHED(c, 1);
    NewtonArgs na;
    na.N = N;
    na.max_iter = c->cfg.newton_max_iterations;
    na.max_restart = c->cfg.newton_max_restarts;
    na.tol = c->cfg.newton_tolerance;
    na.alpha = c->newton_alpha;
    na.mode = c->cfg.newton_mode;
    na.philox_key = c->cfg.seed ^ 0x5DEECE66DULL;
    na.u1x = c->u1x;
    na.u2x = c->u2x;
    na.u1y = c->u1y;
    na.u2y = c->u2y;
    na.ux = c->s64.ux;
    na.uy = c->s64.uy;
    na.iters = c->newton_iters;
    na.status = c->newton_status;
    launch_newton(na, c->stream);
    IPG_LAUNCHED(c, 1);
    IPG_CUDA(c, cudaEventRecord(e[2], c->stream));

    // initial fields: pi from the minus stencil, E = phi = 0 (Init.cpp:2521-2690)
    launch_initial_pi(N, c->cfg.g, c->u1x, c->u2x, c->u1y, c->u2y, c->s64.ux,
                      c->s64.uy, c->s64.pi, c->stream);
    IPG_LAUNCHED(c, 1);
    IPG_CUDA(c, cudaMemsetAsync(c->s64.e1, 0, sizeof(double) * 8 * n, c->stream));
    IPG_CUDA(c, cudaMemsetAsync(c->s64.e2, 0, sizeof(double) * 8 * n, c->stream));
    IPG_CUDA(c, cudaMemsetAsync(c->s64.phi, 0, sizeof(double) * 9 * n, c->stream));
    IPG_TRY(to_fp32_if_needed(c));
    launch_newton_stats(2 * n, c->newton_iters, c->newton_status, c->partial,
                        c->scal + 40, c->stream);
    IPG_LAUNCHED(c, 2);
    IPG_CUDA(c, cudaEventRecord(e[3], c->stream));
    IPG_CUDA(c, cudaMemcpyAsync(c->h_scal + 48, c->scal + 40, 4 * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    return IPG_OK;
}

static ipg_status init_finish(ipg_ctx *c, ipg_init_report *rep) {
    const size_t n = c->n;
    cudaEvent_t *e = c->ie;
    IPG_TRY(sync(c));
    const double *ns = c->h_scal + 48;
    const int mx = (int)ns[0], restarted = (int)ns[2], failed = (int)ns[3];
    const double sum = ns[1];
    if (rep) {
        rep->newton_links = (int)(2 * n);
        rep->newton_restarted = restarted;
        rep->newton_failed = failed;
        rep->newton_max_iterations = mx;
        rep->newton_mean_iterations = sum / (2.0 * n);
        float ms;
        cudaEventElapsedTime(&ms, e[0], e[1]);
        rep->ms_wilson = ms;
        cudaEventElapsedTime(&ms, e[1], e[2]);
        rep->ms_newton = ms;
        cudaEventElapsedTime(&ms, e[2], e[3]);
        rep->ms_fields = ms;
    }
    c->initialized = true;
    c->init_from_inputs = !c->init_from_wilson;
    c->half_done = false;
    c->finished = false;
    c->it = 0;
    if (failed)
        return fail(c, IPG_ERR_NEWTON_NONCONVERGED,
                    "%d of %zu links did not converge", failed, 2 * n);
    return IPG_OK;
}

ipg_status ipg_init_fields(ipg_ctx *c, ipg_init_report *rep) {
    IPG_TRY(init_enqueue(c, false));
    return init_finish(c, rep);
}

ipg_status ipg_init_from_wilson_lines(ipg_ctx *c, ipg_init_report *rep) {
    IPG_TRY(init_enqueue(c, true));
    return init_finish(c, rep);
}

ipg_status ipg_evolve(ipg_ctx *c, int steps) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->initialized || c->finished)
        return fail(c, IPG_ERR_STATE, "ipg_evolve needs fresh initial fields");
    if (steps < 0) return fail(c, IPG_ERR_BAD_CONFIG, "steps < 0");
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int launched = 0;
    if (!c->half_done) {
        IPG_TRY(step(c, 0., c->dtau, c->dtau, 0, 1));
        c->half_done = true;
        launched++;
    }
    for (int k = 0; k < steps; k++) {
        const int itn = c->it + 1;
        IPG_TRY(step(c, itn * c->dtau, c->dtau, c->dtau, 1, 1));
        c->it = itn;
        launched++;
    }
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    IPG_TRY(sync(c));
    c->last_leapfrog_ms = elapsed(c);
    c->last_leapfrog_launches = launched;
    return IPG_OK;
}

ipg_status ipg_run(ipg_ctx *c, ipg_result *res) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->initialized || c->half_done || c->finished)
        return fail(c, IPG_ERR_STATE, "ipg_run needs fresh initial fields");
    IPG_TRY(run_evolution(c));
    IPG_TRY(observables_enqueue(c));
    return observables_finish(c, res);
}

ipg_status ipg_eccentricity_report(ipg_ctx *c, double QsmuRatio, double QsmuRatioB,
                                   ipg_ecc_report *out) {
    if (!c || !out) return IPG_ERR_BAD_CONFIG;
    if (!c->finished) return fail(c, IPG_ERR_STATE, "call ipg_run first");
    if (!c->ecc3) IPG_TRY(dalloc(c, &c->ecc3, 8));
    const int N = c->N;
    const double L = c->cfg.L, a = c->a;
    IPG_TRY(wait_observable_copies(c));
    launch_eccentricity_extras(N, L, a, c->eps, c->u4, c->g2mu2A, c->g2mu2B, c->scal + 0,
                               c->partial, c->ecc3, c->stream);
    IPG_LAUNCHED(c, 2);
    double v[8];
    IPG_CUDA(c, cudaMemcpyAsync(v, c->ecc3, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    IPG_TRY(sync(c));
    const double *s1 = c->h_scal, *s2 = c->h_scal + 8;  // copied by ipg_run
    const double avx = s1[0] / s1[2], avy = s1[1] / s1[2];
    out->tau = c->itmax * a * c->dtau;
    out->r_rms = std::sqrt(s2[1] / v[2]);
    out->max_x = v[6] > 0 ? -L / 2. + a * (v[6] - 1.) - avx : 0.;
    out->max_y = v[7] > 0 ? -L / 2. + a * (v[7] - 1.) - avy : 0.;
    out->area = v[3] * a * a;
    out->Rbar = 1. / std::sqrt(1. / (v[0] / v[2]) + 1. / (v[1] / v[2]));
    out->avg_eps = v[4] * kHbarc / v[3];
    out->avg_qs2a_qs2b = v[5] * QsmuRatio * QsmuRatio * QsmuRatioB * QsmuRatioB / a / a / a / a /
                         v[3] * kHbarc;
    return IPG_OK;
}

ipg_status ipg_gauge_fix(ipg_ctx *c, int max_iterations, ipg_gauge_report *rep) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->initialized) return fail(c, IPG_ERR_STATE, "no fields: call ipg_init_fields first");
    if (max_iterations < 0) return fail(c, IPG_ERR_BAD_CONFIG, "max_iterations < 0");
    IPG_TRY(fields64(c));
    return gauge_fix_run(c, max_iterations, rep);
}

ipg_status ipg_multiplicity(ipg_ctx *c, const ipg_multiplicity_params *p,
                            ipg_multiplicity_result *out) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    return multiplicity_run(c, p, out);
}

ipg_status ipg_run_multiplicity(ipg_ctx *c, const ipg_multiplicity_params *p, ipg_result *res,
                                ipg_multiplicity_result *first, ipg_multiplicity_result *last) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->initialized || c->half_done || c->finished)
        return fail(c, IPG_ERR_STATE, "ipg_run_multiplicity needs fresh initial fields");
    // Evolution::run: the first step, the spectrum at it = 1 (when it is not
    // also the last step), the remaining steps, the observables at itmax with
    // the final half step, then the spectrum at itmax
    const int itmax = c->itmax;
    double ms = 0;
    if (itmax >= 2) {
        IPG_TRY(ipg_evolve(c, 1));
        ms += c->last_leapfrog_ms;
        ipg_multiplicity_result m1;
        IPG_TRY(multiplicity_run(c, p, &m1));
        if (first) *first = m1;
        if (m1.dNdy == 0.)
            return fail(c, IPG_NO_COLLISION, "no collision happened: dN/dy at it = 1 is zero");
        IPG_TRY(ipg_evolve(c, itmax - 2));
        ms += c->last_leapfrog_ms;
    } else {
        IPG_TRY(run_evolution(c));
        ms += c->last_leapfrog_ms;
    }
    c->last_leapfrog_ms = ms;
    c->last_leapfrog_launches = itmax;
    IPG_TRY(observables_enqueue(c));
    IPG_TRY(observables_finish(c, res));
    ipg_multiplicity_result m;
    IPG_TRY(multiplicity_run(c, p, &m));
    if (last) *last = m;
    if (itmax < 2 && first) *first = m;
    return IPG_OK;
}

ipg_status ipg_multiplicity_finish(double dN, double dE, const double *n_sum,
                                   const double *E_sum, const int *count, double a,
                                   const ipg_multiplicity_params *p, ipg_multiplicity_result *out) {
    if (!n_sum || !E_sum || !count || !out || !(a > 0)) return IPG_ERR_BAD_CONFIG;
    ipg_multiplicity_params prm{};
    if (p) prm = *p;
    // Evolution.cpp:2874-2960: bin averages, the binned integrals and the
    // cuts, in the reference's bin order and operation order
    const int bins = kKtBins;
    const double dkt = 2.83 / static_cast<double>(bins);
    const double m = prm.jacobian_m;
    const double y = prm.rapidity;
    double dN2 = 0., dE2 = 0., dNc = 0., dEc = 0., dNc2 = 0., dEc2 = 0.;
    for (int ik = 0; ik < bins; ik++) {
        double nk = n_sum[ik], Ek = E_sum[ik];
        if (count[ik] > 0) {
            nk = nk / static_cast<double>(count[ik]);
            Ek = Ek / static_cast<double>(count[ik]);
            if (prm.use_pseudorapidity == 0) {
                dN2 += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                dE2 += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                if (ik * dkt / a * kHbarc > 3.) {
                    dNc += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                    dEc += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                }
                if (ik * dkt / a * kHbarc > 6.) {
                    dNc2 += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                    dEc2 += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI;
                }
            } else {
                const double pt = (ik + 0.5) * dkt / a * kHbarc;
                const double den = std::sqrt(std::pow(std::cosh(y), 2.) + m * m / (pt * pt));
                dN2 += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                dE2 += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                if (ik * dkt / a * kHbarc > 3.) {
                    dNc += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                    dEc += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                }
                if (ik * dkt / a * kHbarc > 6.) {
                    dNc2 += nk * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                    dEc2 += Ek * (ik + 0.5) * dkt * dkt * 2. * M_PI * std::cosh(y) / den;
                }
            }
        }
        out->n_kt[ik] = count[ik] > 0 ? nk : 0.;
        out->E_kt[ik] = count[ik] > 0 ? Ek : 0.;
        out->count_kt[ik] = count[ik];
    }
    if (prm.use_pseudorapidity == 1) {
        // Evolution.cpp:3098-3108: the k sums take the Jacobian at the mean
        // p_T estimate P(sqrt(s))
        const double P = 0.13 + 0.32 * std::pow(prm.roots / 1000., 0.115);
        const double J = std::cosh(y) / (std::sqrt(std::pow(std::cosh(y), 2.) + m * m / (P * P)));
        dN *= J;
        dE *= J;
    }
    out->dNdy = dN;
    out->dEdy = dE;
    out->dNdy_binned = dN2;
    out->dEdy_binned = dE2;
    out->dNdy_cut3 = dNc;
    out->dEdy_cut3 = dEc;
    out->dNdy_cut6 = dNc2;
    out->dEdy_cut6 = dEc2;
    out->mean_pt = dE / dN;
    return IPG_OK;
}

ipg_status ipg_get_observables(ipg_ctx *c, double *eps, double *u4,
                               double *pi10, double *T10) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->finished) return fail(c, IPG_ERR_STATE, "call ipg_run first");
    const size_t n = c->n;
    // enqueued on the context's stream, one wait at the end (full speed when
    // the destinations are pinned; pageable ones are staged by the driver)
    const auto d2h = cudaMemcpyDeviceToHost;
    if (eps) IPG_CUDA(c, cudaMemcpyAsync(eps, c->eps, sizeof(double) * n, d2h, c->stream));
    if (u4) IPG_CUDA(c, cudaMemcpyAsync(u4, c->u4, sizeof(double) * 4 * n, d2h, c->stream));
    if (pi10) IPG_CUDA(c, cudaMemcpyAsync(pi10, c->pi10, sizeof(double) * 10 * n, d2h, c->stream));
    if (T10) IPG_CUDA(c, cudaMemcpyAsync(T10, c->T10, sizeof(double) * 10 * n, d2h, c->stream));
    IPG_TRY(sync(c));
    return IPG_OK;
}

ipg_status ipg_get_observables_async(ipg_ctx *c, double *eps, double *u4, double *pi10,
                                     double *T10) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->finished) return fail(c, IPG_ERR_STATE, "call ipg_run first");
    const size_t n = c->n;
    const auto d2h = cudaMemcpyDeviceToHost;
    cudaStream_t s = c->stream_copy;
    IPG_CUDA(c, cudaEventRecord(c->ev_obs_ready, c->stream));
    IPG_CUDA(c, cudaStreamWaitEvent(s, c->ev_obs_ready, 0));
    if (eps) IPG_CUDA(c, cudaMemcpyAsync(eps, c->eps, sizeof(double) * n, d2h, s));
    if (u4) IPG_CUDA(c, cudaMemcpyAsync(u4, c->u4, sizeof(double) * 4 * n, d2h, s));
    if (pi10) IPG_CUDA(c, cudaMemcpyAsync(pi10, c->pi10, sizeof(double) * 10 * n, d2h, s));
    if (T10) IPG_CUDA(c, cudaMemcpyAsync(T10, c->T10, sizeof(double) * 10 * n, d2h, s));
    IPG_CUDA(c, cudaEventRecord(c->ev_obs_copied, s));
    c->obs_copy_pending = true;
    return IPG_OK;
}

ipg_status ipg_wait_observables(ipg_ctx *c) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (c->obs_copy_pending) IPG_CUDA(c, cudaEventSynchronize(c->ev_obs_copied));
    return IPG_OK;
}

ipg_status ipg_write_outputs(ipg_ctx *c, const char *hydro_path, const char *tmunu_path,
                             int sizeOutput, double LOutput, int etaSizeOutput,
                             double detaOutput, int it, double dtau, double gfactor,
                             double *Etot) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->finished) return fail(c, IPG_ERR_STATE, "call ipg_run first");
    if (sizeOutput < 1 || etaSizeOutput < 0)
        return fail(c, IPG_ERR_BAD_CONFIG, "sizeOutput < 1 or etaSizeOutput < 0");
    OutputGrid g;
    g.N = c->N;
    g.L = c->cfg.L;
    g.a = g.L / g.N;
    g.hx = sizeOutput;
    g.heta = etaSizeOutput;
    g.hL = LOutput;
    g.ha = LOutput / sizeOutput;
    g.deta = detaOutput;
    g.it = it;
    g.dtau = dtau;
    g.gfactor = gfactor;
    g.tau0 = it * dtau * g.a;
    const OutputFields f{c->eps, c->u4, c->pi10, c->T10};
    auto &o = c->out;
    const long long hydro_lines = (long long)g.heta * g.hx * g.hx;
    const long long tmunu_lines = (long long)g.hx * g.hx;
    const long long need = std::max(hydro_path ? hydro_lines : 0, tmunu_path ? tmunu_lines : 0);
    if (need > o.cap_lines) {
        for (void *p : {(void *)o.chunks, (void *)o.text, (void *)o.chunk_len,
                        (void *)o.chunk_off, (void *)o.term, (void *)o.bad})
            if (p) cudaFree(p);
        for (void *p : {(void *)o.h_text, (void *)o.h_term, (void *)o.h_small})
            if (p) cudaFreeHost(p);
        o = {};
        const size_t bytes = output_text_capacity(need);
        const int chunks = output_text_chunks(need);
        IPG_CUDA(c, cudaMalloc(&o.chunks, bytes));
        IPG_CUDA(c, cudaMalloc(&o.text, bytes));
        IPG_CUDA(c, cudaMalloc(&o.chunk_len, sizeof(int) * chunks));
        IPG_CUDA(c, cudaMalloc(&o.chunk_off, sizeof(long long) * (chunks + 1)));
        IPG_CUDA(c, cudaMalloc(&o.term, sizeof(double) * need));
        IPG_CUDA(c, cudaMalloc(&o.bad, sizeof(int)));
        IPG_CUDA(c, cudaMallocHost(&o.h_text, bytes));
        IPG_CUDA(c, cudaMallocHost(&o.h_term, sizeof(double) * need));
        IPG_CUDA(c, cudaMallocHost(&o.h_small, 2 * sizeof(long long)));
        o.cap_lines = need;
    }
    // one file: body on the GPU, then header + body with one fwrite each; a
    // body that needs the host formatter goes through the host writer
    auto one = [&](int kind, const char *path, long long lines) -> ipg_status {
        IPG_CUDA(c, cudaMemsetAsync(o.bad, 0, sizeof(int), c->stream));
        launch_output_text(kind, g, f, lines, o.chunks, o.chunk_len, o.chunk_off, o.text,
                           o.term, o.bad, c->stream);
        IPG_LAUNCHED(c, lines > 0 ? 3 : 0);
        const int chunks = output_text_chunks(lines);
        long long *hs = o.h_small;
        hs[0] = 0;
        hs[1] = 0;
        if (lines > 0)
            IPG_CUDA(c, cudaMemcpyAsync(&hs[0], o.chunk_off + chunks, sizeof(long long),
                                        cudaMemcpyDeviceToHost, c->stream));
        IPG_CUDA(c, cudaMemcpyAsync(&hs[1], o.bad, sizeof(int), cudaMemcpyDeviceToHost,
                                    c->stream));
        IPG_TRY(sync(c));
        if ((int)hs[1] != 0) {
            const size_t n = c->n;
            std::vector<double> eps(n), u4(4 * n), pi10(10 * n), T10(10 * n);
            IPG_TRY(ipg_get_observables(c, eps.data(), u4.data(), pi10.data(), T10.data()));
            return kind == 0 ? ipg_write_hydro(path, g.N, g.L, g.hx, g.hL, g.heta, g.deta, it,
                                               dtau, eps.data(), u4.data(), pi10.data(),
                                               gfactor, Etot)
                             : ipg_write_tmunu(path, g.N, g.L, g.hx, g.hL, g.heta, g.deta, it,
                                               dtau, T10.data(), gfactor);
        }
        const size_t body = (size_t)hs[0];
        if (body)
            IPG_CUDA(c, cudaMemcpyAsync(o.h_text, o.text, body, cudaMemcpyDeviceToHost,
                                        c->stream));
        if (kind == 0 && Etot && lines > 0)
            IPG_CUDA(c, cudaMemcpyAsync(o.h_term, o.term, sizeof(double) * lines,
                                        cudaMemcpyDeviceToHost, c->stream));
        IPG_TRY(sync(c));
        const std::string head =
            kind == 0 ? hydro_header(g.N, g.L, g.hx, g.hL, g.heta, g.deta, it, dtau)
                      : tmunu_header(g.N, g.L, g.hx, g.hL, g.heta, g.deta);
        FILE *fp = std::fopen(path, "wb");
        if (!fp) return fail(c, IPG_ERR_BAD_CONFIG, "cannot open %s", path);
        bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
        ok = ok && std::fwrite(o.h_text, 1, body, fp) == body;
        ok = (std::fclose(fp) == 0) && ok;
        if (!ok) return fail(c, IPG_ERR_BAD_CONFIG, "writing %s failed", path);
        if (kind == 0 && Etot) {
            // the reference's running sum, in its loop order
            double etot = 0.;
            for (long long i = 0; i < lines; i++) etot += o.h_term[i];
            *Etot = etot;
        }
        return IPG_OK;
    };
    if (hydro_path) IPG_TRY(one(0, hydro_path, hydro_lines));
    if (tmunu_path) IPG_TRY(one(1, tmunu_path, tmunu_lines));
    return IPG_OK;
}

ipg_status ipg_get_field(ipg_ctx *c, int which, double *out) {
    if (!c || !out) return IPG_ERR_BAD_CONFIG;
    IPG_TRY(sync(c));
    const size_t n = c->n;
    if (which == IPG_VA || which == IPG_VB || which == IPG_UX || which == IPG_UY) {
        if (which == IPG_UX || which == IPG_UY) IPG_TRY(state64(c));
        const C<double> *src = which == IPG_VA ? c->VA
                               : which == IPG_VB ? c->VB
                               : which == IPG_UX ? c->s64.ux
                                                 : c->s64.uy;
        std::vector<double> pl(18 * n);
        IPG_CUDA(c, cudaMemcpy(pl.data(), src, sizeof(double) * 18 * n,
                               cudaMemcpyDeviceToHost));
        planes_to_sites_m3(pl, n, out);
        return IPG_OK;
    }
    IPG_TRY(state64(c));
    const bool tl = (which == IPG_E1 || which == IPG_E2);
    const double *src = which == IPG_E1 ? c->s64.e1
                        : which == IPG_E2 ? c->s64.e2
                        : which == IPG_PHI ? c->s64.phi
                        : which == IPG_PI ? c->s64.pi
                                          : nullptr;
    if (!src) return fail(c, IPG_ERR_BAD_CONFIG, "unknown field %d", which);
    std::vector<double> pl((tl ? 8 : 9) * n);
    IPG_CUDA(c, cudaMemcpy(pl.data(), src, sizeof(double) * pl.size(),
                           cudaMemcpyDeviceToHost));
    herm_to_sites(pl, n, tl, out);
    return IPG_OK;
}

ipg_status ipg_set_field(ipg_ctx *c, int which, const double *in) {
    if (!c || !in) return IPG_ERR_BAD_CONFIG;
    const size_t n = c->n;
    c->init_from_inputs = false;
    IPG_TRY(sync(c));
    if (which == IPG_VA || which == IPG_VB || which == IPG_UX || which == IPG_UY) {
        C<double> *dst = which == IPG_VA ? c->VA
                         : which == IPG_VB ? c->VB
                         : which == IPG_UX ? c->s64.ux
                                           : c->s64.uy;
        std::vector<double> pl(18 * n);
        for (size_t p = 0; p < n; p++)
            for (int k = 0; k < 9; k++) {
                pl[2 * (k * n + p)] = in[18 * p + 2 * k];
                pl[2 * (k * n + p) + 1] = in[18 * p + 2 * k + 1];
            }
        IPG_CUDA(c, cudaMemcpy(dst, pl.data(), sizeof(double) * 18 * n,
                               cudaMemcpyHostToDevice));
        return IPG_OK;
    }
    const bool tl = (which == IPG_E1 || which == IPG_E2);
    double *dst = which == IPG_E1 ? c->s64.e1
                  : which == IPG_E2 ? c->s64.e2
                  : which == IPG_PHI ? c->s64.phi
                  : which == IPG_PI ? c->s64.pi
                                    : nullptr;
    if (!dst) return fail(c, IPG_ERR_BAD_CONFIG, "unknown field %d", which);
    std::vector<double> pl;
    sites_to_herm(in, n, tl, pl);
    IPG_CUDA(c, cudaMemcpy(dst, pl.data(), sizeof(double) * pl.size(),
                           cudaMemcpyHostToDevice));
    return IPG_OK;
}

ipg_status ipg_mark_initialized(ipg_ctx *c) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    IPG_TRY(to_fp32_if_needed(c));
    IPG_TRY(sync(c));
    c->initialized = true;
    c->half_done = false;
    c->finished = false;
    c->it = 0;
    return IPG_OK;
}

ipg_status ipg_get_newton_iterations(ipg_ctx *c, int *iters, int *status) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    const size_t n = c->n;
    if (iters) IPG_CUDA(c, cudaMemcpy(iters, c->newton_iters, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost));
    if (status) IPG_CUDA(c, cudaMemcpy(status, c->newton_status, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost));
    return IPG_OK;
}

ipg_status ipg_last_leapfrog_ms(ipg_ctx *c, double *ms, int *launches) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (ms) *ms = c->last_leapfrog_ms;
    if (launches) *launches = c->last_leapfrog_launches;
    return IPG_OK;
}

ipg_status ipg_kernel_launches(const ipg_ctx *c, long long *count) {
    if (!c || !count) return IPG_ERR_BAD_CONFIG;
    *count = c->launches;
    return IPG_OK;
}

}  // extern "C"

// Adjoint of the initial conditions: from the adjoints of the tau = 0 state
// (c->aw.adj, projected) through the initial pi and the Newton links to U1,
// U2, V_A, V_B, then sheet by sheet backwards through the Wilson-line
// products (each sheet's A_k recomputed by the Poisson pipeline), the
// Poisson map (self-adjoint) and rho = g sqrt(g2mu2 / Ny) xi.
namespace {
ipg_status backward_inputs(ipg_ctx *c, double *grad_g2mu, double *grad_rho) {
    auto &A = c->aw;
    const size_t n = c->n;
    const int N = c->N, Ny = c->cfg.Ny;
    if (!A.b1x) {
        for (C<double> **p : {&A.b1x, &A.b2x, &A.b1y, &A.b2y, &A.vbA, &A.vbB, &A.vcur, &A.vcur2})
            IPG_TRY(dalloc(c, p, 9 * n));
        IPG_TRY(dalloc(c, &A.g2mu_bar, 2 * n));
        IPG_TRY(dalloc(c, &A.amp2, n));
    }
    if (grad_rho && !A.rho_all) IPG_TRY(dalloc(c, &A.rho_all, 16 * (size_t)Ny * n));
    for (C<double> *p : {A.b1x, A.b2x, A.b1y, A.b2y, A.vbA, A.vbB})
        IPG_CUDA(c, cudaMemsetAsync(p, 0, 9 * n * sizeof(C<double>), c->stream));
    IPG_CUDA(c, cudaMemsetAsync(A.g2mu_bar, 0, 2 * n * sizeof(double), c->stream));
    AdjInitArgs ai;
    ai.N = N;
    ai.g = c->cfg.g;
    ai.u1x = c->u1x;
    ai.u2x = c->u2x;
    ai.u1y = c->u1y;
    ai.u2y = c->u2y;
    // the tau = 0 links kept by ipg_forward (FP64: checkpoint 0; FP32
    // adjoint: the FP64 copy in work state 0)
    ai.ux = A.fp32 ? A.w[0].ux : A.cp[0].ux;
    ai.uy = A.fp32 ? A.w[0].uy : A.cp[0].uy;
    ai.VA = c->VA;
    ai.VB = c->VB;
    ai.alpha = c->newton_alpha;
    ai.adj = A.adj;
    ai.b1x = A.b1x;
    ai.b2x = A.b2x;
    ai.b1y = A.b1y;
    ai.b2y = A.b2y;
    ai.vbA = A.vbA;
    ai.vbB = A.vbB;
    launch_adjoint_init_links(ai, c->stream);
    IPG_LAUNCHED(c, 3);
    // the two nuclei are independent from here on: nucleus A on the main
    // stream with work, nucleus B on stream_v with work2 and buffers of its
    // own, joined at the end (each chain alone fills under one wave of the
    // GPU on the lattices the adjoint runs on)
    IPG_CUDA(c, cudaEventRecord(c->ev_nuc_fork, c->stream));
    IPG_CUDA(c, cudaStreamWaitEvent(c->stream_v, c->ev_nuc_fork, 0));
    for (int nuc = 0; nuc < 2; nuc++) {
        cudaStream_t st = nuc ? c->stream_v : c->stream;
        double2 *work = nuc ? c->work2 : c->work;
        C<double> *vcur = nuc ? A.vcur2 : A.vcur;
        IPG_CUDA(c, cudaMemcpyAsync(vcur, nuc ? c->VB : c->VA, 9 * n * sizeof(C<double>),
                                    cudaMemcpyDeviceToDevice, st));
        C<double> *vb = nuc ? A.vbB : A.vbA;
        WilsonArgs w;
        w.N = N;
        w.logN = c->logN;
        w.Ny = Ny;
        w.g = c->cfg.g;
        w.g2mu2 = nuc ? c->g2mu2B : c->g2mu2A;
        w.xi = nuc ? c->xiB : c->xiA;
        w.philox_key = c->cfg.seed;
        w.nucleus = (uint32_t)nuc;
        w.twiddle = c->twiddle;
        w.green = c->green;
        w.amp = nuc ? A.amp2 : c->amp;
        w.work = work;
        w.V = vcur;
        w.no_product = 1;
        launch_wilson_amp(w, st);
        IPG_LAUNCHED(c, 1);
        // batches of work_sheets sheets from the top: the transforms of a
        // batch (A_k, then the Poisson map of A_bar_k) run as one launch each,
        // the product recursion and the rho adjoint sheet by sheet in the
        // order k = Ny-1 .. 0 (the accumulation order of g2mu_bar)
        const int S = c->work_sheets;
        for (int kb = Ny; kb > 0; kb -= S) {
            const int k0 = std::max(0, kb - S), ns = kb - k0;
            w.rho_in = nullptr;
            launch_wilson_sheets(w, k0, ns, st);  // slot k - k0 = A_k
            IPG_LAUNCHED(c, 3);
            for (int k = kb - 1; k >= k0; k--) {
                // slot k - k0 becomes A_bar_k
                launch_adjoint_wilson_sheet(N, work + (size_t)(k - k0) * 4 * n, vcur, vb, st);
                IPG_LAUNCHED(c, 1);
            }
            w.rho_in = work;
            launch_poisson_sheets(w, ns, st);  // in place: slot k - k0 = rho_bar_k
            IPG_LAUNCHED(c, 3);
            w.rho_in = nullptr;
            for (int k = kb - 1; k >= k0; k--) {
                WilsonArgs ws = w;
                ws.work = work + (size_t)(k - k0) * 4 * n;
                launch_adjoint_rho(ws, k, A.g2mu_bar + nuc * n,
                                   grad_rho ? A.rho_all + ((size_t)nuc * Ny + k) * n * 8 : nullptr,
                                   st);
                IPG_LAUNCHED(c, 1);
            }
        }
    }
    IPG_CUDA(c, cudaEventRecord(c->ev_nuc_join, c->stream_v));
    IPG_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_nuc_join, 0));
    return IPG_OK;
}
}  // namespace

// ===========================================================================
// Adjoint: forward with checkpoints, reverse sweep with time reversal
// ===========================================================================
extern "C" {

ipg_status ipg_forward(ipg_ctx *c, int checkpoint_every, double *E_T, double *eps2) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (!c->initialized || c->half_done || c->finished)
        return fail(c, IPG_ERR_STATE, "ipg_forward needs the fresh tau = 0 state");
    if (checkpoint_every < 0) return fail(c, IPG_ERR_BAD_CONFIG, "checkpoint_every < 0");
    const size_t n = c->n;
    const int N = c->N;
    const int S = c->itmax;
    auto &A = c->aw;
    if (checkpoint_every == 0) {
        // automatic: every state when the S + 1 states (70 doubles a site
        // each) take at most half of the free device memory, else a
        // checkpoint every ~sqrt(S) steps
        size_t free_b = 0, total_b = 0;
        IPG_CUDA(c, cudaMemGetInfo(&free_b, &total_b));
        const size_t have = A.cp.size() * 70 * n * sizeof(double);  // reused
        const size_t need = (size_t)(S + 1) * 70 * n * sizeof(double);
        checkpoint_every = need <= (free_b + have) / 2
                               ? 1
                               : std::max(2, (int)std::ceil(std::sqrt((double)S)));
    }
    // checkpoint_every = 1 keeps every step's state (S + 1 states): the
    // forward steps from slot s into slot s + 1 and the reverse sweep reads
    // them without time reversal
    const bool store_all = checkpoint_every == 1;
    const int ncp = store_all ? S + 1 : (S - 1) / checkpoint_every + 1;
    auto alloc_state = [&](State<double> &st) -> ipg_status {
        IPG_TRY(dalloc(c, &st.ux, 9 * n));
        IPG_TRY(dalloc(c, &st.uy, 9 * n));
        IPG_TRY(dalloc(c, &st.e1, 8 * n));
        IPG_TRY(dalloc(c, &st.e2, 8 * n));
        IPG_TRY(dalloc(c, &st.phi, 9 * n));
        IPG_TRY(dalloc(c, &st.pi, 9 * n));
        return IPG_OK;
    };
    if (!A.w[0].ux) {
        for (auto &st : A.w) IPG_TRY(alloc_state(st));
        IPG_TRY(dalloc(c, &A.adj.ux, 9 * n));
        IPG_TRY(dalloc(c, &A.adj.uy, 9 * n));
        IPG_TRY(dalloc(c, &A.adj.e1, 9 * n));
        IPG_TRY(dalloc(c, &A.adj.e2, 9 * n));
        IPG_TRY(dalloc(c, &A.adj.phi, 9 * n));
        IPG_TRY(dalloc(c, &A.adj.pi, 9 * n));
        IPG_TRY(dalloc(c, &A.tbar, n));
    }
    while (!is_fp32(c) && (int)A.cp.size() < ncp) {
        State<double> st{};
        IPG_TRY(alloc_state(st));
        A.cp.push_back(st);
    }
    A.k = checkpoint_every;
    A.steps = S;
    A.ready = false;
    A.from_inputs = c->init_from_inputs;
    A.fp32 = is_fp32(c);
    if (A.fp32) {
        // FP32 adjoint: the plain form (full links, no reunitarisation) stepped
        // in FP32 from the FP64 tau = 0 state rounded once
        auto alloc32 = [&](State<float> &st) -> ipg_status {
            IPG_TRY(dalloc(c, &st.ux, 9 * n));
            IPG_TRY(dalloc(c, &st.uy, 9 * n));
            IPG_TRY(dalloc(c, &st.e1, 8 * n));
            IPG_TRY(dalloc(c, &st.e2, 8 * n));
            IPG_TRY(dalloc(c, &st.phi, 9 * n));
            IPG_TRY(dalloc(c, &st.pi, 9 * n));
            return IPG_OK;
        };
        if (!A.w32[0].ux) {
            for (auto &st : A.w32) IPG_TRY(alloc32(st));
            IPG_TRY(dalloc(c, &A.adj32.ux, 9 * n));
            IPG_TRY(dalloc(c, &A.adj32.uy, 9 * n));
            IPG_TRY(dalloc(c, &A.adj32.e1, 9 * n));
            IPG_TRY(dalloc(c, &A.adj32.e2, 9 * n));
            IPG_TRY(dalloc(c, &A.adj32.phi, 9 * n));
            IPG_TRY(dalloc(c, &A.adj32.pi, 9 * n));
            IPG_TRY(dalloc(c, &A.tbar32, n));
        }
        while ((int)A.cp32.size() < (store_all ? S + 1 : ncp)) {
            State<float> st{};
            IPG_TRY(alloc32(st));
            A.cp32.push_back(st);
        }
        while (!store_all && (int)A.seg32.size() < checkpoint_every + 1) {
            State<float> st{};
            IPG_TRY(alloc32(st));
            A.seg32.push_back(st);
        }
    }

    // forward from the tau = 0 state (the context's own state is kept)
    IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    State<double> cur;
    if (A.fp32) {
        // the FP32 bulk form's own steps (deviation storage W = U - 1,
        // reunitarised), from the context's FP32 tau = 0 state
        IPG_TRY(copy_state(c, A.w[0], c->s64));  // FP64 tau = 0 links for the init adjoint
        State<float> c32;
        if (store_all) {
            IPG_TRY(copy_state32(c, A.cp32[0], c->s32));
            for (int s = 0; s < S; s++)
                IPG_TRY(step32_into(c, A.cp32[s], A.cp32[s + 1], evolution_coef(c, s)));
            c32 = A.cp32[S];
        } else {
            IPG_TRY(copy_state32(c, A.w32[0], c->s32));
            c32 = A.w32[0];
            State<float> other = A.w32[1];
            for (int s = 0; s < S; s++) {
                if (s % checkpoint_every == 0)
                    IPG_TRY(copy_state32(c, A.cp32[s / checkpoint_every], c32));
                State<float> out = c32;  // E and pi in place
                out.ux = other.ux;
                out.uy = other.uy;
                out.phi = other.phi;
                IPG_TRY(step32_into(c, c32, out, evolution_coef(c, s)));
                std::swap(c32.ux, other.ux);
                std::swap(c32.uy, other.uy);
                std::swap(c32.phi, other.phi);
            }
        }
        A.fin32 = c32;
        // T^tautau of the final state in FP64 (the loss), from U = 1 + W
        launch_convert_state<float>(n, c32, A.w[2], c->stream);
        IPG_LAUNCHED(c, 1);
        cur = A.w[2];
    } else if (store_all) {
        IPG_TRY(copy_state(c, A.cp[0], c->s64));
        for (int s = 0; s < S; s++) {
            launch_leapfrog_into(c->d_ev, N, A.cp[s], A.cp[s + 1], evolution_coef(c, s),
                                 c->stream);
            IPG_LAUNCHED(c, 1);
        }
        cur = A.cp[S];
    } else {
        IPG_TRY(copy_state(c, A.w[0], c->s64));
        cur = A.w[0];
        C<double> *ux_b = A.w[1].ux, *uy_b = A.w[1].uy;
        double *phi_b = A.w[1].phi;
        for (int s = 0; s < S; s++) {
            if (s % checkpoint_every == 0)
                IPG_TRY(copy_state(c, A.cp[s / checkpoint_every], cur));
            const StepCoef<double> cf = evolution_coef(c, s);
            launch_leapfrog<double>(c->d_ev, N, cur, ux_b, uy_b, phi_b, cf, false, c->stream);
            IPG_LAUNCHED(c, 1);
            std::swap(cur.ux, ux_b);
            std::swap(cur.uy, uy_b);
            std::swap(cur.phi, phi_b);
        }
    }
    A.fin = cur;
    IPG_TRY(wait_observable_copies(c));  // T10 is rewritten below
    TmunuArgs ta;
    ta.N = N;
    ta.g = c->cfg.g;
    ta.tau = S * c->dtau;
    ta.a = c->a;
    ta.s = cur;
    ta.T10 = c->T10;
    launch_tmunu_diag(ta, c->stream);
    IPG_LAUNCHED(c, 1);
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    std::vector<double> ttt(n);
    IPG_CUDA(c, cudaMemcpyAsync(ttt.data(), c->T10, n * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    IPG_TRY(sync(c));
    A.ms_forward = elapsed(c);
    double sum = 0., S6[6] = {0};
    for (size_t p = 0; p < n; p++) {
        sum += ttt[p];
        const int i = (int)(p / N), j = (int)(p % N);
        if (!in_ecc_window(N, i, j)) continue;
        const double w = ttt[p];
        S6[0] += w;
        S6[1] += w * i;
        S6[2] += w * j;
        S6[3] += w * i * i;
        S6[4] += w * j * j;
        S6[5] += w * i * j;
    }
    std::memcpy(A.sums, S6, sizeof(S6));
    A.sum_ttt = sum;
    const double tau_fm = S * c->dtau * c->a;
    A.ET = tau_fm * c->a * c->a * kHbarc * sum;
    A.eps2 = eps2_from_sums(S6, nullptr);
    A.ready = true;
    if (E_T) *E_T = A.ET;
    if (eps2) *eps2 = A.eps2;
    return IPG_OK;
}

ipg_status ipg_adjoint_stats(const ipg_ctx *c, double *ms_forward, double *ms_backward) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    if (ms_forward) *ms_forward = c->aw.ms_forward;
    if (ms_backward) *ms_backward = c->aw.ms_backward;
    return IPG_OK;
}

ipg_status ipg_backward(ipg_ctx *c, double w_ET, double w_eps2, double *grad_state,
                        double *grad_g2mu, double *grad_rho) {
    if (!c) return IPG_ERR_BAD_CONFIG;
    auto &A = c->aw;
    if (!A.ready) return fail(c, IPG_ERR_STATE, "call ipg_forward first");
    if ((grad_g2mu || grad_rho) && !A.from_inputs)
        return fail(c, IPG_ERR_STATE,
                    "input gradients need a tau = 0 state made by ipg_init_fields");
    if ((grad_g2mu || grad_rho) && c->cfg.newton_mode != 0)
        return fail(c, IPG_ERR_STATE,
                    "input gradients differentiate the reference's Newton iteration: "
                    "use newton_mode 0");
    const size_t n = c->n;
    const int N = c->N;
    const int S = A.steps;
    // dL/dTtt_lat per cell: T^tautau in fm^-4 is Ttt_lat / a^4
    const double a4 = std::pow(c->a, 4.);
    const double tau_fm = S * c->dtau * c->a;
    double d6[6];
    eps2_from_sums(A.sums, d6);
    std::vector<double> tb(n);
    for (size_t p = 0; p < n; p++) {
        const int i = (int)(p / N), j = (int)(p % N);
        double v = w_ET * tau_fm * c->a * c->a * kHbarc;
        if (in_ecc_window(N, i, j))
            v += w_eps2 * (d6[0] + d6[1] * i + d6[2] * j + d6[3] * i * i + d6[4] * j * j +
                           d6[5] * i * j);
        tb[p] = v / a4;
    }
    if (A.fp32) {
        // the reverse sweep in FP32 on the plain form's FP32 states, then the
        // tau = 0 adjoint widened to FP64 for the initial conditions
        std::vector<float> tb32(tb.begin(), tb.end());
        IPG_CUDA(c, cudaMemcpyAsync(A.tbar32, tb32.data(), n * sizeof(float),
                                    cudaMemcpyHostToDevice, c->stream));
        IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
        for (C<float> *b : {A.adj32.ux, A.adj32.uy, A.adj32.e1, A.adj32.e2, A.adj32.phi,
                            A.adj32.pi})
            IPG_CUDA(c, cudaMemsetAsync(b, 0, 9 * n * sizeof(C<float>), c->stream));
        launch_adjoint_ttt<float>(N, A.fin32, A.tbar32, A.adj32, c->cfg.g, S * c->dtau,
                                  c->stream);
        IPG_LAUNCHED(c, 1);
        if (A.k == 1) {
            for (int s = S - 1; s >= 0; s--) {
                const StepCoef<double> cf = evolution_coef(c, s);
                launch_adjoint_step<float>(N, A.cp32[s], A.cp32[s + 1], A.adj32, cf, c->stream);
                IPG_LAUNCHED(c, cf.do_pe ? 2 : 1);
            }
        } else {
            // segment by segment from the last: the segment's states are
            // recomputed from its checkpoint with the same FP32 steps as the
            // forward (the exact forward trajectory), then swept backwards
            for (int j = (S - 1) / A.k; j >= 0; j--) {
                const int s0 = j * A.k, s1 = std::min(S, s0 + A.k);
                IPG_TRY(copy_state32(c, A.seg32[0], A.cp32[j]));
                for (int t = s0; t < s1; t++)
                    IPG_TRY(step32_into(c, A.seg32[t - s0], A.seg32[t - s0 + 1],
                                        evolution_coef(c, t)));
                for (int t = s1 - 1; t >= s0; t--) {
                    const StepCoef<double> cf = evolution_coef(c, t);
                    launch_adjoint_step<float>(N, A.seg32[t - s0], A.seg32[t - s0 + 1], A.adj32,
                                               cf, c->stream);
                    IPG_LAUNCHED(c, cf.do_pe ? 2 : 1);
                }
            }
        }
        launch_adjoint_project<float>(n, A.adj32, c->stream);
        launch_adjoint_widen(n, A.adj32, A.adj, c->stream);
        IPG_LAUNCHED(c, 7);
    } else {
        IPG_CUDA(c, cudaMemcpyAsync(A.tbar, tb.data(), n * sizeof(double), cudaMemcpyHostToDevice,
                                    c->stream));
        IPG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
        for (C<double> *b : {A.adj.ux, A.adj.uy, A.adj.e1, A.adj.e2, A.adj.phi, A.adj.pi})
            IPG_CUDA(c, cudaMemsetAsync(b, 0, 9 * n * sizeof(C<double>), c->stream));
        launch_adjoint_ttt<double>(N, A.fin, A.tbar, A.adj, c->cfg.g, S * c->dtau, c->stream);
        IPG_LAUNCHED(c, 1);
        if (A.k == 1) {
            // every state stored: no time reversal, nothing overwritten
            for (int s = S - 1; s >= 0; s--) {
                const StepCoef<double> cf = evolution_coef(c, s);
                launch_adjoint_step(N, A.cp[s], A.cp[s + 1], A.adj, cf, c->stream);
                IPG_LAUNCHED(c, cf.do_pe ? 2 : 1);
            }
        } else {
            // reverse sweep: state s from state s+1 by time reversal, or from the
            // checkpoint when s is a multiple of k; two state sets alternate.
            // From its second step on the sweep overwrites the final state, so a
            // failure anywhere below must leave the forward marked as consumed.
            A.ready = false;
            State<double> sets[2] = {A.w[2], A.fin};
            State<double> nxt = A.fin;
            for (int s = S - 1, q = 0; s >= 0; s--, q++) {
                const State<double> cur = sets[q & 1];
                const StepCoef<double> cf = evolution_coef(c, s);
                if (s % A.k == 0) {
                    IPG_TRY(copy_state(c, cur, A.cp[s / A.k]));
                    launch_adjoint_step(N, cur, nxt, A.adj, cf, c->stream);
                    IPG_LAUNCHED(c, cf.do_pe ? 2 : 1);
                } else {
                    launch_inverse_adjoint_step(N, nxt, cur, A.adj, cf, c->stream);
                    IPG_LAUNCHED(c, cf.do_pe ? 3 : 2);
                }
                nxt = cur;
            }
        }
        launch_adjoint_project<double>(n, A.adj, c->stream);
        IPG_LAUNCHED(c, 1);
    }
    if (grad_g2mu || grad_rho) IPG_TRY(backward_inputs(c, grad_g2mu, grad_rho));
    IPG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    IPG_TRY(sync(c));
    A.ms_backward = elapsed(c);
    if (grad_g2mu)
        IPG_CUDA(c, cudaMemcpy(grad_g2mu, A.g2mu_bar, 2 * n * sizeof(double),
                               cudaMemcpyDeviceToHost));
    if (grad_rho)
        IPG_CUDA(c, cudaMemcpy(grad_rho, A.rho_all, 16 * (size_t)c->cfg.Ny * n * sizeof(double),
                               cudaMemcpyDeviceToHost));
    if (grad_state) {
        if (!A.sites) IPG_TRY(dalloc(c, &A.sites, 18 * n));
        const C<double> *bufs[6] = {A.adj.ux, A.adj.uy, A.adj.e1, A.adj.e2, A.adj.phi, A.adj.pi};
        for (int f = 0; f < 6; f++) {
            launch_planes_to_sites(n, bufs[f], A.sites, c->stream);
            IPG_LAUNCHED(c, 1);
            IPG_CUDA(c, cudaMemcpyAsync(grad_state + (size_t)f * 18 * n, A.sites,
                                        18 * n * sizeof(double), cudaMemcpyDeviceToHost,
                                        c->stream));
        }
    }
    IPG_TRY(sync(c));
    return IPG_OK;
}

}  // extern "C"

// ===========================================================================
// Batches: many events (contexts, possibly of different N) advanced together,
// one persistent launch per leapfrog step over all their sites, the step
// sequence captured once as a CUDA graph and replayed on every run. Per-step
// pointers and coefficients live in a device table that is refreshed before
// each replay, so the graph stays valid while the events' U/phi buffers swap
// roles from run to run.
// ===========================================================================

struct ipg_batch {
    std::vector<ipg_ctx *> ev;
    int device = 0;
    bool fp32 = false;
    int itmax = 0;
    double dtau = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::string err;
    int variant = 1, blocks_per_sm = 0, grid = 0;
    int tiles_variant = -1, total_tiles = 0;
    int *d_tile_begin = nullptr;
    void *d_table = nullptr, *h_table = nullptr;
    size_t event_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_variant = -1, graph_grid = -1;
    double last_ms_evolution = 0, last_ms_total = 0;
    long long launches = 0;
    bool tuned = false;
    // TMA variant: tensor maps of every event for both U/phi buffer
    // arrangements ([2 e + sel]); sel 0 holds the buffers that were the
    // event's current ones when the batch was made (phys0)
    LoadMaps *d_maps = nullptr;
    std::vector<const void *> phys0;
    double *d_status = nullptr;  // a TMA wait gave up
};

namespace {

ipg_status bfail(ipg_batch *b, ipg_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return st;
}

#define IPG_BCUDA(b, expr)                                                        \
    do {                                                                          \
        cudaError_t _e = (expr);                                                  \
        if (_e != cudaSuccess)                                                    \
            return bfail((b), IPG_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

template <typename T>
struct Bufs {
    State<T> *s;
    C<T> **uxb, **uyb;
    T **phib;
};
template <typename T>
Bufs<T> bufs(ipg_ctx *c);
template <>
Bufs<float> bufs<float>(ipg_ctx *c) {
    return {&c->s32, &c->ux32b, &c->uy32b, &c->phi32b};
}
template <>
Bufs<double> bufs<double>(ipg_ctx *c) {
    return {&c->s64, &c->ux64b, &c->uy64b, &c->phi64b};
}

int tile_rows(const ipg_batch *b, int variant) {
    return b->fp32 ? batch_tile_rows<float>(variant) : batch_tile_rows<double>(variant);
}

int max_blocks(const ipg_batch *b, int variant) {
    const int E = (int)b->ev.size();
    return b->fp32 ? batch_max_blocks_per_sm<float>(variant, E)
                   : batch_max_blocks_per_sm<double>(variant, E);
}

// variants the precision supports (FP64 needs <= 256 threads per block)
int n_variants(const ipg_batch *b) {
    return b->fp32 ? batch_variants<float>() : batch_variants<double>();
}
int tma_variant(const ipg_batch *b) {
    return b->fp32 ? batch_plain_variants<float>() : batch_plain_variants<double>();
}

ipg_status upload_tiles(ipg_batch *b, int variant) {
    if (b->tiles_variant == variant) return IPG_OK;
    const int E = (int)b->ev.size();
    std::vector<int> begin(E + 1, 0);
    const int rows = tile_rows(b, variant);
    for (int e = 0; e < E; e++) {
        const int N = b->ev[e]->N;
        begin[e + 1] = begin[e] + (N / 32) * (N / rows);
    }
    IPG_BCUDA(b, cudaMemcpyAsync(b->d_tile_begin, begin.data(), sizeof(int) * (E + 1),
                                 cudaMemcpyHostToDevice, b->stream));
    IPG_BCUDA(b, cudaStreamSynchronize(b->stream));
    b->total_tiles = begin[E];
    b->tiles_variant = variant;
    return IPG_OK;
}

// descriptors of steps [0, steps) for every event, following the schedule of
// run_evolution: step 0 is the tau = 0 half step of phi and U, step k > 0 the
// full step it = k. U/phi buffers alternate after every step. With
// full_first, step 0 is laid out on the current buffers but carries the
// coefficients of the full step it = 1 (the step the tuner times: it reads
// the current U/phi and writes only the other buffers, E and pi).
template <typename T>
void fill_table(ipg_batch *b, BatchEvent<T> *tab, int steps, bool full_first = false) {
    const int E = (int)b->ev.size();
    for (int e = 0; e < E; e++) {
        ipg_ctx *c = b->ev[e];
        Bufs<T> B = bufs<T>(c);
        State<T> s = *B.s;
        C<T> *uxb = *B.uxb, *uyb = *B.uyb;
        T *phib = *B.phib;
        for (int k = 0; k < steps; k++) {
            BatchEvent<T> &d = tab[(size_t)k * E + e];
            d.s = s;
            d.ux_out = uxb;
            d.uy_out = uyb;
            d.phi_out = phib;
            const int it = (full_first && k == 0) ? 1 : k;
            d.cf.tau = (T)(it * c->dtau);
            d.cf.dt_pe = (T)c->dtau;
            d.cf.dt_pu = (T)c->dtau;
            d.cf.g = (T)c->cfg.g;
            d.cf.do_pe = it > 0;
            d.cf.do_pu = 1;
            set_derived(d.cf);
            d.N = c->N;
            d.active = 1;
            d.map_sel = s.ux == b->phys0[e] ? 0 : 1;
            std::swap(s.ux, uxb);
            std::swap(s.uy, uyb);
            std::swap(s.phi, phib);
        }
    }
}

// the events' buffers after `swaps` U/phi exchanges
template <typename T>
void apply_swaps(ipg_batch *b, int swaps) {
    if ((swaps & 1) == 0) return;
    for (ipg_ctx *c : b->ev) {
        Bufs<T> B = bufs<T>(c);
        std::swap(B.s->ux, *B.uxb);
        std::swap(B.s->uy, *B.uyb);
        std::swap(B.s->phi, *B.phib);
    }
}

ipg_status launch_batch(ipg_batch *b, int step) {
    const int E = (int)b->ev.size();
    if (b->fp32) {
        auto *t = static_cast<BatchEvent<float> *>(b->d_table) + (size_t)step * E;
        launch_leapfrog_batch<float>(t, E, b->d_tile_begin, b->total_tiles, b->variant, b->grid,
                                     b->d_maps, b->d_status, b->stream);
    } else {
        auto *t = static_cast<BatchEvent<double> *>(b->d_table) + (size_t)step * E;
        launch_leapfrog_batch<double>(t, E, b->d_tile_begin, b->total_tiles, b->variant, b->grid,
                                      b->d_maps, b->d_status, b->stream);
    }
    b->launches++;
    return IPG_OK;
}

ipg_status capture_graph(ipg_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    IPG_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < b->itmax; k++) launch_batch(b, k);
    b->launches -= b->itmax;  // counted when the graph is launched
    cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
    if (e != cudaSuccess) return bfail(b, IPG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    IPG_BCUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_variant = b->variant;
    b->graph_grid = b->grid;
    return IPG_OK;
}

// tuning cache: key -> (variant, blocks per SM); optionally persisted in the
// file named by IPG_TUNE_CACHE (one "key variant blocks" line per entry)
std::map<std::string, std::pair<int, int>> &tune_cache() {
    static std::map<std::string, std::pair<int, int>> m;
    static bool loaded = false;
    if (!loaded) {
        loaded = true;
        if (const char *path = std::getenv("IPG_TUNE_CACHE")) {
            if (FILE *f = std::fopen(path, "r")) {
                char key[512];
                int v, bps;
                while (std::fscanf(f, "%511s %d %d", key, &v, &bps) == 3) m[key] = {v, bps};
                std::fclose(f);
            }
        }
    }
    return m;
}

std::string tune_key(const ipg_batch *b) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, b->device);
    std::map<int, int> sizes;
    for (const ipg_ctx *c : b->ev) sizes[c->N]++;
    std::string k = std::string(prop.name) + "|sm" + std::to_string(b->sms) +
                    (b->fp32 ? "|fp32" : "|fp64");
    for (auto &p : sizes) k += "|" + std::to_string(p.first) + "x" + std::to_string(p.second);
    for (char &ch : k)
        if (ch == ' ') ch = '_';
    return k;
}

}  // namespace

extern "C" {

const char *ipg_batch_last_error(const ipg_batch *b) {
    return b ? b->err.c_str() : "null batch";
}

ipg_status ipg_batch_create(ipg_ctx *const *events, int count, ipg_batch **out) {
    if (!out) return IPG_ERR_BAD_CONFIG;
    *out = nullptr;
    if (!events || count < 1) return IPG_ERR_BAD_CONFIG;
    ipg_batch *b = new (std::nothrow) ipg_batch();
    if (!b) return IPG_ERR_NOMEM;
    *out = b;
    for (int e = 0; e < count; e++) {
        if (!events[e]) return bfail(b, IPG_ERR_BAD_CONFIG, "event %d is null", e);
        b->ev.push_back(events[e]);
    }
    const ipg_ctx *c0 = events[0];
    b->device = c0->cfg.device;
    b->fp32 = is_fp32(c0);
    b->itmax = c0->itmax;
    b->dtau = c0->dtau;
    for (int e = 0; e < count; e++) {
        const ipg_ctx *c = events[e];
        if (c->cfg.device != b->device)
            return bfail(b, IPG_ERR_BAD_CONFIG, "event %d is on another device", e);
        if (is_fp32(c) != b->fp32)
            return bfail(b, IPG_ERR_BAD_CONFIG, "event %d has another precision", e);
        if (c->itmax != b->itmax || c->dtau != b->dtau)
            return bfail(b, IPG_ERR_BAD_CONFIG,
                         "event %d has another time grid (itmax %d vs %d)", e, c->itmax,
                         b->itmax);
        if (c->N < 32)
            return bfail(b, IPG_ERR_BAD_CONFIG, "event %d: batched lattices need N >= 32", e);
    }
    IPG_BCUDA(b, cudaSetDevice(b->device));
    IPG_BCUDA(b, cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
    IPG_BCUDA(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    IPG_BCUDA(b, cudaEventCreate(&b->e0));
    IPG_BCUDA(b, cudaEventCreate(&b->e1));
    b->event_bytes = b->fp32 ? sizeof(BatchEvent<float>) : sizeof(BatchEvent<double>);
    const size_t table = b->event_bytes * count * (size_t)b->itmax;
    IPG_BCUDA(b, cudaMalloc(&b->d_table, table));
    IPG_BCUDA(b, cudaMallocHost(&b->h_table, table));
    IPG_BCUDA(b, cudaMalloc(&b->d_tile_begin, sizeof(int) * (count + 1)));
    // tensor maps of both buffer arrangements of every event
    {
        std::vector<LoadMaps> maps(2 * (size_t)count);
        bool ok = true;
        for (int e = 0; e < count && ok; e++) {
            ipg_ctx *c = b->ev[e];
            if (b->fp32) {
                State<float> s0 = c->s32, s1 = c->s32;
                s1.ux = c->ux32b;
                s1.uy = c->uy32b;
                s1.phi = c->phi32b;
                ok = encode_step_maps<float>(c->N, s0, &maps[2 * e]) &&
                     encode_step_maps<float>(c->N, s1, &maps[2 * e + 1]);
                b->phys0.push_back(c->s32.ux);
            } else {
                State<double> s0 = c->s64, s1 = c->s64;
                s1.ux = c->ux64b;
                s1.uy = c->uy64b;
                s1.phi = c->phi64b;
                ok = encode_step_maps<double>(c->N, s0, &maps[2 * e]) &&
                     encode_step_maps<double>(c->N, s1, &maps[2 * e + 1]);
                b->phys0.push_back(c->s64.ux);
            }
        }
        IPG_BCUDA(b, cudaMalloc(&b->d_status, sizeof(double)));
        IPG_BCUDA(b, cudaMemsetAsync(b->d_status, 0, sizeof(double), b->stream));
        if (ok) {
            IPG_BCUDA(b, cudaMalloc(&b->d_maps, sizeof(LoadMaps) * maps.size()));
            IPG_BCUDA(b, cudaMemcpyAsync(b->d_maps, maps.data(), sizeof(LoadMaps) * maps.size(),
                                         cudaMemcpyHostToDevice, b->stream));
        }
        IPG_BCUDA(b, cudaStreamSynchronize(b->stream));
    }
    const auto it = tune_cache().find(tune_key(b));
    if (it != tune_cache().end()) {
        b->variant = it->second.first;
        b->blocks_per_sm = it->second.second;
        b->tuned = true;
    } else {
        // the TMA tile kernel when the maps and the descriptors fit, else the
        // plain-load kernel with 4-row tiles
        b->variant = tma_variant(b);
        b->blocks_per_sm = b->d_maps ? max_blocks(b, b->variant) : 0;
        if (b->blocks_per_sm < 1) {
            b->variant = 1;
            b->blocks_per_sm = max_blocks(b, b->variant);
        }
    }
    if (b->blocks_per_sm < 1) return bfail(b, IPG_ERR_CUDA, "batched kernel cannot be resident");
    b->grid = b->blocks_per_sm * b->sms;
    return IPG_OK;
}

ipg_status ipg_batch_destroy(ipg_batch *b) {
    if (!b) return IPG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_table) cudaFree(b->d_table);
    if (b->h_table) cudaFreeHost(b->h_table);
    if (b->d_tile_begin) cudaFree(b->d_tile_begin);
    if (b->d_maps) cudaFree(b->d_maps);
    if (b->d_status) cudaFree(b->d_status);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return IPG_OK;
}

ipg_status ipg_batch_init(ipg_batch *b, ipg_init_report *reports) {
    if (!b) return IPG_ERR_BAD_CONFIG;
    const int E = (int)b->ev.size();
    // every event's initial conditions on its own stream, then one wait each:
    // small lattices overlap on the GPU
    for (int e = 0; e < E; e++) {
        ipg_status st = init_enqueue(b->ev[e], false);
        if (st != IPG_OK) return bfail(b, st, "event %d: %s", e, b->ev[e]->err.c_str());
    }
    ipg_status worst = IPG_OK;
    for (int e = 0; e < E; e++) {
        ipg_status st = init_finish(b->ev[e], reports ? reports + e : nullptr);
        if (st == IPG_ERR_NEWTON_NONCONVERGED) {
            worst = st;
            b->err = "event " + std::to_string(e) + ": " + b->ev[e]->err;
        } else if (st != IPG_OK) {
            return bfail(b, st, "event %d: %s", e, b->ev[e]->err.c_str());
        }
    }
    return worst;
}

ipg_status ipg_batch_tune(ipg_batch *b, ipg_tune_report *rep) {
    if (!b) return IPG_ERR_BAD_CONFIG;
    IPG_BCUDA(b, cudaSetDevice(b->device));
    const std::string key = tune_key(b);
    auto fill_report = [&](double ms, int candidates, int from_cache) {
        if (!rep) return;
        rep->variant = b->variant;
        rep->tile_rows = tile_rows(b, b->variant);
        rep->threads_per_block = 32 * rep->tile_rows;
        rep->blocks_per_sm = b->blocks_per_sm;
        rep->grid = b->grid;
        rep->ms_per_step = ms;
        rep->candidates = candidates;
        rep->from_cache = from_cache;
    };
    auto hit = tune_cache().find(key);
    if (hit != tune_cache().end()) {
        b->variant = hit->second.first;
        b->blocks_per_sm = hit->second.second;
        b->grid = b->blocks_per_sm * b->sms;
        b->tuned = true;
        fill_report(0., 0, 1);
        return IPG_OK;
    }
    for (ipg_ctx *c : b->ev)
        if (!c->initialized || c->half_done || c->finished)
            return bfail(b, IPG_ERR_STATE, "tune needs every event freshly initialised");
    // E and pi are updated in place by a step: keep a copy and put it back
    std::vector<void *> saved;
    const size_t w = b->fp32 ? sizeof(float) : sizeof(double);
    for (ipg_ctx *c : b->ev) {
        void *p = nullptr;
        if (cudaMalloc(&p, 25 * c->n * w) != cudaSuccess) {
            cudaGetLastError();
            for (void *q : saved) cudaFree(q);
            return bfail(b, IPG_ERR_NOMEM, "tuning scratch allocation failed");
        }
        saved.push_back(p);
        char *dst = static_cast<char *>(p);
        const void *e1 = b->fp32 ? (const void *)c->s32.e1 : (const void *)c->s64.e1;
        const void *e2 = b->fp32 ? (const void *)c->s32.e2 : (const void *)c->s64.e2;
        const void *pi = b->fp32 ? (const void *)c->s32.pi : (const void *)c->s64.pi;
        cudaMemcpyAsync(dst, e1, 8 * c->n * w, cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(dst + 8 * c->n * w, e2, 8 * c->n * w, cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(dst + 16 * c->n * w, pi, 9 * c->n * w, cudaMemcpyDeviceToDevice, b->stream);
    }
    // one representative full step (it = 1) for every event, in table slot 0
    const int E = (int)b->ev.size();
    if (b->fp32)
        fill_table<float>(b, static_cast<BatchEvent<float> *>(b->h_table), 1, true);
    else
        fill_table<double>(b, static_cast<BatchEvent<double> *>(b->h_table), 1, true);
    const int slot = 0;
    IPG_BCUDA(b, cudaMemcpyAsync(b->d_table, b->h_table, b->event_bytes * E,
                                 cudaMemcpyHostToDevice, b->stream));
    double best = 1e30;
    int best_v = b->variant, best_bps = b->blocks_per_sm, candidates = 0;
    for (int v = 0; v < n_variants(b); v++) {
        const int maxb = (v == tma_variant(b) && !b->d_maps) ? 0 : max_blocks(b, v);
        for (int bps = 1; bps <= maxb; bps++) {
            b->variant = v;
            b->blocks_per_sm = bps;
            b->grid = bps * b->sms;
            IPG_TRY(upload_tiles(b, v));
            launch_batch(b, slot);  // warm-up
            IPG_BCUDA(b, cudaEventRecord(b->e0, b->stream));
            const int reps = 3;
            for (int r = 0; r < reps; r++) launch_batch(b, slot);
            IPG_BCUDA(b, cudaEventRecord(b->e1, b->stream));
            IPG_BCUDA(b, cudaEventSynchronize(b->e1));
            IPG_BCUDA(b, cudaGetLastError());
            float ms = 0.f;
            cudaEventElapsedTime(&ms, b->e0, b->e1);
            candidates++;
            if (ms / reps < best) {
                best = ms / reps;
                best_v = v;
                best_bps = bps;
            }
        }
    }
    for (int e = 0; e < E; e++) {
        ipg_ctx *c = b->ev[e];
        const char *src = static_cast<const char *>(saved[e]);
        void *e1 = b->fp32 ? (void *)c->s32.e1 : (void *)c->s64.e1;
        void *e2 = b->fp32 ? (void *)c->s32.e2 : (void *)c->s64.e2;
        void *pi = b->fp32 ? (void *)c->s32.pi : (void *)c->s64.pi;
        cudaMemcpyAsync(e1, src, 8 * c->n * w, cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(e2, src + 8 * c->n * w, 8 * c->n * w, cudaMemcpyDeviceToDevice, b->stream);
        cudaMemcpyAsync(pi, src + 16 * c->n * w, 9 * c->n * w, cudaMemcpyDeviceToDevice,
                        b->stream);
    }
    IPG_BCUDA(b, cudaStreamSynchronize(b->stream));
    for (void *q : saved) cudaFree(q);
    b->variant = best_v;
    b->blocks_per_sm = best_bps;
    b->grid = best_bps * b->sms;
    b->tuned = true;
    tune_cache()[key] = {best_v, best_bps};
    if (const char *path = std::getenv("IPG_TUNE_CACHE")) {
        if (FILE *f = std::fopen(path, "a")) {
            std::fprintf(f, "%s %d %d\n", key.c_str(), best_v, best_bps);
            std::fclose(f);
        }
    }
    fill_report(best, candidates, 0);
    return IPG_OK;
}

ipg_status ipg_batch_run(ipg_batch *b, ipg_result *results) {
    if (!b) return IPG_ERR_BAD_CONFIG;
    IPG_BCUDA(b, cudaSetDevice(b->device));
    const int E = (int)b->ev.size();
    for (int e = 0; e < E; e++) {
        const ipg_ctx *c = b->ev[e];
        if (!c->initialized || c->half_done || c->finished)
            return bfail(b, IPG_ERR_STATE, "event %d needs fresh initial fields", e);
    }
    IPG_TRY(upload_tiles(b, b->variant));
    if (b->fp32)
        fill_table<float>(b, static_cast<BatchEvent<float> *>(b->h_table), b->itmax);
    else
        fill_table<double>(b, static_cast<BatchEvent<double> *>(b->h_table), b->itmax);
    IPG_BCUDA(b, cudaMemcpyAsync(b->d_table, b->h_table, b->event_bytes * E * b->itmax,
                                 cudaMemcpyHostToDevice, b->stream));
    if (!b->exec || b->graph_variant != b->variant || b->graph_grid != b->grid)
        IPG_TRY(capture_graph(b));
    IPG_BCUDA(b, cudaMemsetAsync(b->d_status, 0, sizeof(double), b->stream));
    IPG_BCUDA(b, cudaEventRecord(b->e0, b->stream));
    IPG_BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    b->launches += b->itmax;
    IPG_BCUDA(b, cudaEventRecord(b->e1, b->stream));
    IPG_BCUDA(b, cudaEventSynchronize(b->e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    b->last_ms_evolution = ms;
    double gave_up = 0.;
    IPG_BCUDA(b, cudaMemcpy(&gave_up, b->d_status, sizeof(double), cudaMemcpyDeviceToHost));
    if (gave_up != 0.)
        return bfail(b, IPG_ERR_TIMEOUT, "a batched leapfrog step gave up waiting for its tiles");
    if (b->fp32)
        apply_swaps<float>(b, b->itmax);
    else
        apply_swaps<double>(b, b->itmax);
    for (ipg_ctx *c : b->ev) {
        c->half_done = true;
        c->it = b->itmax - 1;
        c->last_leapfrog_ms = ms;
        c->last_leapfrog_launches = b->itmax;
    }
    // observables of all events, each on its own stream
    const auto t0 = std::chrono::steady_clock::now();
    ipg_status worst = IPG_OK;
    for (int e = 0; e < E; e++) {
        ipg_status st = observables_enqueue(b->ev[e]);
        if (st != IPG_OK) return bfail(b, st, "event %d: %s", e, b->ev[e]->err.c_str());
    }
    for (int e = 0; e < E; e++) {
        ipg_status st = observables_finish(b->ev[e], results ? results + e : nullptr);
        if (st == IPG_ERR_NAN) {
            worst = st;
            b->err = "event " + std::to_string(e) + ": " + b->ev[e]->err;
        } else if (st != IPG_OK) {
            return bfail(b, st, "event %d: %s", e, b->ev[e]->err.c_str());
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    b->last_ms_total = ms + std::chrono::duration<double, std::milli>(t1 - t0).count();
    return worst;
}

ipg_status ipg_batch_set_shape(ipg_batch *b, int variant, int blocks_per_sm) {
    if (!b) return IPG_ERR_BAD_CONFIG;
    if (variant < 0 || variant >= n_variants(b) || (variant == tma_variant(b) && !b->d_maps))
        return bfail(b, IPG_ERR_BAD_CONFIG, "variant %d not available", variant);
    const int maxb = max_blocks(b, variant);
    if (blocks_per_sm < 1 || blocks_per_sm > maxb)
        return bfail(b, IPG_ERR_BAD_CONFIG, "blocks_per_sm must be in [1, %d]", maxb);
    b->variant = variant;
    b->blocks_per_sm = blocks_per_sm;
    b->grid = blocks_per_sm * b->sms;
    return IPG_OK;
}

ipg_status ipg_batch_stats(const ipg_batch *b, double *ms_evolution, double *ms_total,
                           long long *launches) {
    if (!b) return IPG_ERR_BAD_CONFIG;
    if (ms_evolution) *ms_evolution = b->last_ms_evolution;
    if (ms_total) *ms_total = b->last_ms_total;
    if (launches) *launches = b->launches;
    return IPG_OK;
}

}  // extern "C"
