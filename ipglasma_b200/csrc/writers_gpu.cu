// The two output files of writers.cpp (hydro: epsilon-u-Hydro-..., MyEigen.cpp:
// 380-797; KoMPoST: Tmunu-t..., MyEigen.cpp:801-1045) with the resampling and
// the number formatting on the GPU, from the observables already in device
// memory. The text is byte-identical to the host writers: this file is
// compiled with -fmad=false, so every sum and product is rounded as the host
// code (built with -ffp-contract=off) rounds it, in the same order, and
// fmt::g6 gives the correctly rounded "%.6g" text.
//
// k_lines: one thread per output line formats it into a 256-byte slot in
// shared memory; the block scans its 128 line lengths, writes its compacted
// text to its own chunk and the chunk's length. k_scan_chunks turns the
// chunk lengths into offsets (and the total), k_gather copies each chunk to
// its offset in the file image, which the host copies back and writes with
// one fwrite. A line holding a number outside fmt::g6's range sets *bad and
// the caller writes that file with the host writer instead.
#include <cstdint>

#include "fmt.cuh"
#include "ipg_internal.h"

namespace ipg {

namespace {

constexpr double kHbarc = 0.1973269718;  // Phys_consts.h
constexpr double kSmallEps = 1e-16;
constexpr int kLineThreads = 128;
constexpr int kSlot = 256;  // bytes: 18 numbers of at most 13 characters, separators
constexpr int kSmemStride = kSlot + 4;  // slots of a warp's threads start in distinct banks

struct Stencil {
    int p1, p2, p3, p4;
    double fx, fy;
};

__device__ Stencil stencil(const OutputGrid &g, double x, double y) {
    Stencil s;
    const int xpos = static_cast<int>(floor((x + g.L / 2.) / g.a + 0.0000000001));
    const int ypos = static_cast<int>(floor((y + g.L / 2.) / g.a + 0.0000000001));
    const int xup = (xpos < g.N - 1) ? xpos + 1 : xpos;
    const int yup = (ypos < g.N - 1) ? ypos + 1 : ypos;
    const double xlow = -g.L / 2. + g.a * xpos;
    const double ylow = -g.L / 2. + g.a * ypos;
    s.fx = (x - xlow) / g.ha;
    s.fy = (y - ylow) / g.ha;
    s.p1 = xpos * g.N + ypos;
    s.p2 = xup * g.N + ypos;
    s.p3 = xpos * g.N + yup;
    s.p4 = xup * g.N + yup;
    return s;
}

__device__ double interp(const Stencil &s, int nn, const double *f, bool absval) {
    auto val = [&](int p) { return absval ? fabs(f[p]) : f[p]; };
    double x1 = 0., x2 = 0.;
    if (s.p1 > 0 && s.p1 < nn && s.p2 > 0 && s.p2 < nn)
        x1 = (1 - s.fx) * val(s.p1) + s.fx * val(s.p2);
    if (s.p3 > 0 && s.p3 < nn && s.p4 > 0 && s.p4 < nn)
        x2 = (1 - s.fx) * val(s.p3) + s.fx * val(s.p4);
    return (1. - s.fy) * x1 + s.fy * x2;
}

struct Line {
    char *p;
    int n;
    bool ok;
    __device__ Line &num(double v) {
        const int k = fmt::g6(v, p + n);
        if (k < 0) {
            ok = false;
        } else {
            n += k;
        }
        return *this;
    }
    __device__ Line &num(int v) {
        n += fmt::integer(v, p + n);
        return *this;
    }
    __device__ Line &ch(char c) {
        p[n++] = c;
        return *this;
    }
};

// hydro line (ieta, ix, iy), as writers.cpp ipg_write_hydro's body
__device__ void hydro_line(const OutputGrid &g, const OutputFields &f, long long line, Line &out,
                           double &term) {
    const int nn = g.N * g.N;
    const size_t n = (size_t)nn;
    const long long r = line / g.hx;
    const int iy = (int)(line - r * g.hx);
    const int ieta = (int)(r / g.hx), ix = (int)(r - (long long)ieta * g.hx);
    const double eta = -(g.heta - 1) / 2. * g.deta + g.deta * ieta;
    const double x = -g.hL / 2. + g.ha * ix;
    const double y = -g.hL / 2. + g.ha * iy;
    term = 0.;
    out.num(eta).ch(' ').num(x).ch(' ').num(y).ch(' ');
    bool placeholder = true;
    if (fabs(x) < g.L / 2. && fabs(y) < g.L / 2.) {
        const Stencil s = stencil(g, x, y);
        const double *p00 = f.pi10, *pxx = f.pi10 + n, *pyy = f.pi10 + 2 * n,
                     *pee = f.pi10 + 3 * n;
        const double *p0x = f.pi10 + 4 * n, *p0y = f.pi10 + 5 * n, *p0e = f.pi10 + 6 * n;
        const double *pxy = f.pi10 + 7 * n, *pxe = f.pi10 + 8 * n, *pye = f.pi10 + 9 * n;
        const double e = interp(s, nn, f.eps, true);
        const double ux = interp(s, nn, f.u4 + n, false);
        const double uy = interp(s, nn, f.u4 + 2 * n, false);
        const double ueta = interp(s, nn, f.u4 + 3 * n, false);
        const double tau0 = g.tau0;
        const double utau = sqrt(1. + ux * ux + uy * uy + tau0 * tau0 * ueta * ueta);
        term = fabs(kHbarc * e * g.gfactor) * g.ha * g.ha * g.it * g.dtau * g.a;
        if (fabs(kHbarc * e * g.gfactor) > 0.0000000001) {
            const double gf = g.gfactor;
            out.num(fabs(kHbarc * e * gf)).ch(' ').num(utau).ch(' ');
            out.num(ux).ch(' ').num(uy).ch(' ').num(ueta).ch(' ');
            out.num(interp(s, nn, p00, false) * gf).ch(' ');
            out.num(interp(s, nn, p0x, false) * gf).ch(' ');
            out.num(interp(s, nn, p0y, false) * gf).ch(' ');
            out.num(interp(s, nn, p0e, false) * gf).ch(' ');
            out.num(interp(s, nn, pxx, false) * gf).ch(' ');
            out.num(interp(s, nn, pxy, false) * gf).ch(' ');
            out.num(interp(s, nn, pxe, false) * gf).ch(' ');
            out.num(interp(s, nn, pyy, false) * gf).ch(' ');
            out.num(interp(s, nn, pye, false) * gf).ch(' ');
            out.num(interp(s, nn, pee, false) * gf).ch('\n');
            placeholder = false;
        }
    }
    if (placeholder) {
        out.num(0.).ch(' ').num(1.);
        for (int k = 0; k < 13; k++) out.ch(' ').num(0.);
        out.ch('\n');
    }
    // a blank line after each eta slice
    if (ix == g.hx - 1 && iy == g.hx - 1) out.ch('\n');
}

// KoMPoST line (iy, ix), as writers.cpp ipg_write_tmunu's body
__device__ void tmunu_line(const OutputGrid &g, const OutputFields &f, long long line, Line &out) {
    const int nn = g.N * g.N;
    const size_t n = (size_t)nn;
    const int iy = (int)(line / g.hx), ix = (int)(line - (long long)iy * g.hx);
    const double x = -g.hL / 2. + g.ha * ix;
    const double y = -g.hL / 2. + g.ha * iy;
    out.num(ix).ch(' ').num(iy).ch(' ');
    bool placeholder = true;
    if (fabs(x) < g.L / 2. && fabs(y) < g.L / 2.) {
        const Stencil s = stencil(g, x, y);
        const double *T = f.T10;
        const double t00 = interp(s, nn, T, false);
        if (t00 * g.gfactor * kHbarc > kSmallEps) {
            const double gf = g.gfactor, tau0 = g.tau0;
            const double t0x = interp(s, nn, T + 4 * n, false);
            const double t0y = interp(s, nn, T + 5 * n, false);
            const double t0e = interp(s, nn, T + 6 * n, false);
            const double txx = interp(s, nn, T + n, false);
            const double txy = interp(s, nn, T + 7 * n, false);
            const double txe = interp(s, nn, T + 8 * n, false);
            const double tyy = interp(s, nn, T + 2 * n, false);
            const double tye = interp(s, nn, T + 9 * n, false);
            const double tee = interp(s, nn, T + 3 * n, false);
            out.num(t00 * gf * kHbarc).ch(' ');
            out.num(txx * gf * kHbarc).ch(' ').num(tyy * gf * kHbarc).ch(' ');
            out.num(tau0 * tau0 * tee * gf * kHbarc).ch(' ');
            out.num(-t0x * gf * kHbarc).ch(' ').num(-t0y * gf * kHbarc).ch(' ');
            out.num(-tau0 * t0e * gf * kHbarc).ch(' ');
            out.num(-txy * gf * kHbarc).ch(' ');
            out.num(-tau0 * tye * gf * kHbarc).ch(' ');
            out.num(-tau0 * txe * gf * kHbarc).ch('\n');
            placeholder = false;
        }
    }
    if (placeholder) {
        out.num(kSmallEps).ch(' ').num(kSmallEps / 2.).ch(' ').num(kSmallEps / 2.);
        for (int k = 0; k < 7; k++) out.ch(' ').num(0.0);
        out.ch('\n');
    }
    // a blank line after each y row
    if (ix == g.hx - 1) out.ch('\n');
}

template <int KIND>  // 0 hydro, 1 KoMPoST
__global__ void __launch_bounds__(kLineThreads)
    k_lines(OutputGrid g, OutputFields f, long long lines, char *chunks, int *chunk_len,
            double *term, int *bad) {
    __shared__ char slot[kLineThreads * kSmemStride];
    __shared__ int offs[kLineThreads + 1];
    __shared__ int warp_sum[kLineThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long line = (long long)blockIdx.x * kLineThreads + tid;
    Line out{slot + tid * kSmemStride, 0, true};
    if (line < lines) {
        if (KIND == 0) {
            double t;
            hydro_line(g, f, line, out, t);
            term[line] = t;
        } else {
            tmunu_line(g, f, line, out);
        }
        if (!out.ok) atomicOr(bad, 1);
    }
    // block-wide exclusive scan of the line lengths
    int v = out.n;
    for (int d = 1; d < 32; d <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += u;
    }
    if (lane == 31) warp_sum[warp] = v;
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; w++) base += warp_sum[w];
    offs[tid + 1] = base + v;
    if (tid == 0) offs[0] = 0;
    __syncthreads();
    const int total = offs[kLineThreads];
    char *dst = chunks + (size_t)blockIdx.x * kLineThreads * kSlot;
    // each warp copies its 32 lines, lanes on consecutive bytes
    for (int l = warp * 32; l < warp * 32 + 32; l++) {
        const int o = offs[l], len = offs[l + 1] - o;
        const char *src = slot + l * kSmemStride;
        for (int b = lane; b < len; b += 32) dst[o + b] = src[b];
    }
    if (tid == 0) chunk_len[blockIdx.x] = total;
}

// chunk_off[c] = sum of chunk_len[0, c), chunk_off[count] = the total; one block
__global__ void k_scan_chunks(const int *chunk_len, long long *chunk_off, int count) {
    __shared__ long long part[1024];
    const int tid = threadIdx.x;
    const int per = (count + 1023) / 1024;
    const int b0 = tid * per, b1 = min(count, b0 + per);
    long long s = 0;
    for (int c = b0; c < b1; c++) s += chunk_len[c];
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        long long acc = 0;
        for (int t = 0; t < 1024; t++) {
            const long long x = part[t];
            part[t] = acc;
            acc += x;
        }
        chunk_off[count] = acc;
    }
    __syncthreads();
    long long acc = part[tid];
    for (int c = b0; c < b1; c++) {
        chunk_off[c] = acc;
        acc += chunk_len[c];
    }
}

__global__ void k_gather(const char *chunks, const int *chunk_len, const long long *chunk_off,
                         char *text) {
    const char *src = chunks + (size_t)blockIdx.x * kLineThreads * kSlot;
    char *dst = text + chunk_off[blockIdx.x];
    const int len = chunk_len[blockIdx.x];
    for (int b = threadIdx.x; b < len; b += blockDim.x) dst[b] = src[b];
}

}  // namespace

size_t output_text_capacity(long long lines) {
    const long long blocks = (lines + kLineThreads - 1) / kLineThreads;
    return (size_t)blocks * kLineThreads * kSlot;
}

int output_text_chunks(long long lines) {
    return (int)((lines + kLineThreads - 1) / kLineThreads);
}

void launch_output_text(int kind, const OutputGrid &g, const OutputFields &f, long long lines,
                        char *chunks, int *chunk_len, long long *chunk_off, char *text,
                        double *term, int *bad, cudaStream_t st) {
    const int blocks = output_text_chunks(lines);
    if (blocks == 0) return;
    if (kind == 0)
        k_lines<0><<<blocks, kLineThreads, 0, st>>>(g, f, lines, chunks, chunk_len, term, bad);
    else
        k_lines<1><<<blocks, kLineThreads, 0, st>>>(g, f, lines, chunks, chunk_len, term, bad);
    k_scan_chunks<<<1, 1024, 0, st>>>(chunk_len, chunk_off, blocks);
    k_gather<<<blocks, 256, 0, st>>>(chunks, chunk_len, chunk_off, text);
}

}  // namespace ipg
