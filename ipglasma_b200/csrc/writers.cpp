// Output files for hydrodynamics and kinetic theory, in the reference's text
// formats (MyEigen::flowVelocity4D output part, MyEigen.cpp:329-1045):
//   epsilon-u-Hydro-TauHydro-<id>.dat   writeOutputs odd   (MyEigen.cpp:380-797)
//   Tmunu-t<tau>-<id>.dat               writeOutputs/4 == 1 (MyEigen.cpp:801-1045)
// Both resample the N x N lattice bilinearly onto sizeOutput^2 points over
// LOutput, keeping the reference's conventions: the fractional offset is
// divided by the OUTPUT spacing, a neighbour pair counts only if both sites
// have an index strictly greater than 0, e <= 1e-10 GeV/fm^3 (hydro) and
// T^tautau <= 1e-16 (Tmunu) become placeholder rows, u^tau is recomputed from
// the normalisation, and numbers are printed as an ostream with default flags
// prints them (printf "%g": 6 significant digits). Host code, fed from
// ipg_get_observables.
//
// The reference streams line by line with a flush per line; here the output
// rows are formatted in parallel (std::to_chars with precision 6 is specified
// as printf "%.6g" in the C locale, so the bytes are the same) into one buffer
// per thread, and the buffers are written in row order with one fwrite each.
// The hydro file's total energy is summed serially in the reference's loop
// order from per-point terms, so it is bit-identical too.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ipglasma_b200.h"
#include "writers.h"

namespace {

constexpr double kHbarc = 0.1973269718;  // Phys_consts.h
constexpr double kSmallEps = 1e-16;

struct Grid {
    int N;
    double L, a;
    int hx, heta;
    double hL, ha, deta;
};

// indices and fractions of the bilinear resampling at output point (x, y)
struct Stencil {
    int p1, p2, p3, p4;
    double fx, fy;
};

Stencil stencil(const Grid &g, double x, double y) {
    Stencil s;
    const int xpos = static_cast<int>(std::floor((x + g.L / 2.) / g.a + 0.0000000001));
    const int ypos = static_cast<int>(std::floor((y + g.L / 2.) / g.a + 0.0000000001));
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

// (1 - fy) x1 + fy x2 with the reference's validity test on each pair
double interp(const Stencil &s, int nn, const double *f, bool absval) {
    auto val = [&](int p) { return absval ? std::abs(f[p]) : f[p]; };
    double x1 = 0., x2 = 0.;
    if (s.p1 > 0 && s.p1 < nn && s.p2 > 0 && s.p2 < nn)
        x1 = (1 - s.fx) * val(s.p1) + s.fx * val(s.p2);
    if (s.p3 > 0 && s.p3 < nn && s.p4 > 0 && s.p4 < nn)
        x2 = (1 - s.fx) * val(s.p3) + s.fx * val(s.p4);
    return (1. - s.fy) * x1 + s.fy * x2;
}

// Text buffer with the two number formats of an ostream with default flags.
// A number takes at most 13 characters ("-1.23457e-308"), an int at most 11.
class Text {
  public:
    explicit Text(size_t reserve) { s_.reserve(reserve); }
    // room for one line of `count` numbers and separators
    void line(int count) {
        const size_t need = n_ + (size_t)count * 16 + 2;
        if (need > s_.size()) s_.resize(std::max(need, 2 * s_.size()));
    }
    Text &num(double v) {
        n_ = std::to_chars(&s_[n_], &s_[0] + s_.size(), v, std::chars_format::general, 6).ptr -
             &s_[0];
        return *this;
    }
    Text &num(int v) {
        n_ = std::to_chars(&s_[n_], &s_[0] + s_.size(), v).ptr - &s_[0];
        return *this;
    }
    Text &ch(char c) {
        s_[n_++] = c;
        return *this;
    }
    const char *data() const { return s_.data(); }
    size_t size() const { return n_; }

  private:
    std::string s_;
    size_t n_ = 0;
};

// "# dummy 1 etamax= .. xmax= .. ymax= .. deta= .. dx= .. dy= .." and, for the
// hydro file, " tau= ..", then a newline
Text header(const Grid &g, bool with_tau, double tau0) {
    Text head(256);
    head.line(16);
    auto label = [&](const char *s) {
        for (; *s; s++) head.ch(*s);
    };
    label("# dummy "), head.num(1);
    label(" etamax= "), head.num(g.heta), label(" xmax= "), head.num(g.hx);
    label(" ymax= "), head.num(g.hx), label(" deta= "), head.num(g.deta);
    label(" dx= "), head.num(g.ha), label(" dy= "), head.num(g.ha);
    if (with_tau) label(" tau= "), head.num(tau0);
    head.ch('\n');
    return head;
}
Text hydro_head(const Grid &g, double tau0) { return header(g, true, tau0); }
Text tmunu_head(const Grid &g) { return header(g, false, 0.); }

// threads used to format a file of `rows` output rows: the host's hardware
// threads (IPG_WRITER_THREADS overrides), at most one per 4 rows
int writer_threads(int rows) {
    int t = (int)std::thread::hardware_concurrency();
    if (const char *e = std::getenv("IPG_WRITER_THREADS")) t = std::atoi(e);
    t = std::min({std::max(t, 1), 64, std::max(rows / 4, 1)});
    return t;
}

// format rows [0, rows) with body(text, r) split over threads in contiguous
// chunks, then write the chunks in order after `head`
template <class Body>
bool format_and_write(const char *path, const Text &head, int rows, size_t bytes_per_row,
                      Body body) {
    const int T = writer_threads(rows);
    std::vector<Text> parts;
    parts.reserve(T);
    for (int t = 0; t < T; t++) parts.emplace_back(bytes_per_row * (rows / T + 1));
    auto run = [&](int t) {
        const int r0 = (int)((long long)rows * t / T), r1 = (int)((long long)rows * (t + 1) / T);
        for (int r = r0; r < r1; r++) body(parts[t], r);
    };
    if (T == 1) {
        run(0);
    } else {
        std::vector<std::thread> pool;
        for (int t = 1; t < T; t++) pool.emplace_back(run, t);
        run(0);
        for (auto &th : pool) th.join();
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    for (const Text &p : parts) ok = ok && std::fwrite(p.data(), 1, p.size(), f) == p.size();
    return (std::fclose(f) == 0) && ok;
}

}  // namespace

namespace ipg {

std::string hydro_header(int N, double L, int sizeOutput, double LOutput, int etaSizeOutput,
                         double detaOutput, int it, double dtau) {
    const Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput,
                 detaOutput};
    const Text h = hydro_head(g, it * dtau * g.a);
    return std::string(h.data(), h.size());
}

std::string tmunu_header(int N, double L, int sizeOutput, double LOutput, int etaSizeOutput,
                         double detaOutput) {
    const Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput,
                 detaOutput};
    const Text h = tmunu_head(g);
    return std::string(h.data(), h.size());
}

}  // namespace ipg

extern "C" {

ipg_status ipg_write_hydro(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *eps,
                           const double *u4, const double *pi10, double gfactor,
                           double *Etot) {
    if (!path || !eps || !u4 || !pi10 || N < 1 || sizeOutput < 1 || etaSizeOutput < 0)
        return IPG_ERR_BAD_CONFIG;
    Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput, detaOutput};
    const int nn = N * N;
    const double a = g.a;
    const double tau0 = it * dtau * a;
    const Text head = hydro_head(g, tau0);
    const size_t n = (size_t)nn;
    // pi10 order: tautau xx yy etaeta taux tauy taueta xy xeta yeta
    const double *p00 = pi10, *pxx = pi10 + n, *pyy = pi10 + 2 * n, *pee = pi10 + 3 * n;
    const double *p0x = pi10 + 4 * n, *p0y = pi10 + 5 * n, *p0e = pi10 + 6 * n;
    const double *pxy = pi10 + 7 * n, *pxe = pi10 + 8 * n, *pye = pi10 + 9 * n;
    // one output row = (ieta, ix): hx lines, and a blank line after each eta slice
    const int rows = g.heta * g.hx;
    std::vector<double> term((size_t)rows * g.hx, 0.);
    auto body = [&](Text &out, int r) {
        const int ieta = r / g.hx, ix = r - ieta * g.hx;
        const double eta = -(g.heta - 1) / 2. * g.deta + g.deta * ieta;
        for (int iy = 0; iy < g.hx; iy++) {
            const double x = -g.hL / 2. + g.ha * ix;
            const double y = -g.hL / 2. + g.ha * iy;
            out.line(18);
            out.num(eta).ch(' ').num(x).ch(' ').num(y).ch(' ');
            if (std::abs(x) < L / 2. && std::abs(y) < L / 2.) {
                const Stencil s = stencil(g, x, y);
                const double e = interp(s, nn, eps, true);
                const double ux = interp(s, nn, u4 + n, false);
                const double uy = interp(s, nn, u4 + 2 * n, false);
                const double ueta = interp(s, nn, u4 + 3 * n, false);
                const double q00 = interp(s, nn, p00, false);
                const double q0x = interp(s, nn, p0x, false);
                const double q0y = interp(s, nn, p0y, false);
                const double q0e = interp(s, nn, p0e, false);
                const double qxy = interp(s, nn, pxy, false);
                const double qxe = interp(s, nn, pxe, false);
                const double qye = interp(s, nn, pye, false);
                const double qxx = interp(s, nn, pxx, false);
                const double qyy = interp(s, nn, pyy, false);
                const double qee = interp(s, nn, pee, false);
                const double utau = std::sqrt(1. + ux * ux + uy * uy + tau0 * tau0 * ueta * ueta);
                term[(size_t)r * g.hx + iy] =
                    std::abs(kHbarc * e * gfactor) * g.ha * g.ha * it * dtau * a;
                if (std::abs(kHbarc * e * gfactor) > 0.0000000001) {
                    out.num(std::abs(kHbarc * e * gfactor)).ch(' ').num(utau).ch(' ');
                    out.num(ux).ch(' ').num(uy).ch(' ').num(ueta).ch(' ');
                    out.num(q00 * gfactor).ch(' ').num(q0x * gfactor).ch(' ');
                    out.num(q0y * gfactor).ch(' ').num(q0e * gfactor).ch(' ');
                    out.num(qxx * gfactor).ch(' ').num(qxy * gfactor).ch(' ');
                    out.num(qxe * gfactor).ch(' ').num(qyy * gfactor).ch(' ');
                    out.num(qye * gfactor).ch(' ').num(qee * gfactor).ch('\n');
                    continue;
                }
            }
            out.num(0.).ch(' ').num(1.);
            for (int k = 0; k < 13; k++) out.ch(' ').num(0.);
            out.ch('\n');
        }
        if (ix == g.hx - 1) {
            out.line(0);
            out.ch('\n');
        }
    };
    const bool ok = format_and_write(path, head, rows, (size_t)g.hx * 140, body);
    if (!ok) return IPG_ERR_BAD_CONFIG;
    if (Etot) {
        // the reference's running sum, in its loop order; points outside the
        // lattice hold +0, which leaves a non-negative sum unchanged
        double etot = 0.;
        for (double v : term) etot += v;
        *Etot = etot;
    }
    return IPG_OK;
}

ipg_status ipg_write_tmunu(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *T10, double gfactor) {
    if (!path || !T10 || N < 1 || sizeOutput < 1) return IPG_ERR_BAD_CONFIG;
    Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput, detaOutput};
    const int nn = N * N;
    const size_t n = (size_t)nn;
    const double tau0 = it * dtau * g.a;
    const Text head = tmunu_head(g);
    // one output row = iy: hx lines and a blank line
    auto body = [&](Text &out, int iy) {
        for (int ix = 0; ix < g.hx; ix++) {
            const double x = -g.hL / 2. + g.ha * ix;
            const double y = -g.hL / 2. + g.ha * iy;
            out.line(12);
            out.num(ix).ch(' ').num(iy).ch(' ');
            if (std::abs(x) < L / 2. && std::abs(y) < L / 2.) {
                const Stencil s = stencil(g, x, y);
                const double t00 = interp(s, nn, T10, false);
                const double t0x = interp(s, nn, T10 + 4 * n, false);
                const double t0y = interp(s, nn, T10 + 5 * n, false);
                const double t0e = interp(s, nn, T10 + 6 * n, false);
                const double txx = interp(s, nn, T10 + n, false);
                const double txy = interp(s, nn, T10 + 7 * n, false);
                const double txe = interp(s, nn, T10 + 8 * n, false);
                const double tyy = interp(s, nn, T10 + 2 * n, false);
                const double tye = interp(s, nn, T10 + 9 * n, false);
                const double tee = interp(s, nn, T10 + 3 * n, false);
                if (t00 * gfactor * kHbarc > kSmallEps) {
                    out.num(t00 * gfactor * kHbarc).ch(' ');
                    out.num(txx * gfactor * kHbarc).ch(' ').num(tyy * gfactor * kHbarc).ch(' ');
                    out.num(tau0 * tau0 * tee * gfactor * kHbarc).ch(' ');
                    out.num(-t0x * gfactor * kHbarc).ch(' ').num(-t0y * gfactor * kHbarc).ch(' ');
                    out.num(-tau0 * t0e * gfactor * kHbarc).ch(' ');
                    out.num(-txy * gfactor * kHbarc).ch(' ');
                    out.num(-tau0 * tye * gfactor * kHbarc).ch(' ');
                    out.num(-tau0 * txe * gfactor * kHbarc).ch('\n');
                    continue;
                }
            }
            out.num(kSmallEps).ch(' ').num(kSmallEps / 2.).ch(' ').num(kSmallEps / 2.);
            for (int k = 0; k < 7; k++) out.ch(' ').num(0.0);
            out.ch('\n');
        }
        out.line(0);
        out.ch('\n');
    };
    return format_and_write(path, head, g.hx, (size_t)g.hx * 110, body) ? IPG_OK
                                                                        : IPG_ERR_BAD_CONFIG;
}

// File names of the reference (MyEigen.cpp:376-383, 804-807): the time is
// printed with the default iostream format.
ipg_status ipg_output_names(int event_id, int it, double dtau, double a, char *hydro,
                            size_t hydro_len, char *tmunu, size_t tmunu_len) {
    std::ostringstream h, t;
    h << "epsilon-u-Hydro-TauHydro-" << event_id << ".dat";
    t << "Tmunu-t" << it * dtau * a << "-" << event_id << ".dat";
    if (hydro && hydro_len) std::snprintf(hydro, hydro_len, "%s", h.str().c_str());
    if (tmunu && tmunu_len) std::snprintf(tmunu, tmunu_len, "%s", t.str().c_str());
    return IPG_OK;
}

}  // extern "C"
