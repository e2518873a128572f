// Output files for hydrodynamics and kinetic theory, in the reference's text
// formats (MyEigen::flowVelocity4D output part, MyEigen.cpp:329-1045):
//   epsilon-u-Hydro-TauHydro-<id>.dat   writeOutputs odd   (MyEigen.cpp:380-797)
//   Tmunu-t<tau>-<id>.dat               writeOutputs/4 == 1 (MyEigen.cpp:801-1045)
// Both resample the N x N lattice bilinearly onto sizeOutput^2 points over
// LOutput, keeping the reference's conventions: the fractional offset is
// divided by the OUTPUT spacing, a neighbour pair counts only if both sites
// have an index strictly greater than 0, e <= 1e-10 GeV/fm^3 (hydro) and
// T^tautau <= 1e-16 (Tmunu) become placeholder rows, u^tau is recomputed from
// the normalisation, and numbers are printed with the default iostream format
// (6 significant digits). Host code, fed from ipg_get_observables.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/ipglasma_b200.h"

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

}  // namespace

extern "C" {

ipg_status ipg_write_hydro(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *eps,
                           const double *u4, const double *pi10, double gfactor,
                           double *Etot) {
    if (!path || !eps || !u4 || !pi10 || N < 1 || sizeOutput < 1) return IPG_ERR_BAD_CONFIG;
    Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput, detaOutput};
    const int nn = N * N;
    const double a = g.a;
    const double tau0 = it * dtau * a;
    std::ofstream out(path, std::ios::out);
    if (!out) return IPG_ERR_BAD_CONFIG;
    out << "# dummy " << 1 << " etamax= " << g.heta << " xmax= " << g.hx
        << " ymax= " << g.hx << " deta= " << g.deta << " dx= " << g.ha
        << " dy= " << g.ha << " tau= " << tau0 << std::endl;
    const size_t n = (size_t)nn;
    // pi10 order: tautau xx yy etaeta taux tauy taueta xy xeta yeta
    const double *p00 = pi10, *pxx = pi10 + n, *pyy = pi10 + 2 * n, *pee = pi10 + 3 * n;
    const double *p0x = pi10 + 4 * n, *p0y = pi10 + 5 * n, *p0e = pi10 + 6 * n;
    const double *pxy = pi10 + 7 * n, *pxe = pi10 + 8 * n, *pye = pi10 + 9 * n;
    double etot = 0.;
    for (int ieta = 0; ieta < g.heta; ieta++) {
        const double eta = -(g.heta - 1) / 2. * g.deta + g.deta * ieta;
        for (int ix = 0; ix < g.hx; ix++) {
            for (int iy = 0; iy < g.hx; iy++) {
                const double x = -g.hL / 2. + g.ha * ix;
                const double y = -g.hL / 2. + g.ha * iy;
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
                    const double utau =
                        std::sqrt(1. + ux * ux + uy * uy + tau0 * tau0 * ueta * ueta);
                    etot += std::abs(kHbarc * e * gfactor) * g.ha * g.ha * it * dtau * a;
                    if (std::abs(kHbarc * e * gfactor) > 0.0000000001) {
                        out << eta << " " << x << " " << y << " "
                            << std::abs(kHbarc * e * gfactor) << " " << utau << " " << ux
                            << " " << uy << " " << ueta << " " << q00 * gfactor << " "
                            << q0x * gfactor << " " << q0y * gfactor << " " << q0e * gfactor
                            << " " << qxx * gfactor << " " << qxy * gfactor << " "
                            << qxe * gfactor << " " << qyy * gfactor << " " << qye * gfactor
                            << " " << qee * gfactor << std::endl;
                        continue;
                    }
                }
                out << eta << " " << x << " " << y << " " << 0. << " " << 1. << " " << 0.
                    << " " << 0. << " " << 0. << " " << 0. << " " << 0. << " " << 0. << " "
                    << 0. << " " << 0. << " " << 0. << " " << 0. << " " << 0. << " " << 0.
                    << " " << 0. << std::endl;
            }
        }
        out << std::endl;
    }
    if (Etot) *Etot = etot;
    return out.good() ? IPG_OK : IPG_ERR_BAD_CONFIG;
}

ipg_status ipg_write_tmunu(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *T10, double gfactor) {
    if (!path || !T10 || N < 1 || sizeOutput < 1) return IPG_ERR_BAD_CONFIG;
    Grid g{N, L, L / N, sizeOutput, etaSizeOutput, LOutput, LOutput / sizeOutput, detaOutput};
    const int nn = N * N;
    const size_t n = (size_t)nn;
    const double tau0 = it * dtau * g.a;
    std::ofstream out(path, std::ios::out);
    if (!out) return IPG_ERR_BAD_CONFIG;
    out << "# dummy " << 1 << " etamax= " << g.heta << " xmax= " << g.hx
        << " ymax= " << g.hx << " deta= " << g.deta << " dx= " << g.ha
        << " dy= " << g.ha << std::endl;
    for (int iy = 0; iy < g.hx; iy++) {
        for (int ix = 0; ix < g.hx; ix++) {
            const double x = -g.hL / 2. + g.ha * ix;
            const double y = -g.hL / 2. + g.ha * iy;
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
                    out << ix << " " << iy << " " << t00 * gfactor * kHbarc << " "
                        << txx * gfactor * kHbarc << " " << tyy * gfactor * kHbarc << " "
                        << tau0 * tau0 * tee * gfactor * kHbarc << " "
                        << -t0x * gfactor * kHbarc << " " << -t0y * gfactor * kHbarc << " "
                        << -tau0 * t0e * gfactor * kHbarc << " " << -txy * gfactor * kHbarc
                        << " " << -tau0 * tye * gfactor * kHbarc << " "
                        << -tau0 * txe * gfactor * kHbarc << std::endl;
                    continue;
                }
            }
            out << ix << " " << iy << " " << kSmallEps << " " << kSmallEps / 2. << " "
                << kSmallEps / 2. << " " << 0.0 << " " << 0.0 << " " << 0.0 << " " << 0.0
                << " " << 0.0 << " " << 0.0 << " " << 0.0 << std::endl;
        }
        out << std::endl;
    }
    return out.good() ? IPG_OK : IPG_ERR_BAD_CONFIG;
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
