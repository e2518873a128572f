// ipglasma_b200 [input] [nev] -- drop-in for the reference executable's event
// loop (main.cpp:47-399) on the per-event hot path.
//
// Reads the reference's key/value input file with the reference's lookup
// rules (Setup.cpp:24-104: keys and values alternate, the file ends with
// EndOfFile, a missing key ends the program), derives dtau like main.cpp:531-534,
// and for each event either
//   - reads V_A, V_B from the Wilson-line files of readInitialWilsonLines
//     = 1 (text, Init.cpp:1879-1911 / 2036-2114) or 2 (binary, Init.cpp:
//     1914-1973 / 2120-2296),
//   - or samples the two nuclei (Woods-Saxon with minimum distance, the
//     algorithm of Init.cpp:2749-2816) on the host and builds the g^2 mu^2
//     maps on the device (ipg_set_nuclei) from the nucleon thickness:
//     T_A = sum of Gaussians of width BG (GeV^-2), and
//     Q_s(x) = QsMax sqrt(T_A(x)/max T_A) with QsMax from the optional key
//     QsMax (default 1.5 GeV), g^2 mu^2 a^2 = Q_s^2/QsmuRatio^2 a^2/(hbar c)^2/g^2;
//     or, when the input names an existing NucleusQsTableFileName, the
//     reference's IP-Sat construction from that Q_s(T_p, y) table
//     (ipg_set_nuclei_ipsat: fluctuating x, rmax cut, hard-sphere wounding).
// then runs the event on the GPU through the C ABI and writes the reference's
// output files (writeOutputs 1, 4, 5) and, on request, the V files
// (writeInitialWilsonLines = 1 text or 2 binary).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "ipglasma_b200.h"

namespace {

constexpr double kHbarc = 0.1973269718;

// ------------------------------------------------------ gluon multiplicity
// The lines Evolution::multiplicity prints (Evolution.cpp:2318-2330,
// 3094-3109, with GaugeFix.cpp:48-92's residual every 10 iterations)
void print_multiplicity(const ipg_multiplicity_result &m, const ipg_multiplicity_params &p) {
    std::cout << "Measuring multiplicity ... " << std::endl;
    std::cout << "gauge fixing" << std::endl;
    for (int k = 0; k < 401 && 10 * k < m.gauge.residual_checks; k++)
        std::cout << 10 * k << " " << m.gauge.residual_every10[k] << std::endl;
    if (p.use_pseudorapidity == 0) {
        std::cout << "dN/dy 1 = " << m.dNdy << ", dE/dy 1 = " << m.dEdy << std::endl;
        std::cout << "dN/dy 2 = " << m.dNdy_binned << ", dE/dy 2 = " << m.dEdy_binned
                  << std::endl;
    } else {
        std::cout << "dN/deta 1 = " << m.dNdy << ", dE/deta 1 = " << m.dEdy << std::endl;
        std::cout << "dN/deta 2 = " << m.dNdy_binned << ", dE/deta 2 = " << m.dEdy_binned
                  << std::endl;
        std::cout << "dN/deta_cut 1 = " << m.dNdy_cut3 << std::endl;
        std::cout << "dN/deta_cut 2 = " << m.dNdy_cut6 << std::endl;
    }
    std::cout << "gluon <p_T> = " << m.mean_pt << std::endl;
    std::cout << " done." << std::endl;
}

// eccentricities<id>.dat, appended, at it = itmax (Evolution.cpp:1800-1810):
// tau, epsilon_n and Psi_n for n = 1..6, the cutoff (0), sqrt(<r^2>), the
// outermost weighted cells on the centroid's row and column, b, T_pp, the
// area, Rbar, the mean e and the mean Q_sA^2 Q_sB^2. The reference also
// writes a line at it = 1, from energy densities its cells do not hold at
// that time; that line is not written here.
void write_eccentricities(ipg_ctx *ctx, int event_id, const ipg_result &r, double b, double Tpp,
                          double QsmuRatio) {
    ipg_ecc_report e;
    if (ipg_eccentricity_report(ctx, QsmuRatio, QsmuRatio, &e) != IPG_OK) {
        std::cerr << "ipg_eccentricity_report: " << ipg_last_error(ctx) << std::endl;
        return;
    }
    std::stringstream name;
    name << "eccentricities" << event_id << ".dat";
    std::ofstream f(name.str().c_str(), std::ios::app);
    f << e.tau;
    for (int k = 0; k < 6; k++) f << " " << r.eccentricity[k] << " " << r.psi[k];
    f << " " << 0. << " " << e.r_rms << " " << e.max_x << " " << e.max_y << " " << b << " "
      << Tpp << " " << e.area << " " << e.Rbar << " " << e.avg_eps << " " << e.avg_qs2a_qs2b
      << std::endl;
}

// NpartdNdy-t<tau>-<id>.dat at it = itmax (Evolution.cpp:3124-3152): N_part,
// dN/dy, T_pp, b, dE/dy, the seed, three N/A, the 3 and 6 GeV cuts and the
// coupling ratio at the event's average Q_s
void write_npart_dndy(int event_id, int itmax, double dtau, double a,
                      const ipg_ipsat_report &ir, double b, unsigned long long seed,
                      const ipg_multiplicity_result &m, double g, double muZero, double c,
                      double qsFactor) {
    std::stringstream name;
    name << "NpartdNdy-t" << itmax * dtau * a << "-" << event_id << ".dat";
    std::ofstream f(name.str().c_str(), std::ios::out);
    f << ir.Npart << " " << m.dNdy << " " << ir.Tpp << " " << b << " " << m.dEdy << " " << seed
      << " " << "N/A" << " " << "N/A" << " " << "N/A" << " " << m.dNdy_cut3 << " "
      << m.dEdy_cut3 << " " << m.dNdy_cut6 << " " << m.dEdy_cut6 << " "
      << g * g /
             (4. * M_PI * 4. * M_PI /
              (9. * std::log(std::pow(std::pow(muZero / 0.2, 2. / c) +
                                          std::pow(qsFactor * ir.average_Qs / 0.2, 2. / c),
                                      c))))
      << std::endl;
}

// ---------------------------------------------------------------- input file
class InputFile {
  public:
    explicit InputFile(const std::string &name) : name_(name) {
        std::ifstream in(name.c_str());
        if (!in) {
            std::cerr << "The input file named " << name << " is absent. Exiting." << std::endl;
            std::exit(1);
        }
        std::string k, v;
        while (in >> k) {
            if (k == "EndOfFile") break;
            if (!(in >> v)) break;
            pairs_.push_back({k, v});
        }
    }
    bool has(const std::string &key) const {
        for (const auto &p : pairs_)
            if (p.first == key) return true;
        return false;
    }
    std::string str(const std::string &key) const {
        for (const auto &p : pairs_)
            if (p.first == key) return p.second;
        std::cerr << key << " not found in " << name_ << std::endl;
        std::cout << "Create a complete input file." << std::endl;
        std::exit(1);
    }
    double d(const std::string &key) const { return std::atof(str(key).c_str()); }
    int i(const std::string &key) const { return static_cast<int>(d(key)); }
    unsigned long long ull(const std::string &key) const {
        return static_cast<unsigned long long>(d(key) + 0.5);
    }
    double d_or(const std::string &key, double def) const { return has(key) ? d(key) : def; }

  private:
    std::string name_;
    std::vector<std::pair<std::string, std::string>> pairs_;
};

// ------------------------------------------------------------ nuclei, g2mu
struct Species {
    int A;
    double R, a;
};

Species species(const std::string &name, const InputFile &in) {
    static const std::map<std::string, Species> table = {
        {"p", {1, 0.0, 0.0}},        {"O", {16, 2.608, 0.513}},
        {"Cu", {63, 4.20641, 0.5977}}, {"Xe", {129, 5.36, 0.59}},
        {"Au", {197, 6.38, 0.535}},  {"Pb", {208, 6.62, 0.546}},
        {"U", {238, 6.81, 0.6}}};
    auto it = table.find(name);
    if (it == table.end()) {
        std::cerr << "nucleus " << name << " is not supported by this executable" << std::endl;
        std::exit(1);
    }
    Species s = it->second;
    if (in.i("setWSDeformParams")) {  // the input's R_WS, a_WS for both nuclei
        s.R = in.d("R_WS");
        s.a = in.d("a_WS");
    }
    return s;
}

std::vector<double> sample_nucleus(std::mt19937_64 &rng, const Species &s, double dmin) {
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::vector<double> xyz(3 * s.A, 0.0);
    if (s.A == 1) return xyz;
    const double rmax = s.R + 10.0 * s.a;
    std::vector<double> r(s.A);
    for (int i = 0; i < s.A; i++) {
        for (;;) {
            const double ri = rmax * std::pow(U(rng), 1.0 / 3.0);
            if (U(rng) <= 1.0 / (1.0 + std::exp((ri - s.R) / s.a))) {
                r[i] = ri;
                break;
            }
        }
    }
    std::sort(r.begin(), r.end());
    const double d2 = dmin * dmin;
    for (int i = 0; i < s.A; i++) {
        double x = 0, y = 0, z = 0;
        for (int tries = 0; tries < 100; tries++) {
            const double phi = 2.0 * M_PI * U(rng);
            const double th = std::acos(1.0 - 2.0 * U(rng));
            x = r[i] * std::sin(th) * std::cos(phi);
            y = r[i] * std::sin(th) * std::sin(phi);
            z = r[i] * std::cos(th);
            bool ok = true;
            for (int j = i - 1; j >= 0 && (r[i] - r[j]) * (r[i] - r[j]) <= d2; j--) {
                const double dx = x - xyz[3 * j], dy = y - xyz[3 * j + 1], dz = z - xyz[3 * j + 2];
                if (dx * dx + dy * dy + dz * dz < d2) {
                    ok = false;
                    break;
                }
            }
            if (ok) break;
        }
        xyz[3 * i] = x;
        xyz[3 * i + 1] = y;
        xyz[3 * i + 2] = z;
    }
    double m[3] = {0, 0, 0};
    for (int i = 0; i < s.A; i++)
        for (int k = 0; k < 3; k++) m[k] += xyz[3 * i + k] / s.A;
    for (int i = 0; i < s.A; i++)
        for (int k = 0; k < 3; k++) xyz[3 * i + k] -= m[k];
    // uniform random orientation: rotate by a random unit quaternion
    std::normal_distribution<double> G(0.0, 1.0);
    double q[4] = {G(rng), G(rng), G(rng), G(rng)};
    const double qn = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (double &v : q) v /= qn;
    const double w = q[0], a = q[1], b = q[2], c = q[3];
    const double R[9] = {1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w),
                         2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w),
                         2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)};
    for (int i = 0; i < s.A; i++) {
        const double v[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        for (int k = 0; k < 3; k++) xyz[3 * i + k] = R[3 * k] * v[0] + R[3 * k + 1] * v[1] + R[3 * k + 2] * v[2];
    }
    return xyz;
}

// ------------------------------------------------------------- V files
void write_vfile(const std::string &name, int N, double L, double y, const std::vector<double> &V) {
    std::ofstream f(name.c_str(), std::ios::out | std::ios::binary);
    int nc = 3;
    double a = L / N;
    f.write((const char *)&N, sizeof(int));
    f.write((const char *)&nc, sizeof(int));
    f.write((const char *)&L, sizeof(double));
    f.write((const char *)&a, sizeof(double));
    f.write((const char *)&y, sizeof(double));
    // record ix*N+iy holds the cell N*iy+ix (Init.cpp:1943-1957)
    for (int ix = 0; ix < N; ix++)
        for (int iy = 0; iy < N; iy++)
            f.write((const char *)&V[18 * ((size_t)N * iy + ix)], 18 * sizeof(double));
}

// Text format of writeInitialWilsonLines = 1 (Init.cpp:1879-1911): per site
// "ix iy" and the 9 entries as (re, im) pairs in column-major order
// (Matrix::MatrixToString, Matrix.cpp:606-622), 15 significant digits, a
// blank line after each ix row.
void write_vtext(const std::string &name, int N, const std::vector<double> &V) {
    FILE *f = std::fopen(name.c_str(), "w");
    if (!f) {
        std::cerr << "cannot write " << name << std::endl;
        std::exit(1);
    }
    static const int colmajor[9] = {0, 3, 6, 1, 4, 7, 2, 5, 8};
    for (int ix = 0; ix < N; ix++) {
        for (int iy = 0; iy < N; iy++) {
            const double *m = &V[18 * ((size_t)ix * N + iy)];
            std::fprintf(f, "%d %d", ix, iy);
            for (int k : colmajor) std::fprintf(f, " %.15g %.15g", m[2 * k], m[2 * k + 1]);
            std::fputc('\n', f);
        }
        std::fputc('\n', f);
    }
    std::fclose(f);
}

// Text read of readInitialWilsonLines = 1 (Init.cpp:2036-2114): the entries
// are taken in row-major order (so a file written by write_vtext comes back
// transposed, as in the reference), and line i goes to ix = (int)((a i -+ b/2)
// / a), truncated toward zero; rows with ix < 0 (nucleus A) or ix >= N
// (nucleus B) are skipped, cells no line reaches keep the identity.
bool read_vtext(const std::string &name, int N, double L, double shift, std::vector<double> &V) {
    std::ifstream f(name.c_str());
    if (!f) return false;
    V.assign((size_t)18 * N * N, 0.0);
    for (int k = 0; k < N * N; k++) V[18 * (size_t)k] = V[18 * (size_t)k + 8] = V[18 * (size_t)k + 16] = 1.0;
    const double a = L / N;
    double dummy, re[9], im[9];
    for (int i = 0; i < N; i++) {
        for (int j = 0; j < N; j++) {
            f >> dummy >> dummy;
            for (int k = 0; k < 9; k++) f >> re[k] >> im[k];
            const int ix = (int)((a * i + shift) / a);
            if (ix < 0 || ix >= N) continue;
            double *m = &V[18 * ((size_t)ix * N + j)];
            for (int k = 0; k < 9; k++) {
                m[2 * k] = re[k];
                m[2 * k + 1] = im[k];
            }
        }
    }
    return true;
}

bool read_vfile(const std::string &name, int N, double L, double shift, std::vector<double> &V) {
    std::ifstream f(name.c_str(), std::ios::in | std::ios::binary);
    if (!f) return false;
    int n = 0, nc = 0;
    double l = 0, a = 0, y = 0;
    f.read((char *)&n, sizeof(int));
    f.read((char *)&nc, sizeof(int));
    f.read((char *)&l, sizeof(double));
    f.read((char *)&a, sizeof(double));
    f.read((char *)&y, sizeof(double));
    if (n != N || std::abs(l - L) > 1e-5) {
        std::cerr << "# ERROR V file " << name << " has N=" << n << " L=" << l << std::endl;
        return false;
    }
    V.assign((size_t)18 * N * N, 0.0);
    for (int k = 0; k < N * N; k++) V[18 * (size_t)k] = V[18 * (size_t)k + 8] = V[18 * (size_t)k + 16] = 1.0;
    const double aa = L / N;
    std::vector<double> rec(18);
    for (long r = 0; r < (long)N * N; r++) {
        if (!f.read((char *)rec.data(), 18 * sizeof(double))) break;
        const int iy = (int)(r / N), ixIn = (int)(r - (long)N * iy);
        const int ix = (int)std::round((aa * ixIn + shift) / aa);  // Init.cpp:2190-2194
        const long idx = (long)N * ix + iy;
        if (idx < 0 || idx >= (long)N * N) continue;
        std::memcpy(&V[18 * (size_t)idx], rec.data(), 18 * sizeof(double));
    }
    return true;
}

// The Q_s^2(T, y) table of readNuclearQs (Init.cpp:441-480): records
// "y T Q_s^2", ny = 44 rapidities 0.25 apart per T, nT = 200 values of T.
bool read_qs_table(const std::string &name, std::vector<double> &Tlist, std::vector<double> &qs2,
                   int nT = 200, int ny = 44) {
    std::ifstream f(name.c_str());
    if (!f) return false;
    Tlist.assign(nT, 0.0);
    qs2.assign((size_t)nT * ny, 0.0);
    double y, T, q;
    for (int iT = 0; iT < nT; iT++)
        for (int iy = 0; iy < ny; iy++) {
            if (!(f >> y >> T >> q)) {
                std::cerr << " End of file reached prematurely. Did the file change? Exiting."
                          << std::endl;
                std::exit(1);
            }
            Tlist[iT] = T;
            qs2[(size_t)iT * ny + iy] = q;
        }
    return true;
}

void check(ipg_ctx *ctx, ipg_status st, const char *what) {
    if (st == IPG_OK) return;
    std::cerr << what << " failed (" << st << "): " << ipg_last_error(ctx) << std::endl;
    if (st != IPG_ERR_NEWTON_NONCONVERGED) std::exit(1);
}

}  // namespace

int main(int argc, char **argv) {
    const std::string file = argc > 1 ? argv[1] : "input";
    const int nev = argc == 3 ? std::atoi(argv[2]) : 1;
    InputFile in(file);

    ipg_config cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.size = in.i("size");
    cfg.Nc = in.i("Nc");
    cfg.Ny = in.i("Ny");
    cfg.L = in.d("L");
    cfg.g = in.d("g");
    cfg.m = in.d("m");
    cfg.UVdamp = in.d("UVdamp");
    cfg.maxtime = in.d("maxtime");
    cfg.dtau = in.d_or("dtauOverride", 0.0);  // the reference derives dtau
    cfg.precision = in.d_or("precisionFP32", 0.0) > 0 ? IPG_FP32 : IPG_FP64;
    cfg.device = (int)in.d_or("device", 0.0);
    cfg.newton_mode = (int)in.d_or("newtonMode", 0.0);  // 1: Newton on the group
    const int writeOutputs = in.i("writeOutputs");
    const int sizeOutput = in.i("sizeOutput");
    const double LOutput = in.d("LOutput");
    const int etaSizeOutput = in.i("etaSizeOutput");
    const double detaOutput = in.d("detaOutput");
    const int readV = in.i("readInitialWilsonLines");
    const int writeV = in.i("writeInitialWilsonLines");
    const int useNucleus = in.i("useNucleus");
    const double bmin = in.d("bmin"), bmax = in.d("bmax");
    const int linearb = in.i("samplebFromLinearDistribution");
    const double BG = in.d("BG"), QsmuRatio = in.d("QsmuRatio");
    const double QsMax = in.d_or("QsMax", 1.5);
    // the IP-Sat Q_s(T, y) table when the input names one that exists,
    // else the Q_s ~ sqrt(T_A) map with QsMax
    std::vector<double> Tlist, qs2tab;
    bool ipsat = false;
    ipg_ipsat_params ips;
    std::memset(&ips, 0, sizeof(ips));
    if (in.has("NucleusQsTableFileName") &&
        read_qs_table(in.str("NucleusQsTableFileName"), Tlist, qs2tab)) {
        ipsat = true;
        ips.BG = in.d("BG");
        ips.QsmuRatio = ips.QsmuRatioB = in.d("QsmuRatio");
        ips.proton_anisotropy = in.d_or("protonAnisotropy", 0.0);
        ips.rapidity = in.d("Rapidity");
        ips.roots = in.d("roots");
        ips.x_factor = in.d("xFromThisFactorTimesQs");
        ips.rmax = in.d("rmax");
        ips.sigmaNN = in.d("SigmaNN");
        ips.use_fluctuating_x = in.i("useFluctuatingx");
        ips.average_over_nuclei = std::max(1, (int)in.d_or("averageOverThisManyNuclei", 1.0));
        if (ips.proton_anisotropy != 0.0 || in.d_or("smearQs", 0.0) != 0.0 ||
            in.d_or("useConstituentQuarkProton", 0.0) != 0.0)
            std::cerr << "note: protonAnisotropy, smearQs and constituent quarks are not used "
                         "by this executable (round nucleons, unit Q_s normalisation)"
                      << std::endl;
    }
    const double rapidity = in.d("Rapidity");
    // Evolution::multiplicity at it = 1 and it = itmax (Evolution.cpp:644-653)
    const int gluonMult = (int)in.d_or("computeGluonMultiplicity", 0.0);
    ipg_multiplicity_params mparams{};
    mparams.max_gauge_iterations = 4000;
    mparams.use_pseudorapidity = (int)in.d_or("usePseudoRapidity", 0.0);
    mparams.rapidity = rapidity;
    mparams.jacobian_m = in.d_or("Jacobianm", 0.35);
    mparams.roots = in.d_or("roots", 7000.0);
    const double muZero = in.d_or("muZero", 0.3), cRun = in.d_or("c", 0.2),
                 qsFactor = in.d_or("runWithThisFactorTimesQs", 0.5);
    unsigned long long seed = in.ull("seed");
    if (in.i("useTimeForSeed") == 1) seed = std::random_device{}();
    if (readV < 0 || readV > 2 || writeV < 0 || writeV > 2) {
        std::cerr << "# Unknown Wilson-line format: readInitialWilsonLines " << readV
                  << ", writeInitialWilsonLines " << writeV << " (supported: 0, 1 text, 2 binary)"
                  << std::endl;
        return 1;
    }
    std::cout << "Random seed = " << seed << std::endl;

    std::mt19937_64 rng(seed);
    ipg_ctx *ctx = nullptr;
    cfg.seed = seed;
    check(ctx, ipg_create(&cfg, &ctx), "ipg_create");
    double dtau = 0;
    int itmax = 0;
    ipg_time_grid(ctx, &dtau, &itmax);
    const int N = cfg.size;
    const size_t n = (size_t)N * N;
    const double a = cfg.L / N;

    for (int iev = 0; iev < nev; iev++) {
        const int event_id = iev;  // rank + iev * size with one rank
        const auto t0 = std::chrono::steady_clock::now();
        std::uniform_real_distribution<double> U(0.0, 1.0);
        const double xb = U(rng);
        double b = 0.0;
        if (useNucleus)
            b = linearb ? std::sqrt((bmax * bmax - bmin * bmin) * xb + bmin * bmin)
                        : (bmax - bmin) * xb + bmin;
        ipg_init_report rep;
        std::memset(&rep, 0, sizeof(rep));
        ipg_ipsat_report irep;
        std::memset(&irep, 0, sizeof(irep));
        if (readV != 0) {
            std::vector<double> VA, VB;
            std::ostringstream n1, n2;
            n1 << "V-" << event_id + 2 * seed;
            n2 << "V-" << event_id + (1 + 2 * seed);
            if (readV == 1) {
                n1 << ".txt";
                n2 << ".txt";
            }
            auto rd = readV == 1 ? read_vtext : read_vfile;
            if (!rd(n1.str(), N, cfg.L, -b / 2., VA) || !rd(n2.str(), N, cfg.L, b / 2., VB)) {
                std::cerr << "cannot read the Wilson-line files " << n1.str() << ", " << n2.str()
                          << std::endl;
                return 1;
            }
            check(ctx, ipg_set_field(ctx, IPG_VA, VA.data()), "ipg_set_field");
            check(ctx, ipg_set_field(ctx, IPG_VB, VB.data()), "ipg_set_field");
            check(ctx, ipg_init_from_wilson_lines(ctx, &rep), "ipg_init_from_wilson_lines");
        } else {
            const Species sA = species(in.str("Projectile"), in);
            const Species sB = species(in.str("Target"), in);
            const double dmin = in.i("setWSDeformParams") ? in.d("d_min") : 0.4;
            const auto nA = sample_nucleus(rng, sA, dmin);
            const auto nB = sample_nucleus(rng, sB, dmin);
            if (ipsat) {
                check(ctx,
                      ipg_set_nuclei_ipsat(ctx, nA.data(), (int)(nA.size() / 3), nB.data(),
                                           (int)(nB.size() / 3), nullptr, nullptr, nullptr,
                                           nullptr, b, &ips, Tlist.data(), qs2tab.data(), 200,
                                           44, 0.25, &irep),
                      "ipg_set_nuclei_ipsat");
                std::cout << "N_part=" << irep.Npart << " N_coll=" << irep.Ncoll
                          << " Average Qs(max) = " << irep.average_Qs << " GeV" << std::endl;
            } else {
                check(ctx,
                      ipg_set_nuclei(ctx, nA.data(), (int)(nA.size() / 3), nB.data(),
                                     (int)(nB.size() / 3), b, BG, QsMax, QsmuRatio),
                      "ipg_set_nuclei");
            }
            check(ctx, ipg_reseed(ctx, seed * 1000003ULL + event_id), "ipg_reseed");
            check(ctx, ipg_use_device_noise(ctx), "ipg_use_device_noise");
            check(ctx, ipg_init_fields(ctx, &rep), "ipg_init_fields");
            if (writeV != 0) {
                std::vector<double> V(18 * n);
                std::ostringstream n1, n2;
                n1 << "V-" << event_id + 2 * seed;
                n2 << "V-" << event_id + (1 + 2 * seed);
                if (writeV == 1) {
                    n1 << ".txt";
                    n2 << ".txt";
                }
                check(ctx, ipg_get_field(ctx, IPG_VA, V.data()), "ipg_get_field");
                if (writeV == 1) write_vtext(n1.str(), N, V);
                else write_vfile(n1.str(), N, cfg.L, rapidity, V);
                check(ctx, ipg_get_field(ctx, IPG_VB, V.data()), "ipg_get_field");
                if (writeV == 1) write_vtext(n2.str(), N, V);
                else write_vfile(n2.str(), N, cfg.L, rapidity, V);
            }
        }
        ipg_result res;
        if (gluonMult) {
            ipg_multiplicity_result m1, m2;
            const ipg_status st = ipg_run_multiplicity(ctx, &mparams, &res, &m1, &m2);
            if (itmax >= 2) print_multiplicity(m1, mparams);
            if (st == IPG_NO_COLLISION) {
                // Evolution.cpp:3111-3122 and 655: the evolution of this event
                // stops after the spectrum at it = 1, no output files
                std::cout << "No collision happened on rank 0. Restarting with new random "
                             "number..."
                          << std::endl;
                continue;
            }
            check(ctx, st, "ipg_run_multiplicity");
            write_eccentricities(ctx, event_id, res, b, irep.Tpp, QsmuRatio);
            print_multiplicity(m2, mparams);
            write_npart_dndy(event_id, itmax, dtau, a, irep, b, seed, m2, cfg.g, muZero, cRun,
                             qsFactor);
        } else {
            check(ctx, ipg_run(ctx, &res), "ipg_run");
        }
        char hname[256], tname[256];
        ipg_output_names(event_id, itmax, dtau, a, hname, sizeof(hname), tname, sizeof(tname));
        // both files resampled and formatted on the GPU from the device
        // observables (the same bytes as the host writers)
        const bool hydro = writeOutputs % 2 == 1, kompost = writeOutputs / 4 == 1;
        if (hydro || kompost) {
            double etot = 0;
            check(ctx,
                  ipg_write_outputs(ctx, hydro ? hname : nullptr, kompost ? tname : nullptr,
                                    sizeOutput, LOutput, etaSizeOutput, detaOutput, itmax, dtau,
                                    1.0, &etot),
                  "ipg_write_outputs");
            if (hydro) std::cout << "Etot = " << etot << " GeV " << std::endl;
        }
        const double sec =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout << "event " << event_id << ": b=" << b << " fm, itmax=" << res.itmax
                  << ", Gauss violation=" << res.gauss_violation
                  << ", eps2=" << res.eccentricity[1] << ", E_T=" << res.E_T
                  << " GeV, Newton restarts/failures=" << rep.newton_restarted << "/"
                  << rep.newton_failed << ", " << sec << " s" << std::endl;
    }
    ipg_destroy(ctx);
    return 0;
}
