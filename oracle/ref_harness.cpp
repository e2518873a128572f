// Oracle harness: drives the UNMODIFIED reference IP-Glasma classes, compiled
// from the reference's own sources (Init.cpp, Evolution.cpp, MyEigen.cpp, ...)
// against the project's FFTW/GSL subset in oracle/shim.
//
// TEST INFRASTRUCTURE ONLY. Only the tests, the smoke check and the CPU
// baseline leg of bench.py run this program; the shipped library never does.
//
// It uses only the reference's public API and file formats:
//   1. Parameters set through setters; useNucleus=0 so Init::init never
//      touches the Glauber / IP-Sat code (Init.cpp:2323-2348).
//   2. Identity Wilson-line files in the binary format of Init.cpp:1914-1973,
//      then Init::init(..., READFROMFILE=2) once so that the Init object
//      holds Nc_, group_ptr_ and one_ (Init.cpp:2308-2312), needed by setV.
//   3. g2mu2A/B set per cell (Cell::setg2mu2A/B), U and U2 reset to 1, then
//      Init::setV (Init.cpp:1678-1849) draws rho from a fresh Random seeded
//      with --seed and writes V files (writeInitialWilsonLines=2).
//   4. Init::init(..., 2) reads them back bit-exactly (Init.cpp:2120-2296)
//      and runs the tau=0 Newton link solve (Init.cpp:2437-2691).
//   5. Either Evolution::run (Evolution.cpp:366-657) or, in --mode steps, the
//      leapfrog sweeps evolvePhi/evolveU/evolvePi/evolveE in the order of
//      Evolution.cpp:393-421.
//   6. Evolution::eccentricity (Evolution.cpp:1280-1810) on the final cells.
// State and observables are dumped as raw little-endian doubles.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include <climits>
#include <cmath>
#include <complex>
#include <map>
#include <set>

#include "Evolution.h"
#include "Glauber.h"
#include "Group.h"
// The nucleon lists of Init are private; the IP-Sat mode fills them with the
// test's positions before calling the reference's own setColorChargeDensity
// (no reference source is changed: the access specifier is lifted for this
// translation unit's view of the class only).
#define private public
#include "Init.h"
#undef private
#include "Lattice.h"
#include "Matrix.h"
#include "Parameters.h"
#include "Random.h"

namespace {

struct Args {
    int N = 32;
    double L = 8.0;
    int Ny = 4;
    double g = 2.0;
    double m = 0.2;
    double uvdamp = 0.0;
    unsigned long long seed = 1;
    double maxtime = 0.2;
    double dtau = -1.0;  // lattice units; <0: derive like main.cpp:531-534
    std::string g2mu_file;
    std::string out = ".";
    std::string mode = "full";  // full | steps | init
    int steps = 0;
    int write_outputs = 0;
    int size_output = 0;
    double L_output = 0.0;
    int dumps = 1;  // 0: no state, noise or observable dumps (timing runs)
    // --mode ipsat: nucleon positions (binary: nA, nB as doubles, then x, y of
    // A, then of B, fm, unshifted), the Q_s table file, impact parameter and
    // the IP-Sat parameters
    std::string nucleons, table;
    double b = 0.0, BG = 4.0, QsmuRatio = 0.8, roots = 5020.0, rapidity = 0.0;
    double xfactor = 0.5, rmax = 3.0, sigmaNN = 70.0;
    int fluct = 1;
    // --multiplicity 1: Evolution::run with computeGluonMultiplicity set
    // (gauge fixing and the gluon spectrum at it = 1 and it = itmax); its
    // printed values come out with 17 digits
    int multiplicity = 0, pseudo = 0;
    double jacobian_m = 0.35;
};

void usage() {
    std::cerr << "usage: ipg_ref_harness --g2mu FILE --out DIR [--N n] [--L fm]"
                 " [--Ny n] [--g g] [--m GeV] [--uvdamp x] [--seed s]"
                 " [--maxtime fm] [--dtau lattice] [--mode full|steps|init]"
                 " [--steps k] [--write-outputs w] [--size-output n]"
                 " [--L-output fm] [--dumps 0|1] [--multiplicity 0|1 [--pseudo 0|1]"
                 " [--rapidity y] [--jacobian-m GeV] [--roots GeV]]\n"
                 "       ipg_ref_harness --mode ipsat --nucleons FILE --table FILE --out DIR"
                 " [--N n] [--L fm] [--g g] [--b fm] [--BG GeV^-2] [--QsmuRatio r]"
                 " [--roots GeV] [--rapidity y] [--xfactor f] [--rmax fm]"
                 " [--sigmaNN mb] [--fluct 0|1] [--seed s]\n";
    std::exit(2);
}

Args parse(int argc, char **argv) {
    Args a;
    for (int i = 1; i < argc; i++) {
        std::string k = argv[i];
        if (i + 1 >= argc) usage();
        std::string v = argv[++i];
        if (k == "--N") a.N = std::atoi(v.c_str());
        else if (k == "--L") a.L = std::atof(v.c_str());
        else if (k == "--Ny") a.Ny = std::atoi(v.c_str());
        else if (k == "--g") a.g = std::atof(v.c_str());
        else if (k == "--m") a.m = std::atof(v.c_str());
        else if (k == "--uvdamp") a.uvdamp = std::atof(v.c_str());
        else if (k == "--seed") a.seed = std::strtoull(v.c_str(), nullptr, 10);
        else if (k == "--maxtime") a.maxtime = std::atof(v.c_str());
        else if (k == "--dtau") a.dtau = std::atof(v.c_str());
        else if (k == "--g2mu") a.g2mu_file = v;
        else if (k == "--out") a.out = v;
        else if (k == "--mode") a.mode = v;
        else if (k == "--steps") a.steps = std::atoi(v.c_str());
        else if (k == "--write-outputs") a.write_outputs = std::atoi(v.c_str());
        else if (k == "--size-output") a.size_output = std::atoi(v.c_str());
        else if (k == "--L-output") a.L_output = std::atof(v.c_str());
        else if (k == "--dumps") a.dumps = std::atoi(v.c_str());
        else if (k == "--nucleons") a.nucleons = v;
        else if (k == "--table") a.table = v;
        else if (k == "--b") a.b = std::atof(v.c_str());
        else if (k == "--BG") a.BG = std::atof(v.c_str());
        else if (k == "--QsmuRatio") a.QsmuRatio = std::atof(v.c_str());
        else if (k == "--roots") a.roots = std::atof(v.c_str());
        else if (k == "--rapidity") a.rapidity = std::atof(v.c_str());
        else if (k == "--xfactor") a.xfactor = std::atof(v.c_str());
        else if (k == "--rmax") a.rmax = std::atof(v.c_str());
        else if (k == "--sigmaNN") a.sigmaNN = std::atof(v.c_str());
        else if (k == "--fluct") a.fluct = std::atoi(v.c_str());
        else if (k == "--multiplicity") a.multiplicity = std::atoi(v.c_str());
        else if (k == "--pseudo") a.pseudo = std::atoi(v.c_str());
        else if (k == "--jacobian-m") a.jacobian_m = std::atof(v.c_str());
        else usage();
    }
    if (a.g2mu_file.empty() && a.mode != "ipsat") usage();
    if (a.size_output <= 0) a.size_output = a.N;
    if (a.L_output <= 0) a.L_output = a.L;
    return a;
}

void write_identity_vfile(const std::string &name, int N, double L) {
    std::ofstream f(name.c_str(), std::ios::out | std::ios::binary);
    int nc = 3;
    double a = L / N, y = 0.0;
    f.write((char *)&N, sizeof(int));
    f.write((char *)&nc, sizeof(int));
    f.write((char *)&L, sizeof(double));
    f.write((char *)&a, sizeof(double));
    f.write((char *)&y, sizeof(double));
    for (long r = 0; r < (long)N * N; r++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double v[2] = {i == j ? 1.0 : 0.0, 0.0};
                f.write((char *)v, sizeof(v));
            }
}

void dump_matrices(const std::string &name, Lattice &lat, int N,
                   Matrix &(Cell::*get)() const) {
    std::vector<double> buf((size_t)N * N * 18);
    for (int pos = 0; pos < N * N; pos++) {
        Matrix &M = (lat.cells[pos]->*get)();
        for (int k = 0; k < 9; k++) {
            buf[(size_t)pos * 18 + 2 * k] = M.getRe(k);
            buf[(size_t)pos * 18 + 2 * k + 1] = M.getIm(k);
        }
    }
    std::ofstream f(name.c_str(), std::ios::out | std::ios::binary);
    f.write((char *)buf.data(), buf.size() * sizeof(double));
}

void dump_observables(const std::string &name, Lattice &lat, int N) {
    std::vector<double> buf((size_t)N * N * 25);
    for (int pos = 0; pos < N * N; pos++) {
        Cell *c = lat.cells[pos];
        double v[25] = {c->getEpsilon(),  c->getutau(),     c->getux(),
                        c->getuy(),       c->getueta(),     c->getTtautau(),
                        c->getTxx(),      c->getTyy(),      c->getTetaeta(),
                        c->getTtaux(),    c->getTtauy(),    c->getTtaueta(),
                        c->getTxy(),      c->getTxeta(),    c->getTyeta(),
                        c->getpitautau(), c->getpixx(),     c->getpiyy(),
                        c->getpietaeta(), c->getpitaux(),   c->getpitauy(),
                        c->getpitaueta(), c->getpixy(),     c->getpixeta(),
                        c->getpiyeta()};
        std::memcpy(&buf[(size_t)pos * 25], v, sizeof(v));
    }
    std::ofstream f(name.c_str(), std::ios::out | std::ios::binary);
    f.write((char *)buf.data(), buf.size() * sizeof(double));
}

void dump_state(const std::string &prefix, Lattice &lat, int N) {
    dump_matrices(prefix + "_Ux.bin", lat, N, &Cell::getUx);
    dump_matrices(prefix + "_Uy.bin", lat, N, &Cell::getUy);
    dump_matrices(prefix + "_E1.bin", lat, N, &Cell::getE1);
    dump_matrices(prefix + "_E2.bin", lat, N, &Cell::getE2);
    dump_matrices(prefix + "_phi.bin", lat, N, &Cell::getphi);
    dump_matrices(prefix + "_pi.bin", lat, N, &Cell::getpi);
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
        .count();
}

}  // namespace

void write_doubles(const std::string &name, const std::vector<double> &v) {
    std::ofstream f(name.c_str(), std::ios::out | std::ios::binary);
    f.write((const char *)v.data(), v.size() * sizeof(double));
}

// IP-Sat maps through Init::readNuclearQs and Init::setColorChargeDensity
// (Init.cpp:441-480, 753-1676) for given nucleon positions; dumps T_A, T_B,
// g2mu2A, g2mu2B per cell and the event figures.
int run_ipsat(const Args &A) {
    const int N = A.N;
    std::vector<double> raw;
    {
        std::ifstream f(A.nucleons.c_str(), std::ios::in | std::ios::binary);
        double hdr[2];
        f.read((char *)hdr, sizeof(hdr));
        if (!f) {
            std::cerr << "cannot read " << A.nucleons << "\n";
            return 2;
        }
        raw.resize(2 * (size_t)(hdr[0] + hdr[1]) + 2);
        raw[0] = hdr[0];
        raw[1] = hdr[1];
        f.read((char *)(raw.data() + 2), (raw.size() - 2) * sizeof(double));
        if (!f) {
            std::cerr << "short nucleon file\n";
            return 2;
        }
    }
    const int nA = (int)raw[0], nB = (int)raw[1];
    // the table is opened after the chdir below: resolve it first
    char resolved[4096];
    const std::string table =
        realpath(A.table.c_str(), resolved) ? std::string(resolved) : A.table;
    mkdir(A.out.c_str(), 0755);
    if (chdir(A.out.c_str()) != 0) return 2;
    Parameters param;
    param.setSize(N);
    param.setL(A.L);
    param.setNc(3);
    param.setg(A.g);
    param.setEventId(0);
    param.setUseNucleus(1);
    param.setb(A.b);
    param.setBG(A.BG);
    param.setQsmuRatio(A.QsmuRatio);
    param.setRoots(A.roots);
    param.setRapidity(A.rapidity);
    param.setUsePseudoRapidity(0);
    param.setxFromThisFactorTimesQs(A.xfactor);
    param.setRmax(A.rmax);
    param.setSigmaNN(A.sigmaNN);
    param.setUseFluctuatingx(A.fluct);
    param.setProtonAnisotropy(0.0);
    param.setUseConstituentQuarkProton(0);
    param.setSmearQs(0);
    param.setSmearingWidth(0.0);
    param.setAverageOverNuclei(1);
    param.setRotateReactionPlane(0);
    param.setUseSmoothNucleus(0);
    param.setGaussianWounding(0);
    param.setUseFixedNpart(0);
    param.setMinimumQs2ST(0.0);
    param.setRunningCoupling(0);
    param.setNucleusQsTableFileName(table);
    int nn[2] = {N, N};
    Init init(nn);
    init.readNuclearQs(&param);
    for (int k = 0; k < nA + nB; k++) {
        ReturnValue r;
        r.x = raw[2 + 2 * k];
        r.y = raw[2 + 2 * k + 1];
        r.z = 0.0;
        r.phi = 0.0;
        r.collided = 0;
        r.proton = true;
        (k < nA ? init.nucleusA_ : init.nucleusB_).push_back(r);
    }
    Lattice lat(&param, 3, N);
    Random random;
    random.init_genrand64(A.seed);
    Glauber glauber;
    glauber.currentA1 = nA;
    glauber.currentA2 = nB;
    init.setColorChargeDensity(&lat, &param, &random, &glauber);
    std::vector<double> out(4 * (size_t)N * N);
    for (int pos = 0; pos < N * N; pos++) {
        out[pos] = lat.cells[pos]->getTpA();
        out[(size_t)N * N + pos] = lat.cells[pos]->getTpB();
        out[2 * (size_t)N * N + pos] = lat.cells[pos]->getg2mu2A();
        out[3 * (size_t)N * N + pos] = lat.cells[pos]->getg2mu2B();
    }
    write_doubles("ipsat.bin", out);
    long ncoll = 0;
    {
        std::ifstream f("NcollList0.dat");
        std::string line;
        while (std::getline(f, line))
            if (!line.empty()) ncoll++;
    }
    std::ofstream js("harness.json");
    js.precision(17);
    js << "{\"N\": " << N << ", \"mode\": \"ipsat\", \"Npart\": " << param.getNpart()
       << ", \"Ncoll\": " << ncoll << ", \"Tpp\": " << param.getTpp()
       << ", \"average_Qs\": " << param.getAverageQs()
       << ", \"average_Qs_avg\": " << param.getAverageQsAvg()
       << ", \"average_Qs_min\": " << param.getAverageQsmin() << "}\n";
    return 0;
}

int main(int argc, char **argv) {
    Args A = parse(argc, argv);
    if (A.mode == "ipsat") return run_ipsat(A);
    const int N = A.N;

    std::vector<double> g2mu((size_t)2 * N * N);
    {
        std::ifstream f(A.g2mu_file.c_str(), std::ios::in | std::ios::binary);
        f.read((char *)g2mu.data(), g2mu.size() * sizeof(double));
        if (!f) {
            std::cerr << "cannot read " << 2 * N * N << " doubles from "
                      << A.g2mu_file << "\n";
            return 2;
        }
    }
    mkdir(A.out.c_str(), 0755);
    if (chdir(A.out.c_str()) != 0) {
        std::cerr << "cannot chdir to " << A.out << "\n";
        return 2;
    }

    Parameters param;
    param.setSize(N);
    param.setL(A.L);
    param.setNc(3);
    param.setNy(A.Ny);
    param.setg(A.g);
    param.setm(A.m);
    param.setUVdamp(A.uvdamp);
    param.setSeed(0);  // only names the V files: V-0 and V-1
    param.setMPIRank(0);
    param.setMPISize(1);
    param.setEventId(0);
    param.setUseNucleus(0);
    param.setbmin(0.0);
    param.setbmax(0.0);
    param.setb(0.0);
    param.setLinearb(0);
    param.setUseFixedNpart(0);
    param.setlightNucleusOption(0);
    param.setRapidity(0.0);
    param.setWriteInitialWilsonLines(2);
    param.setReadInitialWilsonLines(2);
    param.setMaxtime(A.maxtime);
    param.setInverseQsForMaxTime(0);
    const double a = A.L / N;
    if (A.dtau > 0) {
        param.setdtau(A.dtau);
    } else {
        int iTimeSteps = static_cast<int>(10 * A.maxtime / a) + 1;
        param.setdtau(A.maxtime / (iTimeSteps * a));
    }
    param.setComputeGluonMultiplicity(A.multiplicity);
    if (A.multiplicity) {
        param.setUsePseudoRapidity(A.pseudo);
        param.setRapidity(A.rapidity);
        param.setJacobianm(A.jacobian_m);
        param.setRoots(A.roots);
        param.setRunWithkt(0);
        param.setRandomSeed(A.seed);
        param.setb(A.b);
        std::cout.precision(17);
    }
    param.setWriteOutputs(A.write_outputs);
    param.setSizeOutput(A.size_output);
    param.setEtaSizeOutput(1);
    param.setDetaOutput(0.0);
    param.setLOutput(A.L_output);
    param.setRunningCoupling(0);
    param.setRunWithQs(2);
    param.setRunWithLocalQs(0);
    param.setRunWithThisFactorTimesQs(0.5);
    param.setMuZero(0.3);
    param.setc(0.2);
    param.setalphas(0.3);
    param.setQsmuRatio(0.8);
    param.setQsmuRatioB(0.8);
    param.setAverageQs(1.0);
    param.setAverageQsAvg(1.0);
    param.setAverageQsmin(1.0);
    param.setNpart(2);
    param.setTpp(0.0);
    param.setArea(0.0);
    param.setSuccess(0);

    int nn[2] = {N, N};
    Init init(nn);
    Group group(3);
    Glauber glauber;
    glauber.currentA1 = 197;  // no light-nucleus configuration file is read
    glauber.currentA2 = 197;
    Evolution evolution(nn);
    Lattice lat(&param, 3, N);
    Random bootRandom;
    bootRandom.init_genrand64(A.seed + 7919ULL);

    // (2) bootstrap the Init object
    write_identity_vfile("V-0", N, A.L);
    write_identity_vfile("V-1", N, A.L);
    init.init(&lat, &group, &param, &bootRandom, &glauber, 2);

    // (3) colour charges and Wilson lines
    Matrix one(3, 1.);
    for (int pos = 0; pos < N * N; pos++) {
        lat.cells[pos]->setg2mu2A(g2mu[pos]);
        lat.cells[pos]->setg2mu2B(g2mu[(size_t)N * N + pos]);
        lat.cells[pos]->setU(one);
        lat.cells[pos]->setU2(one);
    }
    Random rhoRandom;
    rhoRandom.init_genrand64(A.seed);
    auto t0 = std::chrono::steady_clock::now();
    init.setV(&lat, &param, &rhoRandom);
    const double t_setv = seconds_since(t0);
    if (A.dumps) {
    dump_matrices("VA.bin", lat, N, &Cell::getU);
    dump_matrices("VB.bin", lat, N, &Cell::getU2);
    {
        // the unit normals setV drew, in its order (nucleus, k, pos, colour):
        // a second Random with the same seed replays the same stream
        Random replay;
        replay.init_genrand64(A.seed);
        const size_t cnt = (size_t)A.Ny * N * N * 8;
        std::vector<double> xi(cnt);
        for (int nuc = 0; nuc < 2; nuc++) {
            for (size_t k = 0; k < cnt; k++) xi[k] = replay.Gauss();
            std::ofstream f(nuc ? "xiB.bin" : "xiA.bin",
                            std::ios::out | std::ios::binary);
            f.write((char *)xi.data(), cnt * sizeof(double));
        }
    }
    }

    // (4) tau = 0 fields; count the restart draws made on bootRandom
    Random probe;
    probe.init_genrand64(A.seed + 7919ULL);
    probe.genrand64_real1();  // Init::init draws xb once (Init.cpp:2321)
    probe.genrand64_real1();  // ... on each of the two calls
    t0 = std::chrono::steady_clock::now();
    init.init(&lat, &group, &param, &bootRandom, &glauber, 2);
    const double t_tau0 = seconds_since(t0);
    // extra 64-bit draws consumed by Newton restarts (Init.cpp:3446-3468)
    long restart_draws = -1;
    {
        const unsigned long long next = bootRandom.genrand64_int64();
        for (long k = 0; k < 1000000; k++) {
            if (probe.genrand64_int64() == next) {
                restart_draws = k;
                break;
            }
        }
    }
    if (A.dumps) dump_state("tau0", lat, N);

    double t_evo = 0.0, t_ecc = 0.0;
    int itmax = static_cast<int>(param.getMaxtime() / (a * param.getdtau()) + 0.1);
    if (A.mode == "steps") {
        // (5b) leapfrog only, K full steps after the tau=0 half step
        const double dtau = param.getdtau();
        t0 = std::chrono::steady_clock::now();
        evolution.evolvePhi(&lat, &param, dtau, 0.);
        evolution.evolveU(&lat, &param, dtau, 0.);
        for (int it = 1; it <= A.steps; it++) {
            evolution.evolvePi(&lat, &param, dtau, it * dtau);
            evolution.evolveE(&lat, &param, dtau, it * dtau);
            evolution.evolvePhi(&lat, &param, dtau, it * dtau);
            evolution.evolveU(&lat, &param, dtau, it * dtau);
        }
        t_evo = seconds_since(t0);
        if (A.dumps) dump_state("steps", lat, N);
        itmax = A.steps;
    } else if (A.mode == "full") {
        // (5a) the reference schedule, then (6) eccentricity
        t0 = std::chrono::steady_clock::now();
        evolution.run(&lat, &group, &param);
        t_evo = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        evolution.eccentricity(&lat, &param, itmax, 0.0, 0);
        t_ecc = seconds_since(t0);
        if (A.dumps) {
            dump_observables("obs.bin", lat, N);
            dump_state("final", lat, N);
        }
    }

    std::ofstream js("harness.json");
    js.precision(17);
    js << "{\"N\": " << N << ", \"L\": " << A.L << ", \"Ny\": " << A.Ny
       << ", \"a\": " << a << ", \"dtau\": " << param.getdtau()
       << ", \"itmax\": " << itmax << ", \"mode\": \"" << A.mode << "\""
       << ", \"eccentricity2\": "
       << (A.mode == "full" ? param.getEccentricity2() : 0.0)
       << ", \"newton_restart_draws\": " << restart_draws
       << ", \"t_setV\": " << t_setv << ", \"t_tau0\": " << t_tau0
       << ", \"t_evolution\": " << t_evo << ", \"t_eccentricity\": " << t_ecc
       << "}\n";
    return 0;
}
