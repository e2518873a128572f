// Checks the device number formatter (ipglasma_b200/csrc/fmt.cuh, compiled
// here as plain C++) against std::to_chars with precision 6, the format of
// the host writers: random doubles over the whole supported range, ties,
// decade and rounding boundaries, integers. Prints "checked <n> mismatches
// <k> unsupported <u>" and exits non-zero on any mismatch.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>

#include "../../ipglasma_b200/csrc/fmt.cuh"

static long checked = 0, bad = 0, unsupported = 0;

static void check(double v) {
    char a[64], b[64];
    const int n = ipg::fmt::g6(v, a);
    const bool in_range = v == 0 || (std::fabs(v) >= 1e-130 && std::fabs(v) < 1e6);
    if (n < 0) {
        if (in_range) {
            if (bad++ < 20) std::printf("unsupported in range: %.17g\n", v);
        } else {
            unsupported++;
        }
        return;
    }
    const char *e = std::to_chars(b, b + sizeof(b), v, std::chars_format::general, 6).ptr;
    checked++;
    if ((size_t)n != (size_t)(e - b) || std::memcmp(a, b, n) != 0) {
        if (bad++ < 20)
            std::printf("mismatch %.17g: got %.*s want %.*s\n", v, n, a, (int)(e - b), b);
    }
}

static void check_int(int v) {
    char a[32], b[32];
    const int n = ipg::fmt::integer(v, a);
    const char *e = std::to_chars(b, b + sizeof(b), v).ptr;
    checked++;
    if ((size_t)n != (size_t)(e - b) || std::memcmp(a, b, n) != 0) {
        if (bad++ < 20) std::printf("int mismatch %d\n", v);
    }
}

int main(int argc, char **argv) {
    const long count = argc > 1 ? std::atol(argv[1]) : 2000000;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> ue(-131.0, 6.5), uu(0.0, 1.0);
    for (long i = 0; i < count; i++) {
        // log-uniform magnitudes over and beyond the range, both signs
        double v = std::pow(10.0, ue(rng)) * (rng() & 1 ? -1 : 1);
        check(v);
        // neighbours of a 6-digit rounding boundary (d.ddddd5 x 10^E)
        const int E = (int)(rng() % 136) - 130;
        const double mant = 100000 + (double)(rng() % 900000) + 0.5;
        double w = mant * std::pow(10.0, E - 5);
        check(w);
        check(std::nextafter(w, 0.0));
        check(std::nextafter(w, 1e300));
        // random bit patterns
        uint64_t bits = rng();
        double r;
        std::memcpy(&r, &bits, 8);
        check(r);
    }
    // exact ties at the sixth digit: N + 1/2 for 6-digit N
    for (long N = 100000; N < 1000000; N += 7) check(N + 0.5);
    // powers of ten and their neighbours, decade edges, special values
    for (int E = -135; E <= 7; E++) {
        const double p = std::pow(10.0, E);
        for (double f : {1.0, 9.999995, 9.9999949999, 9.99999500001, 1.000005, 5.0, 0.5}) {
            const double v = f * p;
            check(v);
            check(std::nextafter(v, 0.0));
            check(std::nextafter(v, 1e300));
            check(-v);
        }
    }
    for (double v : {0.0, -0.0, 1.0, -1.0, 1e-16, 5e-17, 0.1973269718, 1e-4, 9.99999e-5,
                     0.000099999949999, 999999.4, 999999.5, 999999.6, 123456.5, 123457.5})
        check(v);
    check(std::nan(""));
    check(INFINITY);
    check(-INFINITY);
    for (int v : {0, 1, -1, 9, 10, 99, 100, 511, 512, 2147483647, -2147483647 - 1}) check_int(v);
    for (int i = 0; i < 100000; i++) check_int((int)rng());
    std::printf("checked %ld mismatches %ld unsupported %ld\n", checked, bad, unsupported);
    return bad ? 1 : 0;
}
