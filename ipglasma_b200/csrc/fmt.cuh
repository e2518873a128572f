// Number formatting of an ostream with default flags (printf "%.6g" in the C
// locale, the format the reference's output files use, MyEigen.cpp:380-1045)
// for device code, and compiled as plain C++ for its tests.
//
// fmt_g6 rounds exactly: v = m 2^q (m < 2^53) is scaled by 10^k with a
// 384-bit integer m 5^k 2^(k+q), so the six significant digits are the
// correctly rounded ones (ties to even, as printf and std::to_chars round the
// exact binary value). The range is |v| in [1e-130, 1e6) and zero; other
// values (and NaN, infinities) return -1 so that the caller formats them on
// the host.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define IPG_FMT_HD __host__ __device__ __forceinline__
#else
#define IPG_FMT_HD inline
#endif

namespace ipg {
namespace fmt {

// little-endian 384-bit unsigned integer
struct Big {
    uint64_t w[6];
};

// b *= f over its nl low limbs (nl grows by the carry out)
IPG_FMT_HD void mul_small(Big &b, int &nl, uint64_t f) {
    uint64_t carry = 0;
    for (int i = 0; i < nl; i++) {
#ifdef __CUDA_ARCH__
        const uint64_t lo = b.w[i] * f, hi = __umul64hi(b.w[i], f);
#else
        const unsigned __int128 p = (unsigned __int128)b.w[i] * f;
        const uint64_t lo = (uint64_t)p, hi = (uint64_t)(p >> 64);
#endif
        const uint64_t s = lo + carry;
        carry = hi + (s < lo ? 1 : 0);
        b.w[i] = s;
    }
    if (carry && nl < 6) b.w[nl++] = carry;
}

IPG_FMT_HD int clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

IPG_FMT_HD int bit_length(const Big &b, int nl) {
    for (int i = nl - 1; i >= 0; i--)
        if (b.w[i]) return 64 * i + 64 - clz64(b.w[i]);
    return 0;
}

IPG_FMT_HD int bit_at(const Big &b, int i) { return (int)((b.w[i >> 6] >> (i & 63)) & 1u); }

// any of bits [0, n) set
IPG_FMT_HD bool low_bits_set(const Big &b, int n) {
    for (int i = 0; i < 6 && n > 0; i++, n -= 64) {
        const uint64_t mask = n >= 64 ? ~0ull : ((1ull << n) - 1);
        if (b.w[i] & mask) return true;
    }
    return false;
}

// bits [r, r + 64) of b
IPG_FMT_HD uint64_t bits_from(const Big &b, int r) {
    const int i = r >> 6, sh = r & 63;
    uint64_t lo = i < 6 ? b.w[i] >> sh : 0;
    if (sh && i + 1 < 6) lo |= b.w[i + 1] << (64 - sh);
    return lo;
}

IPG_FMT_HD double abs_d(double v) { return v < 0 ? -v : v; }

// floor(log10(v)) for v = m 2^q with the binary exponent eb = q + 52
// (m in [2^52, 2^53)): floor(eb log10 2) is within one of it; the caller
// corrects it exactly
IPG_FMT_HD int decade(int eb) {
    // 78913 / 2^18 = 0.30102920... (log10 2 = 0.30102999...), exact floor for |eb| < 1700
    return (eb * 78913) >> 18;
}

// 5^k for k in [0, 27]
IPG_FMT_HD uint64_t pow5(int k) {
    uint64_t r = 1, b = 5;
    while (k) {
        if (k & 1) r *= b;
        b *= b;
        k >>= 1;
    }
    return r;
}

// text of v as printf "%.6g" into p (at most 13 characters); returns the
// length, or -1 when v is outside the supported range
IPG_FMT_HD int g6(double v, char *p) {
    uint64_t bits;
    {
        union {
            double d;
            uint64_t u;
        } cvt;
        cvt.d = v;
        bits = cvt.u;
    }
    int n = 0;
    if (bits >> 63) p[n++] = '-';
    const uint64_t mbits = bits & ((1ull << 52) - 1);
    const int ebits = (int)((bits >> 52) & 0x7ff);
    if (ebits == 0x7ff) return -1;
    if (ebits == 0 && mbits == 0) {
        p[n++] = '0';
        return n;
    }
    const double av = abs_d(v);
    if (!(av >= 1e-130 && av < 1e6)) return -1;
    const uint64_t m = mbits | (1ull << 52);  // normal numbers only in this range
    const int q = ebits - 1075;
    int E = decade(q + 52);
    uint64_t N = 0;
    for (int tries = 0;; tries++) {
        const int k = 5 - E;  // v 10^k = m 5^k 2^(k+q) should lie in [1e5, 1e6)
        if (k < 0 || k > 140 || tries > 3) return -1;
        Big P = {{m, 0, 0, 0, 0, 0}};
        int nl = 1;
        int k5 = k;
        while (k5 >= 27) {
            mul_small(P, nl, 7450580596923828125ull);  // 5^27
            k5 -= 27;
        }
        mul_small(P, nl, pow5(k5));
        const int s = k + q;
        const int len = bit_length(P, nl);
        uint64_t F;
        bool up = false;
        if (s >= 0) {
            if (len + s > 40) {  // >= 2^40 > 1e6
                E++;
                continue;
            }
            F = P.w[0] << s;
        } else {
            const int r = -s;
            if (len - r > 40) {
                E++;
                continue;
            }
            F = len > r ? bits_from(P, r) : 0;
            if (r <= len) {
                const bool half = bit_at(P, r - 1) != 0;
                up = half && (low_bits_set(P, r - 1) || (F & 1));
            }
        }
        if (F >= 1000000) {
            E++;
            continue;
        }
        if (F < 100000) {
            E--;
            continue;
        }
        N = F + (up ? 1 : 0);
        if (N == 1000000) {
            N = 100000;
            E++;
        }
        break;
    }
    char d[6];
    for (int i = 5; i >= 0; i--) {
        d[i] = (char)('0' + (int)(N % 10));
        N /= 10;
    }
    int last = 5;
    if (E < -4 || E >= 6) {
        while (last > 0 && d[last] == '0') last--;
        p[n++] = d[0];
        if (last > 0) {
            p[n++] = '.';
            for (int i = 1; i <= last; i++) p[n++] = d[i];
        }
        p[n++] = 'e';
        p[n++] = E < 0 ? '-' : '+';
        int ae = E < 0 ? -E : E;
        if (ae >= 100) {
            p[n++] = (char)('0' + ae / 100);
            ae %= 100;
        }
        p[n++] = (char)('0' + ae / 10);
        p[n++] = (char)('0' + ae % 10);
    } else if (E >= 0) {
        while (last > E && d[last] == '0') last--;
        for (int i = 0; i <= E; i++) p[n++] = d[i];
        if (last > E) {
            p[n++] = '.';
            for (int i = E + 1; i <= last; i++) p[n++] = d[i];
        }
    } else {
        while (last > 0 && d[last] == '0') last--;
        p[n++] = '0';
        p[n++] = '.';
        for (int i = 0; i < -E - 1; i++) p[n++] = '0';
        for (int i = 0; i <= last; i++) p[n++] = d[i];
    }
    return n;
}

// decimal text of an int (at most 11 characters)
IPG_FMT_HD int integer(int v, char *p) {
    int n = 0;
    unsigned u = (unsigned)v;
    if (v < 0) {
        p[n++] = '-';
        u = 0u - u;
    }
    char t[10];
    int k = 0;
    do {
        t[k++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    while (k) p[n++] = t[--k];
    return n;
}

}  // namespace fmt
}  // namespace ipg
