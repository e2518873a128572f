// Counter-based Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) and Box-Muller
// normals. Used for the device-side colour-charge noise and the Newton
// restart draws: every (nucleus, sheet, site, colour) gets its own counter,
// so draws are independent of the launch shape.
#pragma once

#include <cstdint>

namespace ipg {

struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ uint32_t mulhilo(uint32_t a, uint32_t b,
                                                     uint32_t *hi) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 ctr, uint32_t k0,
                                                     uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, hi1;
        uint32_t lo0 = mulhilo(M0, ctr.x, &hi0);
        uint32_t lo1 = mulhilo(M1, ctr.z, &hi1);
        ctr = {hi1 ^ ctr.y ^ k0, lo1, hi0 ^ ctr.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return ctr;
}

// uniform in (0, 1]
__host__ __device__ __forceinline__ double u01(uint32_t a, uint32_t b) {
    uint64_t v = ((uint64_t)a << 21) ^ (uint64_t)b;  // 53 random bits
    v &= ((1ull << 53) - 1);
    return ((double)v + 1.0) * (1.0 / 9007199254740992.0);
}

// uniform in (0, 1] with 24 random bits
__host__ __device__ __forceinline__ float u01f(uint32_t a) {
    return ((float)(a >> 8) + 1.0f) * (1.0f / 16777216.0f);
}

// four standard normals from one counter (Box-Muller in single precision:
// the noise only has to be Gaussian, not reproducible to more than 24 bits)
__device__ __forceinline__ void normal4(U4 ctr, uint64_t key, double out[4]) {
    const U4 r = philox4x32_10(ctr, (uint32_t)key, (uint32_t)(key >> 32));
    const float rad1 = sqrtf(-2.0f * logf(u01f(r.x)));
    const float rad2 = sqrtf(-2.0f * logf(u01f(r.z)));
    float s1, c1, s2, c2;
    sincospif(2.0f * u01f(r.y), &s1, &c1);
    sincospif(2.0f * u01f(r.w), &s2, &c2);
    out[0] = rad1 * c1;
    out[1] = rad1 * s1;
    out[2] = rad2 * c2;
    out[3] = rad2 * s2;
}

// the Box-Muller pair of normal4 made from the words (a, b): (r.x, r.y) give
// out[0..1] of normal4, (r.z, r.w) give out[2..3], with the same operations
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, double out[2]) {
    const float rad = sqrtf(-2.0f * logf(u01f(a)));
    float s, c;
    sincospif(2.0f * u01f(b), &s, &c);
    out[0] = rad * c;
    out[1] = rad * s;
}

// one Box-Muller pair of normal4 for the same counter: half 0 gives out[0..1],
// half 1 gives out[2..3], with the same values
__device__ __forceinline__ void normal2(U4 ctr, uint64_t key, int half, double out[2]) {
    const U4 r = philox4x32_10(ctr, (uint32_t)key, (uint32_t)(key >> 32));
    box_muller(half ? r.z : r.x, half ? r.w : r.y, out);
}

}  // namespace ipg
