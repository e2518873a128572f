// Two FP32 lanes in one 64-bit register pair, computed with the sm_100 packed
// instructions (one FFMA2 / FADD2 / FMUL2 does two lanes): P2 is the scalar
// type that lets the templated SU(3) helpers (su3.cuh) run the x-direction
// and the y-direction work of a lattice site in one thread.
//
// a * b yields a pending product, so that `c += a * b` and `c -= a * b` (the
// form of every accumulation in su3.cuh) become one fused multiply-add of
// both lanes instead of a multiply and an add.
#pragma once

#include <cuda_runtime.h>

namespace ipg {

struct P2 {
    float2 v;
    __device__ __forceinline__ P2() = default;
    __device__ __forceinline__ P2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ P2(int s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ P2(double s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ P2(float2 x) : v(x) {}
    __device__ __forceinline__ P2(float x, float y) : v(make_float2(x, y)) {}
    // found by argument-dependent lookup only, so it does not hide ::sqrt
    friend __device__ __forceinline__ P2 sqrt(P2 a) { return P2(sqrtf(a.v.x), sqrtf(a.v.y)); }
};

struct P2Prod {
    float2 a, b;
    __device__ __forceinline__ operator P2() const { return P2(__fmul2_rn(a, b)); }
};

__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }

__device__ __forceinline__ P2Prod operator*(P2 a, P2 b) { return {a.v, b.v}; }
__device__ __forceinline__ P2Prod operator*(P2Prod p, P2 b) {
    return {__fmul2_rn(p.a, p.b), b.v};
}
__device__ __forceinline__ P2Prod operator*(P2 a, P2Prod p) {
    return {a.v, __fmul2_rn(p.a, p.b)};
}
__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return P2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ P2 operator-(P2 a, P2 b) { return P2(__fadd2_rn(a.v, neg2(b.v))); }
__device__ __forceinline__ P2 operator-(P2 a) { return P2(neg2(a.v)); }
__device__ __forceinline__ P2 operator+(P2 c, P2Prod p) { return P2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ P2 operator+(P2Prod p, P2 c) { return P2(__ffma2_rn(p.a, p.b, c.v)); }
__device__ __forceinline__ P2 operator-(P2 c, P2Prod p) {
    return P2(__ffma2_rn(neg2(p.a), p.b, c.v));
}
__device__ __forceinline__ P2 operator-(P2Prod p, P2 c) {
    return P2(__ffma2_rn(p.a, p.b, neg2(c.v)));
}
__device__ __forceinline__ P2 operator+(P2Prod p, P2Prod q) {
    return P2(__ffma2_rn(p.a, p.b, __fmul2_rn(q.a, q.b)));
}
__device__ __forceinline__ P2 operator-(P2Prod p, P2Prod q) {
    return P2(__ffma2_rn(p.a, p.b, __fmul2_rn(neg2(q.a), q.b)));
}
__device__ __forceinline__ P2 operator-(P2Prod p) { return P2(__fmul2_rn(neg2(p.a), p.b)); }
__device__ __forceinline__ P2 &operator+=(P2 &c, P2 b) { return c = c + b; }
__device__ __forceinline__ P2 &operator-=(P2 &c, P2 b) { return c = c - b; }
__device__ __forceinline__ P2 &operator+=(P2 &c, P2Prod p) { return c = c + p; }
__device__ __forceinline__ P2 &operator-=(P2 &c, P2Prod p) { return c = c - p; }
__device__ __forceinline__ P2 &operator*=(P2 &c, P2 b) { return c = P2(__fmul2_rn(c.v, b.v)); }
__device__ __forceinline__ P2 operator/(P2 a, P2 b) {
    return P2(a.v.x / b.v.x, a.v.y / b.v.y);
}
__device__ __forceinline__ P2 operator/(P2 a, P2Prod b) { return a / P2(b); }
__device__ __forceinline__ P2 operator/(P2Prod a, P2 b) { return P2(a) / b; }

__device__ __forceinline__ float lane_x(P2 a) { return a.v.x; }
__device__ __forceinline__ float lane_y(P2 a) { return a.v.y; }

}  // namespace ipg
