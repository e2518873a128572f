// Boost-invariant leapfrog step, fused into one stencil kernel per step.
//
// One launch performs, for every site, what the reference does in four
// separate OpenMP sweeps (Evolution.cpp:35-293):
//   evolvePi   pi  += dtau/tau * (sum_{+-x,+-y} U phi U^dag - 4 phi)   (117-178)
//   evolveE    E_i += i tau dtau/(2g^2) TL(staples) + i dtau/tau [phi~_i, phi],
//              then E_i is made traceless                              (180-293)
//   evolvePhi  phi += (tau + dtau/2) dtau pi                            (90-115)
//   evolveU    U_i  = (1 + X + X^2/2) U_i,  X = i g^2 dtau/(tau+dtau/2) E_i (35-88)
// pi and E are read and written only at their own site, so they are updated
// in place; U and phi are read at neighbours, so they are ping-ponged
// between two buffers. Neighbours are clamped (Lattice.cpp:19-28,
// Evolution.cpp:207-210).
//
// Per site the kernel moves the state once: read U(2x18) E(2x8) phi(9) pi(9)
// and write the same, 70 reals each way; neighbour reads hit L1/L2.
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "fields.cuh"
#include "ipg_internal.h"
#include "pair2.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace ipg {

// i * (P Q - (P Q)^dag) without forming P Q.
// U_new = (1 + X + X^2/2) U with X = i c E, E Hermitian:
// (1 + X + X^2/2) = (1 - c^2 E^2 / 2) + i c E.
template <typename T>
__device__ __forceinline__ M3<T> taylor2_update(const H3<T> &e, T c,
                                                const M3<T> &u) {
    M3<T> em = from_h(e);
    M3<T> e2 = mul_g<false, false, true, true>(em, em);
    M3<T> t;
    const T h = T(-0.5) * c * c;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        // real part: delta - c^2/2 (E^2)  ;  imaginary part: c E
        t.m[k].r = h * e2.m[k].r - c * em.m[k].i;
        t.m[k].i = h * e2.m[k].i + c * em.m[k].r;
    }
    t.m[0].r += T(1);
    t.m[4].r += T(1);
    t.m[8].r += T(1);
    return mul(t, u);
}

// One site in full-matrix storage (the FP64 plain form): loads through `ld`,
// writes the new pi and E through it and returns the new links and phi when
// cf.do_pu is set. The site's own links and phi are loaded again at each use
// rather than held (from a shared-memory tile that is cheaper than keeping
// 90 registers live across the site, which spilled).
// The staple sums of E1 and E2 at one site, traceless (Evolution.cpp:228-275).
template <typename T, class Ld>
__device__ __forceinline__ void full_staples(const Ld &ld, H3<T> &t1, H3<T> &t2) {
        // plaquette U12 = Ux Uy(x+1) Ux(y+1)^dag Uy^dag  (Evolution.cpp:228-232)
        H3<T> h12;
        {
            M3<T> a = mul(ld.template link<kLx, 0, 0>(), ld.template link<kLy, 1, 0>());
            M3<T> b = mul(ld.template link<kLy, 0, 0>(), ld.template link<kLx, 0, 1>());
            M3<T> u12 = mul_nd(a, b);
            h12 = i_antiherm(u12);
        }
        // E1 staple sum: U12 + U1m2 - h.c.  (234-257)
        t1 = h12;
        {
            M3<T> p = mul_nd(ld.template link<kLx, 0, 0>(), ld.template link<kLy, 1, -1>());
            M3<T> q = mul_dn(ld.template link<kLx, 0, -1>(), ld.template link<kLy, 0, -1>());
            h_add(t1, i_antiherm_mul(p, q));
        }
        // E2 staple sum: U12^dag + U2m1 - h.c.  (240-244, 266-275)
        {
            M3<T> p = mul_nd(ld.template link<kLy, 0, 0>(), ld.template link<kLx, -1, 1>());
            M3<T> q = mul_dn(ld.template link<kLy, -1, 0>(), ld.template link<kLx, -1, 0>());
            t2 = i_antiherm_mul(p, q);
            h_axpy(t2, T(-1), h12);
        }
        h_traceless(t1);
        h_traceless(t2);
}

template <typename T, bool REUNIT, class Ld>
__device__ __forceinline__ void leapfrog_full_core(const Ld &ld, const StepCoef<T> &cf,
                                                   M3<T> &nx, M3<T> &ny, H3<T> &phin) {
    if (cf.do_pe) {
        H3<T> t1, t2;
        full_staples<T>(ld, t1, t2);

        H3<T> pi = ld.pi();
        H3<T> e1 = ld.e1();
        H3<T> e2 = ld.e2();
        const T cst = cf.tau * cf.dt_pe / (T(2) * cf.g * cf.g);
        const T cdt = cf.dt_pe / cf.tau;
        h_axpy(e1, cst, t1);
        h_axpy(e2, cst, t2);

        // parallel transports of phi (evolvePi 139-157, evolveE 221-223, 278-279)
        H3<T> br;
        {
            H3<T> phx = conj_h(ld.template link<kLx, 0, 0>(), ld.template phi<1, 0>());
            h_axpy(e1, cdt, i_commutator(phx, ld.template phi<0, 0>()));
            br = phx;
        }
        {
            H3<T> phy = conj_h(ld.template link<kLy, 0, 0>(), ld.template phi<0, 1>());
            h_axpy(e2, cdt, i_commutator(phy, ld.template phi<0, 0>()));
            h_add(br, phy);
        }
        h_add(br, conj_h_dag(ld.template link<kLx, -1, 0>(), ld.template phi<-1, 0>()));
        h_add(br, conj_h_dag(ld.template link<kLy, 0, -1>(), ld.template phi<0, -1>()));
        h_axpy(br, T(-4), ld.template phi<0, 0>());
        h_axpy(pi, cdt, br);
        h_traceless(e1);
        h_traceless(e2);
        ld.put_pi(pi);
        ld.put_e(e1, e2);

        if (cf.do_pu) {
            phin = ld.template phi<0, 0>();
            h_axpy(phin, (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu, pi);
            const T c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
            nx = taylor2_update(e1, c, ld.template link<kLx, 0, 0>());
            if (REUNIT) reunitarize(nx);
            ny = taylor2_update(e2, c, ld.template link<kLy, 0, 0>());
            if (REUNIT) reunitarize(ny);
        }
    } else if (cf.do_pu) {
        // phi and U only (the tau = 0 half step, Evolution.cpp:393-394)
        phin = ld.template phi<0, 0>();
        const H3<T> pi = ld.pi();
        h_axpy(phin, (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu, pi);
        const T c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
        nx = taylor2_update(ld.e1(), c, ld.template link<kLx, 0, 0>());
        if (REUNIT) reunitarize(nx);
        ny = taylor2_update(ld.e2(), c, ld.template link<kLy, 0, 0>());
        if (REUNIT) reunitarize(ny);
    }
}

// one site (ix, iy) from the global planes
template <typename T, bool REUNIT>
__device__ __forceinline__ void leapfrog_full_site(int N, int ix, int iy, const State<T> &s,
                                                   C<T> *ux_out, C<T> *uy_out, T *phi_out,
                                                   const StepCoef<T> &cf) {
    const FullLoadGlobal<T> ld(s, N, ix, iy);
    M3<T> nx, ny;
    H3<T> phin;
    leapfrog_full_core<T, REUNIT>(ld, cf, nx, ny, phin);
    if (cf.do_pu) {
        st_h(phi_out, ld.pos, ld.n, phin);
        st_m3(ux_out, ld.pos, ld.n, nx);
        st_m3(uy_out, ld.pos, ld.n, ny);
    }
}

// Time reversal of the E and pi half of a step: three thread roles per site
// (blockIdx.y: E1, E2, pi; inverse_se_role), three times the warps of one
// thread per site at two thirds of the registers
template <typename T>
__global__ void __launch_bounds__(128, 3)
    k_inv_se(int N, State<T> nxt, State<T> cur, StepCoef<double> cf) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (size_t)N * N) return;
    const int role = blockIdx.y;
    if (cf.do_pe) {
        inverse_se_role<T>(N, role, p, nxt, cur, (T)(cf.tau * cf.dt_pe / (2. * cf.g * cf.g)),
                           (T)(cf.dt_pe / cf.tau));
    } else if (role == 2) {
        st_h(cur.pi, p, (size_t)N * N, ld_h(nxt.pi, p, (size_t)N * N));
    } else {
        st_h8(role == 0 ? cur.e1 : cur.e2, p, (size_t)N * N,
              ld_h8(role == 0 ? nxt.e1 : nxt.e2, p, (size_t)N * N));
    }
}



template <typename T, bool REUNIT>
__global__ void __launch_bounds__(128)
    k_leapfrog(const EventGeom *__restrict__ ev, State<T> s, C<T> *ux_out,
               C<T> *uy_out, T *phi_out, StepCoef<T> cf) {
    const int N = ev->N;
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= N || iy >= N) return;
    leapfrog_full_site<T, REUNIT>(N, ix, iy, s, ux_out, uy_out, phi_out, cf);
}

// ===========================================================================
// FP32 bulk form: links stored as their deviation from the identity,
// W = U - 1. Every product of links is formed as
//   (1 + a)(1 + b) - 1 = a + b + ab,
// so plaquettes, staples and parallel transports keep FP32 *relative*
// precision on the small deviations that carry the physics; the identity
// part (which would swallow them in a plain FP32 3x3) cancels exactly in
// U - U^dag and in U phi U^dag - phi. The observables are evaluated in FP64
// from U = 1 + W. Links are reunitarised every step (Gram-Schmidt on the
// first two rows, third row = conj(row0 x row1), as Matrix::reu,
// Matrix.h:67-109), also in deviation form.
// ===========================================================================

// (1+a)(1+b) - 1 = (a + b) + ab, the product chained onto a + b
template <typename T>
__device__ __forceinline__ M3<T> dmul(const M3<T> &a, const M3<T> &b) {
    M3<T> z = a;
    add_to(z, b);
    return mul_acc<false, false>(a, b, z);
}
// (1+a)(1+b)^dag - 1
template <typename T>
__device__ __forceinline__ M3<T> dmul_nd(const M3<T> &a, const M3<T> &b) {
    M3<T> z = a;
    add_to(z, dagger(b));
    return mul_acc<false, true>(a, b, z);
}
// (1+a)^dag (1+b) - 1
template <typename T>
__device__ __forceinline__ M3<T> dmul_dn(const M3<T> &a, const M3<T> &b) {
    M3<T> z = dagger(a);
    add_to(z, b);
    return mul_acc<true, false>(a, b, z);
}

// connection part of (1+w) H (1+w)^dag, i.e. the transport minus H:
// X + X^dag + X w^dag with X = w H
template <typename T>
__device__ __forceinline__ H3<T> transport_dev(const M3<T> &w, const H3<T> &h) {
    const M3<T> x = mul_g<false, false, false, true>(w, from_h(h));
    const M3<T> y = mul_nd(x, w);
    H3<T> o;
    o.d0 = T(2) * x.m[0].r + y.m[0].r;
    o.d1 = T(2) * x.m[4].r + y.m[4].r;
    o.d2 = T(2) * x.m[8].r + y.m[8].r;
    o.o01 = {x.m[1].r + x.m[3].r + y.m[1].r, x.m[1].i - x.m[3].i + y.m[1].i};
    o.o02 = {x.m[2].r + x.m[6].r + y.m[2].r, x.m[2].i - x.m[6].i + y.m[2].i};
    o.o12 = {x.m[5].r + x.m[7].r + y.m[5].r, x.m[5].i - x.m[7].i + y.m[5].i};
    return o;
}
// connection part of (1+w)^dag H (1+w): X + X^dag + w^dag X with X = H w
template <typename T>
__device__ __forceinline__ H3<T> transport_dev_back(const M3<T> &w, const H3<T> &h) {
    const M3<T> x = mul_g<false, false, true, false>(from_h(h), w);
    const M3<T> y = mul_dn(w, x);
    H3<T> o;
    o.d0 = T(2) * x.m[0].r + y.m[0].r;
    o.d1 = T(2) * x.m[4].r + y.m[4].r;
    o.d2 = T(2) * x.m[8].r + y.m[8].r;
    o.o01 = {x.m[1].r + x.m[3].r + y.m[1].r, x.m[1].i - x.m[3].i + y.m[1].i};
    o.o02 = {x.m[2].r + x.m[6].r + y.m[2].r, x.m[2].i - x.m[6].i + y.m[2].i};
    o.o12 = {x.m[5].r + x.m[7].r + y.m[5].r, x.m[5].i - x.m[7].i + y.m[5].i};
    return o;
}

template <typename T>
__device__ __forceinline__ H3<T> h_diff(const H3<T> &a, const H3<T> &b) {
    H3<T> r;
    r.d0 = a.d0 - b.d0;
    r.d1 = a.d1 - b.d1;
    r.d2 = a.d2 - b.d2;
    r.o01 = {a.o01.r - b.o01.r, a.o01.i - b.o01.i};
    r.o02 = {a.o02.r - b.o02.r, a.o02.i - b.o02.i};
    r.o12 = {a.o12.r - b.o12.r, a.o12.i - b.o12.i};
    return r;
}

// 1/sqrt(1 + e) - 1 without cancellation
template <typename T>
__device__ __forceinline__ T inv_sqrt1p_m1(T e) {
    const T s = sqrt(T(1) + e);
    return -e / (s * (T(1) + s));
}

// the same per lane of the packed form, without a division slow path:
// with r = 1/sqrt(1 + e) (rsqrtf, a few ulp), r - 1 = -e r / (1 + (1 + e) r),
// which keeps the relative precision of a small e; the division is the fast
// one (its denominator is near 2)
__device__ __forceinline__ float inv_sqrt1p_m1_fast(float e) {
    const float r = rsqrtf(1.f + e);
    return __fdividef(-e * r, 1.f + (1.f + e) * r);
}
__device__ __forceinline__ P2 inv_sqrt1p_m1(P2 e) {
    return P2(inv_sqrt1p_m1_fast(e.v.x), inv_sqrt1p_m1_fast(e.v.y));
}

// Gram-Schmidt reunitarisation of U = 1 + w, in deviation form
template <typename T>
__device__ __forceinline__ void reunitarize_dev(M3<T> &w) {
    // row 0: r0 = e0 + w0
    {
        const T e = T(2) * w.m[0].r + w.m[0].r * w.m[0].r + w.m[0].i * w.m[0].i +
                    w.m[1].r * w.m[1].r + w.m[1].i * w.m[1].i + w.m[2].r * w.m[2].r +
                    w.m[2].i * w.m[2].i;
        const T f = inv_sqrt1p_m1(e);
        w.m[0] = {w.m[0].r + f * (T(1) + w.m[0].r), w.m[0].i + f * w.m[0].i};
        w.m[1] = {w.m[1].r + f * w.m[1].r, w.m[1].i + f * w.m[1].i};
        w.m[2] = {w.m[2].r + f * w.m[2].r, w.m[2].i + f * w.m[2].i};
    }
    // row 1: r1 - <r0, r1> r0, proj = conj(r0) . r1
    {
        const C<T> a0 = w.m[0], a1 = w.m[1], a2 = w.m[2];
        const C<T> b0 = w.m[3], b1 = w.m[4], b2 = w.m[5];
        // (1 + conj a0) b0 + conj(a1) (1 + b1) + conj(a2) b2
        C<T> pr = {b0.r + a1.r, b0.i - a1.i};
        const C<T> t0 = cmulc(b0, a0), t1 = cmulc(b1, a1), t2 = cmulc(b2, a2);
        pr.r += t0.r + t1.r + t2.r;
        pr.i += t0.i + t1.i + t2.i;
        const C<T> p0 = cmul(pr, a0), p1 = cmul(pr, a1), p2 = cmul(pr, a2);
        w.m[3] = {b0.r - pr.r - p0.r, b0.i - pr.i - p0.i};
        w.m[4] = {b1.r - p1.r, b1.i - p1.i};
        w.m[5] = {b2.r - p2.r, b2.i - p2.i};
        const T e = T(2) * w.m[4].r + w.m[3].r * w.m[3].r + w.m[3].i * w.m[3].i +
                    w.m[4].r * w.m[4].r + w.m[4].i * w.m[4].i + w.m[5].r * w.m[5].r +
                    w.m[5].i * w.m[5].i;
        const T f = inv_sqrt1p_m1(e);
        w.m[3] = {w.m[3].r + f * w.m[3].r, w.m[3].i + f * w.m[3].i};
        w.m[4] = {w.m[4].r + f * (T(1) + w.m[4].r), w.m[4].i + f * w.m[4].i};
        w.m[5] = {w.m[5].r + f * w.m[5].r, w.m[5].i + f * w.m[5].i};
    }
    // row 2 = conj((e0 + a) x (e1 + b)) - e2
    {
        const C<T> a0 = w.m[0], a1 = w.m[1], a2 = w.m[2];
        const C<T> b0 = w.m[3], b1 = w.m[4], b2 = w.m[5];
        const C<T> a1b2 = cmul(a1, b2), a2b1 = cmul(a2, b1), a2b0 = cmul(a2, b0);
        const C<T> a0b2 = cmul(a0, b2), a0b1 = cmul(a0, b1), a1b0 = cmul(a1, b0);
        const C<T> c0 = {a1b2.r - a2.r - a2b1.r, a1b2.i - a2.i - a2b1.i};
        const C<T> c1 = {a2b0.r - b2.r - a0b2.r, a2b0.i - b2.i - a0b2.i};
        const C<T> c2 = {a0.r + b1.r + a0b1.r - a1b0.r, a0.i + b1.i + a0b1.i - a1b0.i};
        w.m[6] = {c0.r, -c0.i};
        w.m[7] = {c1.r, -c1.i};
        w.m[8] = {c2.r, -c2.i};
    }
}

// (1 + t)(1 + w) - 1 with t = T2(i c E) - 1 = i c E - (c^2/2) E^2
template <typename T>
__device__ __forceinline__ M3<T> taylor2_update_dev(const H3<T> &e, T c,
                                                    const M3<T> &w) {
    const M3<T> em = from_h(e);
    const M3<T> e2 = mul_g<false, false, true, true>(em, em);
    M3<T> t;
    const T h = T(-0.5) * c * c;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        t.m[k].r = h * e2.m[k].r - c * em.m[k].i;
        t.m[k].i = h * e2.m[k].i + c * em.m[k].r;
    }
    return dmul(t, w);
}

template <typename T>
__global__ void __launch_bounds__(128)
    k_leapfrog_dev(const EventGeom *__restrict__ ev, State<T> s, C<T> *wx_out,
                   C<T> *wy_out, T *phi_out, StepCoef<T> cf) {
    const int N = ev->N;
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    const int ix = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= N || iy >= N) return;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)ix * N + iy;

    if (cf.do_pe) {
        const int ixp = min(N - 1, ix + 1), ixm = max(0, ix - 1);
        const int iyp = min(N - 1, iy + 1), iym = max(0, iy - 1);
        const size_t pX = (size_t)ixp * N + iy, mX = (size_t)ixm * N + iy;
        const size_t pY = (size_t)ix * N + iyp, mY = (size_t)ix * N + iym;
        const size_t mXpY = (size_t)ixm * N + iyp, pXmY = (size_t)ixp * N + iym;

        const M3<T> wx = ld_m3(s.ux, pos, n);
        const M3<T> wy = ld_m3(s.uy, pos, n);
        H3<T> h12;
        {
            const M3<T> a = dmul(wx, ld_m3(s.uy, pX, n));
            const M3<T> b = dmul(wy, ld_m3(s.ux, pY, n));
            h12 = i_antiherm(dmul_nd(a, b));
        }
        H3<T> t1 = h12;
        {
            const M3<T> p = dmul_nd(wx, ld_m3(s.uy, pXmY, n));
            const M3<T> q = dmul_dn(ld_m3(s.ux, mY, n), ld_m3(s.uy, mY, n));
            h_add(t1, i_antiherm(dmul(p, q)));
        }
        H3<T> t2;
        {
            const M3<T> p = dmul_nd(wy, ld_m3(s.ux, mXpY, n));
            const M3<T> q = dmul_dn(ld_m3(s.uy, mX, n), ld_m3(s.ux, mX, n));
            t2 = i_antiherm(dmul(p, q));
            h_axpy(t2, T(-1), h12);
        }
        h_traceless(t1);
        h_traceless(t2);

        const H3<T> phi = ld_h(s.phi, pos, n);
        H3<T> pi = ld_h(s.pi, pos, n);
        H3<T> e1 = ld_h8(s.e1, pos, n);
        H3<T> e2 = ld_h8(s.e2, pos, n);
        const T cst = cf.tau * cf.dt_pe / (T(2) * cf.g * cf.g);
        const T cdt = cf.dt_pe / cf.tau;
        h_axpy(e1, cst, t1);
        h_axpy(e2, cst, t2);

        // bracket = sum_dirs (phi_nb - phi) + connection parts
        H3<T> br;
        {
            const H3<T> fX = ld_h(s.phi, pX, n);
            const H3<T> cX = transport_dev(wx, fX);
            H3<T> pt = fX;
            h_add(pt, cX);
            h_axpy(e1, cdt, i_commutator(pt, phi));
            br = h_diff(fX, phi);
            h_add(br, cX);
        }
        {
            const H3<T> fY = ld_h(s.phi, pY, n);
            const H3<T> cY = transport_dev(wy, fY);
            H3<T> pt = fY;
            h_add(pt, cY);
            h_axpy(e2, cdt, i_commutator(pt, phi));
            h_add(br, h_diff(fY, phi));
            h_add(br, cY);
        }
        {
            const H3<T> f = ld_h(s.phi, mX, n);
            h_add(br, h_diff(f, phi));
            h_add(br, transport_dev_back(ld_m3(s.ux, mX, n), f));
        }
        {
            const H3<T> f = ld_h(s.phi, mY, n);
            h_add(br, h_diff(f, phi));
            h_add(br, transport_dev_back(ld_m3(s.uy, mY, n), f));
        }
        h_axpy(pi, cdt, br);
        h_traceless(e1);
        h_traceless(e2);
        st_h(s.pi, pos, n, pi);
        st_h8(s.e1, pos, n, e1);
        st_h8(s.e2, pos, n, e2);

        if (cf.do_pu) {
            H3<T> phin = phi;
            h_axpy(phin, (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu, pi);
            st_h(phi_out, pos, n, phin);
            const T c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
            M3<T> nx = taylor2_update_dev(e1, c, wx);
            reunitarize_dev(nx);
            st_m3(wx_out, pos, n, nx);
            M3<T> ny = taylor2_update_dev(e2, c, wy);
            reunitarize_dev(ny);
            st_m3(wy_out, pos, n, ny);
        }
    } else if (cf.do_pu) {
        H3<T> phin = ld_h(s.phi, pos, n);
        const H3<T> pi = ld_h(s.pi, pos, n);
        h_axpy(phin, (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu, pi);
        st_h(phi_out, pos, n, phin);
        const T c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
        M3<T> nx = taylor2_update_dev(ld_h8(s.e1, pos, n), c, ld_m3(s.ux, pos, n));
        reunitarize_dev(nx);
        st_m3(wx_out, pos, n, nx);
        M3<T> ny = taylor2_update_dev(ld_h8(s.e2, pos, n), c, ld_m3(s.uy, pos, n));
        reunitarize_dev(ny);
        st_m3(wy_out, pos, n, ny);
    }
}

// Parallel transport of phi from a neighbour, minus phi itself, for a link
// in deviation storage (DEV: U = 1 + w, the FP32 bulk form) or full storage.
// U phi_nb U^dag - phi
template <typename T, bool DEV>
__device__ __forceinline__ H3<T> transport_fwd_minus(const M3<T> &u, const H3<T> &nb,
                                                     const H3<T> &phi) {
    if constexpr (DEV) {
        H3<T> d = h_diff(nb, phi);
        h_add(d, transport_dev(u, nb));
        return d;
    } else {
        return h_diff(conj_h(u, nb), phi);
    }
}
// U^dag phi_nb U - phi
template <typename T, bool DEV>
__device__ __forceinline__ H3<T> transport_bwd_minus(const M3<T> &u, const H3<T> &nb,
                                                     const H3<T> &phi) {
    if constexpr (DEV) {
        H3<T> d = h_diff(nb, phi);
        h_add(d, transport_dev_back(u, nb));
        return d;
    } else {
        return h_diff(conj_h_dag(u, nb), phi);
    }
}

// ---------------------------------------------------------------------------
// FP32 deviation form, one thread per site with both directions packed in the
// two lanes of P2 (pair2.cuh): lane x advances direction d = x (U_d = U_x,
// U_o = U_y, +d = +x, +o = +y), lane y direction d = y. With the plaquette
// written in the (d, o) orientation,
//   P_do  = U_d U_o(+d) U_d(+o)^dag U_o^dag   (for d = x this is U12, for
//           d = y it is U12^dag, so AH(P_do) = +-h12 as in evolveE),
//   S_d   = (U_d U_o(+d-o)^dag)(U_d(-o)^dag U_o(-o))   (U1m2 / U2m1),
// both directions run the same code. Every product of the two directions then costs one
// packed instruction; pi and phi, which belong to the site, stay scalar and
// take the sum of the two lanes' brackets.
// ---------------------------------------------------------------------------
namespace {

// traceless part of a packed pair: (d0 + d1 + d2) / 3 as a product with the
// rounded 1/3 (an IEEE division per lane costs a range check and, for tiny
// traces, a slow-path call)
__device__ __forceinline__ void h_traceless(H3<P2> &h) {
    const P2 t = (h.d0 + h.d1 + h.d2) * P2(1.f / 3.f);
    h.d0 -= t;
    h.d1 -= t;
    h.d2 -= t;
}

// lane x from px at ix, lane y from py at iy
__device__ __forceinline__ M3<P2> ld_m3_pair(const C<float> *__restrict__ px, size_t ix,
                                             const C<float> *__restrict__ py, size_t iy,
                                             size_t n) {
    M3<P2> a;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const C<float> u = px[k * n + ix], w = py[k * n + iy];
        a.m[k] = {P2(u.r, w.r), P2(u.i, w.i)};
    }
    return a;
}

__device__ __forceinline__ void st_m3_pair(C<float> *__restrict__ px, C<float> *__restrict__ py,
                                           size_t pos, size_t n, const M3<P2> &a) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        px[k * n + pos] = {lane_x(a.m[k].r), lane_x(a.m[k].i)};
        py[k * n + pos] = {lane_y(a.m[k].r), lane_y(a.m[k].i)};
    }
}

__device__ __forceinline__ H3<P2> pair_h(const H3<float> &a, const H3<float> &b) {
    H3<P2> h;
    h.d0 = P2(a.d0, b.d0);
    h.d1 = P2(a.d1, b.d1);
    h.d2 = P2(a.d2, b.d2);
    h.o01 = {P2(a.o01.r, b.o01.r), P2(a.o01.i, b.o01.i)};
    h.o02 = {P2(a.o02.r, b.o02.r), P2(a.o02.i, b.o02.i)};
    h.o12 = {P2(a.o12.r, b.o12.r), P2(a.o12.i, b.o12.i)};
    return h;
}

__device__ __forceinline__ M3<P2> swap_lanes(const M3<P2> &a) {
    M3<P2> b;
#pragma unroll
    for (int k = 0; k < 9; k++)
        b.m[k] = {P2(a.m[k].r.v.y, a.m[k].r.v.x), P2(a.m[k].i.v.y, a.m[k].i.v.x)};
    return b;
}

__device__ __forceinline__ H3<float> lane_h(const H3<P2> &h, int y) {
    auto l = [&](P2 v) { return y ? lane_y(v) : lane_x(v); };
    H3<float> r;
    r.d0 = l(h.d0);
    r.d1 = l(h.d1);
    r.d2 = l(h.d2);
    r.o01 = {l(h.o01.r), l(h.o01.i)};
    r.o02 = {l(h.o02.r), l(h.o02.i)};
    r.o12 = {l(h.o12.r), l(h.o12.i)};
    return r;
}

}  // namespace

// Loads from the global planes, neighbours clamped at the lattice edge
// (Lattice.cpp:19-28).
struct PairLoadGlobal {
    const State<float> &s;
    size_t pos, n;
    long ox[3], oy[3];  // index offsets of dx (dy) = -1, 0, +1, clamped
    __device__ __forceinline__ PairLoadGlobal(const State<float> &s_, int N, int ix, int iy)
        : s(s_), pos((size_t)ix * N + iy), n((size_t)N * N) {
        ox[0] = ix > 0 ? -(long)N : 0;
        ox[1] = 0;
        ox[2] = ix + 1 < N ? N : 0;
        oy[0] = iy > 0 ? -1 : 0;
        oy[1] = 0;
        oy[2] = iy + 1 < N ? 1 : 0;
        own = ld_m3_pair(s.ux, pos, s.uy, pos, n);
    }
    // the site's own pair is loaded once and held (from global memory a
    // reload costs more than the registers; the tile loader reloads it)
    M3<P2> own;
    template <int FA, int DXA, int DYA, int FB, int DXB, int DYB>
    __device__ __forceinline__ M3<P2> links() const {
        if constexpr (FA == kLx && DXA == 0 && DYA == 0 && FB == kLy && DXB == 0 && DYB == 0)
            return own;
        else
            return ld_m3_pair(FA == kLy ? s.uy : s.ux, pos + ox[DXA + 1] + oy[DYA + 1],
                              FB == kLy ? s.uy : s.ux, pos + ox[DXB + 1] + oy[DYB + 1], n);
    }
    template <int DX, int DY>
    __device__ __forceinline__ H3<float> phi() const {
        return ld_h(s.phi, pos + ox[DX + 1] + oy[DY + 1], n);
    }
    __device__ __forceinline__ H3<float> pi() const { return ld_h(s.pi, pos, n); }
    __device__ __forceinline__ H3<float> e1() const { return ld_h8(s.e1, pos, n); }
    __device__ __forceinline__ H3<float> e2() const { return ld_h8(s.e2, pos, n); }
    // E and pi are site-local: written back in place
    __device__ __forceinline__ void put_e(const H3<float> &a, const H3<float> &b) const {
        st_h8(s.e1, pos, n, a);
        st_h8(s.e2, pos, n, b);
    }
    __device__ __forceinline__ void put_pi(const H3<float> &h) const { st_h(s.pi, pos, n, h); }
};

// One site of the FP32 step, both directions in the packed lanes. Loads
// through `ld` (global planes or a shared-memory tile), writes the new E and
// pi through it (site-local, so they may go back in place at once) and
// returns the new links (nu) and phi (phin) when cf.do_pu is set, for the
// caller to store once no other thread reads the old ones. The site's own
// link pair is loaded again at each use instead of being held (the tile
// kernel then fits in 252 registers without spilling).
template <class Ld>
__device__ __forceinline__ void leapfrog_pair_core(const Ld &ld, const StepCoef<float> &cf,
                                                   M3<P2> &nu, H3<float> &phin) {
    const H3<float> phi = ld.template phi<0, 0>();
    H3<float> pi = ld.pi();
    H3<P2> Ed = pair_h(ld.e1(), ld.e2());

    if (cf.do_pe) {
        const H3<P2> phi2 = pair_h(phi, phi);
        H3<P2> stap;
        {
            // P_do = (U_d U_o(+d)) (U_o U_d(+o))^dag: lane x of a = U_d U_o(+d)
            // is Ux Uy(+x), lane y is Uy Ux(+y); U_o U_d(+o) is the same pair
            // of products with the lanes swapped
            const M3<P2> a = dmul(ld.template links<kLx, 0, 0, kLy, 0, 0>(), ld.template links<kLy, 1, 0, kLx, 0, 1>());
            stap = i_antiherm(dmul_nd(a, swap_lanes(a)));
        }
        {
            // S_d = (U_d U_o(+d-o)^dag) (U_d(-o)^dag U_o(-o))
            const M3<P2> p = dmul_nd(ld.template links<kLx, 0, 0, kLy, 0, 0>(), ld.template links<kLy, 1, -1, kLx, -1, 1>());
            const M3<P2> q = dmul_dn(ld.template links<kLx, 0, -1, kLy, -1, 0>(),
                                     ld.template links<kLy, 0, -1, kLx, -1, 0>());
            h_add(stap, i_antiherm(dmul(p, q)));
        }
        h_traceless(stap);
        const P2 cst = P2(cf.c_e);
        const P2 cdt = P2(cf.c_pi);
        h_axpy(Ed, cst, stap);
        const H3<P2> fp = pair_h(ld.template phi<1, 0>(), ld.template phi<0, 1>());
        H3<P2> br = transport_fwd_minus<P2, true>(ld.template links<kLx, 0, 0, kLy, 0, 0>(), fp, phi2);
        h_axpy(Ed, cdt, i_commutator(br, phi2));  // i[phi~ - phi, phi] = i[phi~, phi]
        const H3<P2> fm = pair_h(ld.template phi<-1, 0>(), ld.template phi<0, -1>());
        h_add(br, transport_bwd_minus<P2, true>(ld.template links<kLx, -1, 0, kLy, 0, -1>(), fm,
                                                phi2));
        H3<float> brs = lane_h(br, 0);
        h_add(brs, lane_h(br, 1));
        h_axpy(pi, cf.c_pi, brs);
        h_traceless(Ed);
        ld.put_e(lane_h(Ed, 0), lane_h(Ed, 1));
        ld.put_pi(pi);
    }
    if (cf.do_pu) {
        nu = taylor2_update_dev(Ed, P2(cf.c_u), ld.template links<kLx, 0, 0, kLy, 0, 0>());
        reunitarize_dev(nu);
        phin = phi;
        h_axpy(phin, cf.c_phi, pi);
    }
}

__device__ __forceinline__ void leapfrog_pair_site(int N, int ix, int iy, const State<float> &s,
                                                   C<float> *ux_out, C<float> *uy_out,
                                                   float *phi_out, const StepCoef<float> &cf) {
    const PairLoadGlobal ld(s, N, ix, iy);
    M3<P2> nu;
    H3<float> phin;
    leapfrog_pair_core(ld, cf, nu, phin);
    if (cf.do_pu) {
        st_m3_pair(ux_out, uy_out, ld.pos, ld.n, nu);
        st_h(phi_out, ld.pos, ld.n, phin);
    }
}

// block: 256 threads = 32 sites along y x 8 along x; the grid covers the
// lattice exactly (N a multiple of 32)
__global__ void __launch_bounds__(256, 1)
    k_leapfrog_pair(const EventGeom *__restrict__ ev, State<float> s, C<float> *ux_out,
                    C<float> *uy_out, float *phi_out, StepCoef<float> cf) {
    const int iy = blockIdx.x * 32 + (threadIdx.x & 31);
    const int ix = blockIdx.y * 8 + (threadIdx.x >> 5);
    leapfrog_pair_site(ev->N, ix, iy, s, ux_out, uy_out, phi_out, cf);
}

// ---------------------------------------------------------------------------
// FP32 step with the fields staged in shared memory by TMA. A persistent
// block per SM walks tiles of 8 rows (x) x 32 columns (y), one thread per
// site (warp r takes row r); the loads of tile i+2 are in flight while tile i
// is computed (two stages). A stage holds, per tile,
//   Ux, Uy   [9][10][36] complex   rows ix0-1 .. ix0+8, columns iy0-2 .. iy0+33
//   phi      [9][10][40] real      rows ix0-1 .. ix0+8, columns iy0-4 .. iy0+35
//   E1, E2   [8][8][32], pi [9][8][32]   the tile's own sites
// (the column starts keep each box's first column 16-byte aligned, as TMA
// requires). Boxes reaching past the lattice are zero filled; on edge tiles
// each warp then overwrites the halo cells of the rows it reads with the
// clamped neighbours (Lattice.cpp:19-28), so every neighbour read is a fixed
// offset from the thread's own cell. There is no block-wide barrier in the
// loop: a stage's "full" barrier completes with its TMA bytes, each warp
// arrives on its "empty" barrier once it has read the stage, and thread 0
// waits on "empty" before loading the stage again. Results go to global
// memory from registers (E and pi in place).
// ---------------------------------------------------------------------------
namespace tile {
constexpr int R = 8, Cn = 32;            // tile rows (x) and columns (y)
constexpr int UR = R + 2, UC = Cn + 4;   // link box
constexpr int PR = R + 2, PC = Cn + 8;   // phi box
constexpr int kU = UR * UC, kP = PR * PC, kS = R * Cn;  // component strides
constexpr int round128(int b) { return (b + 127) / 128 * 128; }
constexpr int UX = 0;
constexpr int UY = UX + round128(9 * kU * 8);
constexpr int PHI = UY + round128(9 * kU * 8);
constexpr int E1 = PHI + round128(9 * kP * 4);
constexpr int E2 = E1 + round128(8 * kS * 4);
constexpr int PI = E2 + round128(8 * kS * 4);
constexpr int STAGE = PI + round128(9 * kS * 4);
constexpr uint32_t TX_BYTES = 2 * 9 * kU * 8 + 9 * kP * 4 + 2 * 8 * kS * 4 + 9 * kS * 4;
constexpr int SMEM = 2 * STAGE + 64 + 128;  // two stages, four barriers, alignment slack
constexpr uint32_t MAX_POLLS = 1u << 22;
static_assert(STAGE % 128 == 0, "stage alignment");
static_assert(SMEM <= 227 * 1024, "shared memory per block");
}  // namespace tile


// 32-bit shared-memory accesses by address: one value per instruction, so
// each lands directly in its lane of a packed pair
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts_f32(uint32_t a, float v) {
    asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

// Loads from one stage; the thread sits at row r, column c of the tile.
// Addresses are a per-thread base plus compile-time offsets: bu and bp point
// at the (-1, -1) corner of the thread's 3 x 3 neighbourhood in the link and
// phi boxes, bs at its cell of the site-local boxes. Imaginary parts of links
// are read through bi = bu + imag, with imag (= 4) a kernel argument: were the
// adjacency of a link's real and imaginary parts visible, the compiler would
// fuse the two 32-bit loads into one 64-bit load, whose register pair is
// (re, im) of one link while the packed arithmetic needs (re, re) of the two
// lanes, and every use would then be preceded by moves (measured: 35 M
// instructions a step at 512^2 instead of 18.5 M).
struct PairLoadTile {
    uint32_t bu, bi, bp, bs;
    const State<float> &g;  // E and pi are written here, in place
    size_t pos, n;
    __device__ __forceinline__ PairLoadTile(uint32_t stage, int r, int c, uint32_t imag,
                                            const State<float> &g_, size_t pos_, size_t n_)
        : bu(stage + (uint32_t)((r * tile::UC + c + 1) * 8)),
          bi(stage + (uint32_t)((r * tile::UC + c + 1) * 8) + imag),
          bp(stage + tile::PHI + (uint32_t)((r * tile::PC + c + 3) * 4)),
          bs(stage + (uint32_t)((r * tile::Cn + c) * 4)), g(g_), pos(pos_), n(n_) {}
    template <int FA, int DXA, int DYA, int FB, int DXB, int DYB>
    __device__ __forceinline__ M3<P2> links() const {
        constexpr uint32_t oa =
            (FA == kLy ? tile::UY : tile::UX) + ((DXA + 1) * tile::UC + DYA + 1) * 8;
        constexpr uint32_t ob =
            (FB == kLy ? tile::UY : tile::UX) + ((DXB + 1) * tile::UC + DYB + 1) * 8;
        M3<P2> m;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const uint32_t o = k * tile::kU * 8;
            m.m[k] = {P2(lds_f32(bu + oa + o), lds_f32(bu + ob + o)),
                      P2(lds_f32(bi + oa + o), lds_f32(bi + ob + o))};
        }
        return m;
    }
    static __device__ __forceinline__ H3<float> h9(uint32_t a, uint32_t stride) {
        H3<float> h;
        h.d0 = lds_f32(a);
        h.d1 = lds_f32(a + stride);
        h.d2 = lds_f32(a + 2 * stride);
        h.o01 = {lds_f32(a + 3 * stride), lds_f32(a + 4 * stride)};
        h.o02 = {lds_f32(a + 5 * stride), lds_f32(a + 6 * stride)};
        h.o12 = {lds_f32(a + 7 * stride), lds_f32(a + 8 * stride)};
        return h;
    }
    static __device__ __forceinline__ H3<float> h8(uint32_t a) {
        constexpr uint32_t S = tile::kS * 4;
        H3<float> h;
        h.d0 = lds_f32(a);
        h.d1 = lds_f32(a + S);
        h.d2 = -(h.d0 + h.d1);
        h.o01 = {lds_f32(a + 2 * S), lds_f32(a + 3 * S)};
        h.o02 = {lds_f32(a + 4 * S), lds_f32(a + 5 * S)};
        h.o12 = {lds_f32(a + 6 * S), lds_f32(a + 7 * S)};
        return h;
    }
    template <int DX, int DY>
    __device__ __forceinline__ H3<float> phi() const {
        return h9(bp + ((DX + 1) * tile::PC + DY + 1) * 4, tile::kP * 4);
    }
    __device__ __forceinline__ H3<float> pi() const { return h9(bs + tile::PI, tile::kS * 4); }
    __device__ __forceinline__ H3<float> e1() const { return h8(bs + tile::E1); }
    __device__ __forceinline__ H3<float> e2() const { return h8(bs + tile::E2); }
    __device__ __forceinline__ void put_e(const H3<float> &a, const H3<float> &b) const {
        st_h8(g.e1, pos, n, a);
        st_h8(g.e2, pos, n, b);
    }
    __device__ __forceinline__ void put_pi(const H3<float> &h) const { st_h(g.pi, pos, n, h); }
};

// Edge tiles: halo cells outside the lattice take the clamped neighbour,
// each coordinate clamped on its own (corners included). Sources are cells of
// the lattice, which no thread writes here, so one pass suffices. A box of
// ROWS rows holds the tile's rows 1 .. ROWS-2 between two halo rows; the
// halo columns are LO (column -1 of the tile) and LO + 33 (column 32). UT is
// the link element, PT the phi element; 9 components of each.
template <class UT, class PT, int ROWS, int UC, int ULO, int PC, int PLO>
__device__ __forceinline__ void fill_edge_halo(UT *ux, UT *uy, PT *ph, bool top, bool bottom,
                                               bool left, bool right) {
    constexpr int ROW = 34, COL = ROWS;  // cells per halo row / halo column
    constexpr int CELLS = 2 * ROW + 2 * COL;
    for (int w = threadIdx.x; w < 9 * 2 * CELLS; w += blockDim.x) {
        const int k = w / (2 * CELLS);
        int cell = w - k * (2 * CELLS);
        const bool link = cell < CELLS;
        if (!link) cell -= CELLS;
        const int cols = link ? UC : PC;
        const int c_lo = link ? ULO : PLO, c_hi = c_lo + 33;
        int j, m;
        bool edge;
        if (cell < 2 * ROW) {
            const int side = cell / ROW;
            j = side ? ROWS - 1 : 0;
            m = c_lo + cell % ROW;
            edge = side ? bottom : top;
        } else {
            cell -= 2 * ROW;
            const int side = cell / COL;
            j = cell % COL;
            m = side ? c_hi : c_lo;
            edge = side ? right : left;
        }
        if (!edge) continue;
        int sj = j, sm = m;
        if (top && j == 0) sj = 1;
        if (bottom && j == ROWS - 1) sj = ROWS - 2;
        if (left && m == c_lo) sm = c_lo + 1;
        if (right && m == c_hi) sm = c_hi - 1;
        if (link) {
            constexpr int KU = ROWS * UC;
            const int d = k * KU + j * cols + m, s = k * KU + sj * cols + sm;
            ux[d] = ux[s];
            uy[d] = uy[s];
        } else {
            constexpr int KP = ROWS * PC;
            ph[k * KP + j * cols + m] = ph[k * KP + sj * cols + sm];
        }
    }
}

// Edge tiles, one warp: the halo cells of the box rows r .. r+2 that warp r
// reads (its tile row and the rows on either side) take the clamped
// neighbour, each coordinate clamped on its own. Sources are lattice cells,
// which nobody writes; warps whose rows overlap write the same values.
__device__ __forceinline__ void fill_warp_halo(unsigned char *st, int r, int lane, bool top,
                                               bool bottom, bool left, bool right) {
    C<float> *ux = reinterpret_cast<C<float> *>(st + tile::UX);
    C<float> *uy = reinterpret_cast<C<float> *>(st + tile::UY);
    float *ph = reinterpret_cast<float *>(st + tile::PHI);
    auto clamp_j = [&](int j) { return (top && j == 0) ? 1 : ((bottom && j == tile::UR - 1) ? j - 1 : j); };
    // halo columns (links 1 and 34, phi 3 and 36) of rows r .. r+2
    if (left || right) {
        for (int w = lane; w < 9 * 3 * 2; w += 32) {
            const int k = w / 6, j = r + (w % 6) / 2, side = w & 1;
            if (side ? !right : !left) continue;
            const int sj = clamp_j(j);
            const int mu = side ? 34 : 1, su = side ? 33 : 2;
            const int mp = side ? 36 : 3, sp = side ? 35 : 4;
            ux[k * tile::kU + j * tile::UC + mu] = ux[k * tile::kU + sj * tile::UC + su];
            uy[k * tile::kU + j * tile::UC + mu] = uy[k * tile::kU + sj * tile::UC + su];
            ph[k * tile::kP + j * tile::PC + mp] = ph[k * tile::kP + sj * tile::PC + sp];
        }
    }
    // the halo row above (warp 0, top edge) or below (warp 7, bottom edge)
    const bool row_top = top && r == 0, row_bottom = bottom && r == tile::R - 1;
    if (row_top || row_bottom) {
        const int j = row_top ? 0 : tile::UR - 1, sj = row_top ? 1 : tile::UR - 2;
        for (int w = lane; w < 9 * 34; w += 32) {
            const int k = w / 34, q = w % 34;
            int mu = 1 + q, mp = 3 + q;  // links 1..34, phi 3..36
            int su = mu, sp = mp;
            if (left && q == 0) su = 2, sp = 4;
            if (right && q == 33) su = 33, sp = 35;
            ux[k * tile::kU + j * tile::UC + mu] = ux[k * tile::kU + sj * tile::UC + su];
            uy[k * tile::kU + j * tile::UC + mu] = uy[k * tile::kU + sj * tile::UC + su];
            ph[k * tile::kP + j * tile::PC + mp] = ph[k * tile::kP + sj * tile::PC + sp];
        }
    }
}

// Where the tiles of a persistent FP32 tile loop come from: one event
// (tensor maps in the kernel's parameter space) or a batch of events (tile
// lists concatenated, per-event descriptors in shared memory and tensor maps
// in global memory).
struct OneEventTiles {
    const LoadMaps *maps;
    int N;
    StepCoef<float> cf;
    State<float> gs;
    C<float> *ux_out, *uy_out;
    float *phi_out;
    int total;
    __device__ __forceinline__ int find(int) const { return 0; }
    __device__ __forceinline__ int first_tile(int) const { return 0; }
    __device__ __forceinline__ int n_of(int) const { return N; }
    __device__ __forceinline__ const LoadMaps *maps_of(int) const { return maps; }
    static constexpr bool kGlobalMaps = false;
    __device__ __forceinline__ bool active(int) const { return true; }
    __device__ __forceinline__ const StepCoef<float> &cf_of(int) const { return cf; }
    __device__ __forceinline__ const State<float> &state_of(int) const { return gs; }
    __device__ __forceinline__ C<float> *ux_out_of(int) const { return ux_out; }
    __device__ __forceinline__ C<float> *uy_out_of(int) const { return uy_out; }
    __device__ __forceinline__ float *phi_out_of(int) const { return phi_out; }
};

struct BatchTiles {
    const BatchEvent<float> *ev;  // shared memory
    const int *begin;             // shared memory, [n_events + 1]
    int n_events;
    const LoadMaps *maps;         // global memory, [2 n_events]
    int total;
    // last e with begin[e] <= t
    __device__ __forceinline__ int find(int t) const {
        int lo = 0, hi = n_events - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (begin[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    }
    __device__ __forceinline__ int first_tile(int e) const { return begin[e]; }
    __device__ __forceinline__ int n_of(int e) const { return ev[e].N; }
    __device__ __forceinline__ const LoadMaps *maps_of(int e) const {
        return maps + 2 * e + ev[e].map_sel;
    }
    static constexpr bool kGlobalMaps = true;
    __device__ __forceinline__ bool active(int e) const { return ev[e].active != 0; }
    __device__ __forceinline__ const StepCoef<float> &cf_of(int e) const { return ev[e].cf; }
    __device__ __forceinline__ const State<float> &state_of(int e) const { return ev[e].s; }
    __device__ __forceinline__ C<float> *ux_out_of(int e) const { return ev[e].ux_out; }
    __device__ __forceinline__ C<float> *uy_out_of(int e) const { return ev[e].uy_out; }
    __device__ __forceinline__ float *phi_out_of(int e) const { return ev[e].phi_out; }
};

// The persistent FP32 tile loop. smem: two stages (128-byte aligned) then
// four barriers. Tile t of the list belongs to event find(t); its local index
// gives (tx, ty) in that event's N/8 x N/32 tile grid.
template <class Tiles>
__device__ __forceinline__ void tile32_loop(const Tiles &T, unsigned char *smem, double *status,
                                            uint32_t imag) {
    const uint32_t sbase = smem_addr(smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + 2 * tile::STAGE);
    uint64_t *empty = full + 2;
    const int tid = threadIdx.x, r = tid >> 5, c = tid & 31;
    const int tiles = T.total;
    const LoadMaps *fenced = nullptr;  // thread 0: the maps acquired last

    auto issue = [&](int t, int s) {
        const int e = T.find(t);
        const int N = T.n_of(e), tiles_y = N / tile::Cn, local = t - T.first_tile(e);
        const int iy0 = (local % tiles_y) * tile::Cn, ix0 = (local / tiles_y) * tile::R;
        const LoadMaps *m = T.maps_of(e);
        if (Tiles::kGlobalMaps && m != fenced) {
            fence_map_acquire(&m->ux);
            fence_map_acquire(&m->uy);
            fence_map_acquire(&m->phi);
            fence_map_acquire(&m->e1);
            fence_map_acquire(&m->e2);
            fence_map_acquire(&m->pi);
            fenced = m;
        }
        unsigned char *st = smem + s * tile::STAGE;
        mbar_arrive_expect_tx(&full[s], tile::TX_BYTES);
        tma_load_3d(st + tile::UX, &m->ux, iy0 - 2, ix0 - 1, 0, &full[s]);
        tma_load_3d(st + tile::UY, &m->uy, iy0 - 2, ix0 - 1, 0, &full[s]);
        tma_load_3d(st + tile::PHI, &m->phi, iy0 - 4, ix0 - 1, 0, &full[s]);
        tma_load_3d(st + tile::E1, &m->e1, iy0, ix0, 0, &full[s]);
        tma_load_3d(st + tile::E2, &m->e2, iy0, ix0, 0, &full[s]);
        tma_load_3d(st + tile::PI, &m->pi, iy0, ix0, 0, &full[s]);
    };

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(&empty[0], tile::R);  // one arrival per warp
        mbar_init(&empty[1], tile::R);
        fence_barrier_init();
        if (!Tiles::kGlobalMaps) {
            const LoadMaps *m = T.maps_of(0);
            prefetch_map(&m->ux);
            prefetch_map(&m->uy);
            prefetch_map(&m->phi);
        }
        if (blockIdx.x < tiles) issue(blockIdx.x, 0);
        if (blockIdx.x + gridDim.x < tiles) issue(blockIdx.x + gridDim.x, 1);
    }
    __syncthreads();  // barriers initialised before anyone waits on them

    int i = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, i++) {
        const int s = i & 1;
        const uint32_t use = (uint32_t)(i >> 1) & 1u;
        if (!mbar_wait_bounded(&full[s], use, tile::MAX_POLLS)) {
            if (status) *status = 1.0;  // the tile never arrived
            break;
        }
        unsigned char *st = smem + s * tile::STAGE;
        const int e = T.find(t);
        const int N = T.n_of(e), tiles_y = N / tile::Cn, tiles_x = N / tile::R;
        const int local = t - T.first_tile(e);
        const int ty = local % tiles_y, tx = local / tiles_y;
        const bool top = tx == 0, bottom = tx == tiles_x - 1;
        const bool left = ty == 0, right = ty == tiles_y - 1;
        const bool edge = top || bottom || left || right;
        const bool act = T.active(e);
        if (edge && act) {
            fill_warp_halo(st, r, c, top, bottom, left, right);
            __syncwarp();
        }
        const size_t n = (size_t)N * N;
        const size_t pos = (size_t)(tx * tile::R + r) * N + ty * tile::Cn + c;
        const StepCoef<float> &cf = T.cf_of(e);
        M3<P2> nu;
        H3<float> phin;
        if (act) {
            const PairLoadTile ld(sbase + (uint32_t)(s * tile::STAGE), r, c, imag, T.state_of(e),
                                  pos, n);
            leapfrog_pair_core(ld, cf, nu, phin);
        }
        // this warp is done with the stage (its halo writes ordered before the
        // TMA unit writes the stage again)
        if (edge && act) fence_async_smem();
        __syncwarp();
        if (c == 0) mbar_arrive(&empty[s]);
        if (act && cf.do_pu) {
            st_m3_pair(T.ux_out_of(e), T.uy_out_of(e), pos, n, nu);
            st_h(T.phi_out_of(e), pos, n, phin);
        }
        if (tid == 0 && t + 2 * (int)gridDim.x < tiles) {
            if (!mbar_wait_bounded(&empty[s], use, tile::MAX_POLLS)) {
                if (status) *status = 1.0;  // a warp never released the stage
                break;
            }
            issue(t + 2 * gridDim.x, s);
        }
    }
}

__global__ void __launch_bounds__(256, 1)
    k_leapfrog_tile(const __grid_constant__ LoadMaps maps, int N, StepCoef<float> cf,
                    double *status, uint32_t imag, State<float> gs, C<float> *ux_out,
                    C<float> *uy_out, float *phi_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // 128-byte aligned start, kept as an offset into the shared array so that
    // accesses through it stay shared-memory accesses
    const uint32_t pad = (128u - (smem_addr(smem_raw) & 127u)) & 127u;
    const OneEventTiles T{&maps, N, cf, gs, ux_out, uy_out, phi_out,
                          (N / tile::R) * (N / tile::Cn)};
    tile32_loop(T, smem_raw + pad, status, imag);
}

// The FP32 batch over the TMA tiles: the descriptors of this step and the
// tile prefix sums are copied to shared memory behind the two stages.
__global__ void __launch_bounds__(256, 1)
    k_leapfrog_tile_batch(const BatchEvent<float> *__restrict__ evs, int n_events,
                          const int *__restrict__ tile_begin, int total_tiles,
                          const LoadMaps *__restrict__ maps, double *status, uint32_t imag) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t pad = (128u - (smem_addr(smem_raw) & 127u)) & 127u;
    unsigned char *smem = smem_raw + pad;
    BatchEvent<float> *s_ev =
        reinterpret_cast<BatchEvent<float> *>(smem + 2 * tile::STAGE + 64);
    int *s_begin = reinterpret_cast<int *>(s_ev + n_events);
    {
        const int words = n_events * (int)(sizeof(BatchEvent<float>) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(evs);
        int *dst = reinterpret_cast<int *>(s_ev);
        for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
    }
    for (int e = threadIdx.x; e <= n_events; e += blockDim.x) s_begin[e] = tile_begin[e];
    __syncthreads();
    const BatchTiles T{s_ev, s_begin, n_events, maps, total_tiles};
    tile32_loop(T, smem, status, imag);
}

// ---------------------------------------------------------------------------
// FP64 step with the fields staged in shared memory by TMA: one block of 128
// threads per tile of 4 rows (x) x 32 columns (y), one thread per site, two
// blocks resident per SM (one stage each, so one block's loads overlap the
// other's arithmetic). The stage holds
//   Ux, Uy   [9][6][34] complex   rows ix0-1 .. ix0+4, columns iy0-1 .. iy0+32
//   phi      [9][6][36] real      rows ix0-1 .. ix0+4, columns iy0-2 .. iy0+33
//   E1, E2   [8][4][32], pi [9][4][32]   the tile's own sites
// with edge halos clamped as in the FP32 tile kernel. The per-site code is
// the one of the global-memory kernel (leapfrog_full_core); results go to
// global memory from registers (E and pi in place).
// ---------------------------------------------------------------------------
namespace tile64 {
constexpr int R = 4, Cn = 32;
constexpr int UR = R + 2, UC = Cn + 2;  // link box
constexpr int PR = R + 2, PC = Cn + 4;  // phi box
constexpr int kU = UR * UC, kP = PR * PC, kS = R * Cn;
constexpr int UX = 0;
constexpr int UY = UX + tile::round128(9 * kU * 16);
constexpr int PHI = UY + tile::round128(9 * kU * 16);
constexpr int E1 = PHI + tile::round128(9 * kP * 8);
constexpr int E2 = E1 + tile::round128(8 * kS * 8);
constexpr int PI = E2 + tile::round128(8 * kS * 8);
constexpr int STAGE = PI + tile::round128(9 * kS * 8);
constexpr uint32_t TX_BYTES = 2 * 9 * kU * 16 + 9 * kP * 8 + 2 * 8 * kS * 8 + 9 * kS * 8;
constexpr int SMEM = STAGE + 64 + 128;
static_assert(2 * (SMEM + 1024) <= 228 * 1024, "two blocks per SM");
}  // namespace tile64

// Loads from the stage (shared memory) by 32-bit address; the thread sits at
// row r, column c. bl and bp point at the (-1, -1) corner of its 3 x 3
// neighbourhood in the link and phi boxes, bs at its own cell of the
// site-local boxes. The loads are explicit shared-memory instructions, so a
// link loaded twice is read twice rather than kept live in registers; E and
// pi are written to global memory in place.
__device__ __forceinline__ C<double> lds_c64(uint32_t a) {
    double re, im;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(re), "=d"(im) : "r"(a));
    return {re, im};
}
__device__ __forceinline__ double lds_f64(uint32_t a) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}

struct FullLoadTile64 {
    uint32_t bl, bp, bs;
    const State<double> &g;
    size_t pos, n;
    __device__ __forceinline__ FullLoadTile64(uint32_t stage, int r, int c,
                                              const State<double> &g_, size_t pos_, size_t n_)
        : bl(stage + (uint32_t)((r * tile64::UC + c) * 16)),
          bp(stage + tile64::PHI + (uint32_t)((r * tile64::PC + c + 1) * 8)),
          bs(stage + (uint32_t)((r * tile64::Cn + c) * 8)),
          g(g_), pos(pos_), n(n_) {}
    template <int F, int DX, int DY>
    __device__ __forceinline__ M3<double> link() const {
        constexpr uint32_t o =
            (F == kLy ? tile64::UY : tile64::UX) + ((DX + 1) * tile64::UC + DY + 1) * 16;
        M3<double> m;
#pragma unroll
        for (int k = 0; k < 9; k++) m.m[k] = lds_c64(bl + o + k * tile64::kU * 16);
        return m;
    }
    static __device__ __forceinline__ H3<double> h9(uint32_t a, uint32_t S) {
        H3<double> h;
        h.d0 = lds_f64(a);
        h.d1 = lds_f64(a + S);
        h.d2 = lds_f64(a + 2 * S);
        h.o01 = {lds_f64(a + 3 * S), lds_f64(a + 4 * S)};
        h.o02 = {lds_f64(a + 5 * S), lds_f64(a + 6 * S)};
        h.o12 = {lds_f64(a + 7 * S), lds_f64(a + 8 * S)};
        return h;
    }
    static __device__ __forceinline__ H3<double> h8(uint32_t a) {
        constexpr uint32_t S = tile64::kS * 8;
        H3<double> h;
        h.d0 = lds_f64(a);
        h.d1 = lds_f64(a + S);
        h.d2 = -(h.d0 + h.d1);
        h.o01 = {lds_f64(a + 2 * S), lds_f64(a + 3 * S)};
        h.o02 = {lds_f64(a + 4 * S), lds_f64(a + 5 * S)};
        h.o12 = {lds_f64(a + 6 * S), lds_f64(a + 7 * S)};
        return h;
    }
    template <int DX, int DY>
    __device__ __forceinline__ H3<double> phi() const {
        return h9(bp + ((DX + 1) * tile64::PC + DY + 1) * 8, tile64::kP * 8);
    }
    __device__ __forceinline__ H3<double> pi() const { return h9(bs + tile64::PI, tile64::kS * 8); }
    __device__ __forceinline__ H3<double> e1() const { return h8(bs + tile64::E1); }
    __device__ __forceinline__ H3<double> e2() const { return h8(bs + tile64::E2); }
    __device__ __forceinline__ void put_e(const H3<double> &a, const H3<double> &b) const {
        st_h8(g.e1, pos, n, a);
        st_h8(g.e2, pos, n, b);
    }
    __device__ __forceinline__ void put_pi(const H3<double> &h) const { st_h(g.pi, pos, n, h); }
};

// One 4 x 32 tile of the FP64 step: load the stage, wait, clamp the halo on
// edge tiles, advance the tile's sites. tx, ty: the tile in the event's
// N/4 x N/32 grid.
template <bool GLOBAL_MAPS>
__device__ __forceinline__ void tile64_body(const LoadMaps *maps, int N, int tx, int ty,
                                            const StepCoef<double> &cf, double *status,
                                            const State<double> &s, C<double> *ux_out,
                                            C<double> *uy_out, double *phi_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t pad = (128u - (smem_addr(smem_raw) & 127u)) & 127u;
    unsigned char *smem = smem_raw + pad;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + tile64::STAGE);
    int *abort_flag = reinterpret_cast<int *>(full + 1);
    const int tiles_y = N / tile64::Cn, tiles_x = N / tile64::R;
    const int iy0 = ty * tile64::Cn, ix0 = tx * tile64::R;
    const int tid = threadIdx.x, r = tid >> 5, c = tid & 31;
    if (tid == 0) {
        mbar_init(full, 1);
        *abort_flag = 0;
        fence_barrier_init();
        if (GLOBAL_MAPS) {
            fence_map_acquire(&maps->ux);
            fence_map_acquire(&maps->uy);
            fence_map_acquire(&maps->phi);
            fence_map_acquire(&maps->e1);
            fence_map_acquire(&maps->e2);
            fence_map_acquire(&maps->pi);
        }
        mbar_arrive_expect_tx(full, tile64::TX_BYTES);
        // links as pairs of 8-byte words: column iy0-1 is word 2 (iy0 - 1)
        tma_load_3d(smem + tile64::UX, &maps->ux, 2 * (iy0 - 1), ix0 - 1, 0, full);
        tma_load_3d(smem + tile64::UY, &maps->uy, 2 * (iy0 - 1), ix0 - 1, 0, full);
        tma_load_3d(smem + tile64::PHI, &maps->phi, iy0 - 2, ix0 - 1, 0, full);
        tma_load_3d(smem + tile64::E1, &maps->e1, iy0, ix0, 0, full);
        tma_load_3d(smem + tile64::E2, &maps->e2, iy0, ix0, 0, full);
        tma_load_3d(smem + tile64::PI, &maps->pi, iy0, ix0, 0, full);
    }
    __syncthreads();
    if (!mbar_wait_bounded(full, 0, tile::MAX_POLLS)) *abort_flag = 1;
    __syncthreads();
    if (*abort_flag) {
        if (tid == 0 && status) *status = 1.0;
        return;
    }
    const bool top = tx == 0, bottom = tx == tiles_x - 1;
    const bool left = ty == 0, right = ty == tiles_y - 1;
    if (top || bottom || left || right) {
        fill_edge_halo<C<double>, double, tile64::UR, tile64::UC, 0, tile64::PC, 1>(
            reinterpret_cast<C<double> *>(smem + tile64::UX),
            reinterpret_cast<C<double> *>(smem + tile64::UY),
            reinterpret_cast<double *>(smem + tile64::PHI), top, bottom, left, right);
        __syncthreads();
    }
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)(ix0 + r) * N + iy0 + c;
    const FullLoadTile64 ld(smem_addr(smem), r, c, s, pos, n);
    M3<double> nx, ny;
    H3<double> phin;
    leapfrog_full_core<double, false>(ld, cf, nx, ny, phin);
    if (cf.do_pu) {
        st_h(phi_out, pos, n, phin);
        st_m3(ux_out, pos, n, nx);
        st_m3(uy_out, pos, n, ny);
    }
}

// (128, 1): ptxas then fits the site in 190 registers without spilling (with
// a stated minimum of 2 blocks it used 255 and spilled), and two blocks per SM
// still fit in registers and shared memory
__global__ void __launch_bounds__(128, 1)
    k_leapfrog_tile64(const __grid_constant__ LoadMaps maps, int N, StepCoef<double> cf,
                      double *status, State<double> s, C<double> *ux_out, C<double> *uy_out,
                      double *phi_out) {
    const int tiles_y = N / tile64::Cn;
    tile64_body<false>(&maps, N, blockIdx.x / tiles_y, blockIdx.x % tiles_y, cf, status, s,
                       ux_out, uy_out, phi_out);
}

// The FP64 batch over the TMA tiles: one block per 4 x 32 tile of the
// concatenated tile lists; the block reads its event's descriptor and tensor
// maps from global memory.
__global__ void __launch_bounds__(128, 1)
    k_leapfrog_tile64_batch(const BatchEvent<double> *__restrict__ evs, int n_events,
                            const int *__restrict__ tile_begin, const LoadMaps *__restrict__ maps,
                            double *status) {
    const int t = blockIdx.x;
    int lo = 0, hi = n_events - 1;  // last e with tile_begin[e] <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tile_begin + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    const BatchEvent<double> &E = evs[lo];
    if (!E.active) return;
    const int N = E.N, tiles_y = N / tile64::Cn, local = t - __ldg(tile_begin + lo);
    tile64_body<true>(maps + 2 * lo + E.map_sel, N, local / tiles_y, local % tiles_y, E.cf,
                      status, E.s, E.ux_out, E.uy_out, E.phi_out);
}

// ---------------------------------------------------------------------------
// Batched events: one persistent launch advances every site of every event in
// a batch (lattices of different N, each a multiple of 32) by one step. The
// tile list of the batch is the concatenation of the events' tiles (32 sites
// along y x TX rows along x, one thread per site); event e owns tiles [tile_begin[e],
// tile_begin[e+1]). Each block takes tiles blockIdx.x, blockIdx.x + gridDim.x,
// ... and finds the owning event by binary search over tile_begin held in
// shared memory. Per-event pointers and coefficients of this step come from a
// descriptor table in device memory, so a captured sequence of launches stays
// valid when the events' buffers swap roles between runs.
// ---------------------------------------------------------------------------
template <int TX, typename T>
// one thread per site and up to 255 registers in both forms: 256 threads per SM
__global__ void __launch_bounds__(32 * TX, 8 / TX)
    k_leapfrog_batch(const BatchEvent<T> *__restrict__ evs, int n_events,
                     const int *__restrict__ tile_begin, int total_tiles) {
    // the step's descriptors, then tile_begin[n_events + 1], in shared memory
    extern __shared__ __align__(16) unsigned char s_raw[];
    BatchEvent<T> *s_ev = reinterpret_cast<BatchEvent<T> *>(s_raw);
    int *s_begin = reinterpret_cast<int *>(s_ev + n_events);
    {
        const int words = n_events * (int)(sizeof(BatchEvent<T>) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(evs);
        int *dst = reinterpret_cast<int *>(s_ev);
        for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
    }
    for (int e = threadIdx.x; e <= n_events; e += blockDim.x) s_begin[e] = tile_begin[e];
    __syncthreads();
    const int ly = threadIdx.x & 31, lx = threadIdx.x >> 5;
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        int lo = 0, hi = n_events - 1;  // last e with s_begin[e] <= t
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_begin[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchEvent<T> &E = s_ev[lo];
        if (!E.active) continue;
        const int local = t - s_begin[lo];
        const int tiles_y = E.N >> 5;
        const int ty = local % tiles_y, tx = local / tiles_y;
        // the same per-site code as the single-event kernels of this precision
        if constexpr (sizeof(T) == 4)
            leapfrog_pair_site(E.N, tx * TX + lx, ty * 32 + ly, E.s, E.ux_out, E.uy_out,
                               E.phi_out, E.cf);
        else
            leapfrog_full_site<T, false>(E.N, tx * TX + lx, ty * 32 + ly, E.s, E.ux_out,
                                         E.uy_out, E.phi_out, E.cf);
    }
}

template <typename T>
size_t batch_smem(int n_events) {
    return sizeof(BatchEvent<T>) * n_events + sizeof(int) * (n_events + 1);
}

// shared memory of the FP32 TMA batch kernel: two stages, the barriers, the
// descriptors and tile prefix sums, alignment slack
size_t tile_batch_smem(int n_events) {
    return 2 * (size_t)tile::STAGE + 64 + batch_smem<float>(n_events) + 128;
}


template <typename T>
int batch_tile_rows(int variant) {
    if (variant == batch_plain_variants<T>()) return sizeof(T) == 4 ? tile::R : tile64::R;
    return variant == 0 ? 2 : (variant == 1 ? 4 : 8);
}

template <typename T>
const void *batch_kernel(int variant) {
    switch (variant) {
        case 0: return (const void *)k_leapfrog_batch<2, T>;
        case 1: return (const void *)k_leapfrog_batch<4, T>;
        default: return (const void *)k_leapfrog_batch<8, T>;
    }
}

template <typename T>
int batch_max_blocks_per_sm(int variant, int n_events) {
    int nb = 0;
    if (variant == batch_plain_variants<T>()) {
        if constexpr (sizeof(T) == 4) {
            const size_t smem = tile_batch_smem(n_events);
            if (smem > 227 * 1024) return 0;  // too many events for the descriptors
            cudaFuncSetAttribute(k_leapfrog_tile_batch,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_leapfrog_tile_batch, 256, smem);
            return nb > 1 ? 1 : nb;  // persistent: one block per SM
        } else {
            cudaFuncSetAttribute(k_leapfrog_tile64_batch,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, tile64::SMEM);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_leapfrog_tile64_batch, 128,
                                                          tile64::SMEM);
            return nb > 0 ? 1 : 0;  // one block per tile: the grid is the tile count
        }
    }
    const int threads = 32 * batch_tile_rows<T>(variant);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_kernel<T>(variant), threads,
                                                  batch_smem<T>(n_events));
    return nb;
}

template <typename T>
void launch_leapfrog_batch(const BatchEvent<T> *d_evs, int n_events, const int *d_tile_begin,
                           int total_tiles, int variant, int grid, const LoadMaps *d_maps,
                           double *status, cudaStream_t st) {
    if (variant == batch_plain_variants<T>()) {
        if constexpr (sizeof(T) == 4) {
            const size_t smem = tile_batch_smem(n_events);
            // imag = 4: the byte offset of a link's imaginary part
            k_leapfrog_tile_batch<<<grid < total_tiles ? grid : total_tiles, 256, smem, st>>>(
                d_evs, n_events, d_tile_begin, total_tiles, d_maps, status, 4u);
        } else {
            k_leapfrog_tile64_batch<<<total_tiles, 128, tile64::SMEM, st>>>(
                d_evs, n_events, d_tile_begin, d_maps, status);
        }
        return;
    }
    const size_t smem = batch_smem<T>(n_events);
    switch (variant) {
        case 0:
            k_leapfrog_batch<2, T><<<grid, 64, smem, st>>>(d_evs, n_events, d_tile_begin,
                                                           total_tiles);
            break;
        case 1:
            k_leapfrog_batch<4, T><<<grid, 128, smem, st>>>(d_evs, n_events, d_tile_begin,
                                                            total_tiles);
            break;
        default:
            k_leapfrog_batch<8, T><<<grid, 256, smem, st>>>(d_evs, n_events, d_tile_begin,
                                                            total_tiles);
            break;
    }
}

template int batch_tile_rows<float>(int);
template int batch_tile_rows<double>(int);
template int batch_max_blocks_per_sm<float>(int, int);
template int batch_max_blocks_per_sm<double>(int, int);
template void launch_leapfrog_batch<float>(const BatchEvent<float> *, int, const int *, int,
                                           int, int, const LoadMaps *, double *, cudaStream_t);
template void launch_leapfrog_batch<double>(const BatchEvent<double> *, int, const int *, int,
                                            int, int, const LoadMaps *, double *, cudaStream_t);

template <typename T>
void launch_leapfrog_site(const EventGeom *d_ev, int N, const State<T> &s,
                          C<T> *ux_out, C<T> *uy_out, T *phi_out,
                          const StepCoef<T> &cf, bool reunit, cudaStream_t st);

bool encode_tiled_3d(CUtensorMap *map, void *base, CUtensorMapDataType type, size_t esize,
                     uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1,
                     uint32_t b2) {
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {d0 * esize, d0 * d1 * esize};
    const cuuint32_t box[3] = {b0, b1, b2};
    const cuuint32_t unit[3] = {1, 1, 1};
    return encode(map, type, 3, base, dims, strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <>
bool encode_step_maps<float>(int N, const State<float> &s, LoadMaps *m) {
    using namespace tile;
    const uint64_t n = (uint64_t)N;
    const auto U64 = CU_TENSOR_MAP_DATA_TYPE_UINT64, U32 = CU_TENSOR_MAP_DATA_TYPE_UINT32;
    return encode_tiled_3d(&m->ux, s.ux, U64, 8, n, n, 9, UC, UR, 9) &&
           encode_tiled_3d(&m->uy, s.uy, U64, 8, n, n, 9, UC, UR, 9) &&
           encode_tiled_3d(&m->phi, s.phi, U32, 4, n, n, 9, PC, PR, 9) &&
           encode_tiled_3d(&m->e1, s.e1, U32, 4, n, n, 8, Cn, R, 8) &&
           encode_tiled_3d(&m->e2, s.e2, U32, 4, n, n, 8, Cn, R, 8) &&
           encode_tiled_3d(&m->pi, s.pi, U32, 4, n, n, 9, Cn, R, 9);
}

template <>
bool encode_step_maps<double>(int N, const State<double> &s, LoadMaps *m) {
    using namespace tile64;
    const uint64_t n = (uint64_t)N;
    const auto U64 = CU_TENSOR_MAP_DATA_TYPE_UINT64;
    // a complex link entry is two 8-byte words
    return encode_tiled_3d(&m->ux, s.ux, U64, 8, 2 * n, n, 9, 2 * UC, UR, 9) &&
           encode_tiled_3d(&m->uy, s.uy, U64, 8, 2 * n, n, 9, 2 * UC, UR, 9) &&
           encode_tiled_3d(&m->phi, s.phi, U64, 8, n, n, 9, PC, PR, 9) &&
           encode_tiled_3d(&m->e1, s.e1, U64, 8, n, n, 8, Cn, R, 8) &&
           encode_tiled_3d(&m->e2, s.e2, U64, 8, n, n, 8, Cn, R, 8) &&
           encode_tiled_3d(&m->pi, s.pi, U64, 8, n, n, 9, Cn, R, 9);
}

namespace {

// The FP32 form's step kernel: the TMA-staged tile kernel unless
// IPG_FP32_KERNEL=pair selects the plain-load kernel (both run the same
// per-site code and give the same bits).
bool use_tile_kernel() {
    static const bool tile = [] {
        const char *e = std::getenv("IPG_FP32_KERNEL");
        return !(e && std::strcmp(e, "pair") == 0);
    }();
    return tile;
}

// false if a tensor map could not be encoded (nothing launched)
bool launch_leapfrog_tile(int N, const State<float> &s, C<float> *ux_out, C<float> *uy_out,
                          float *phi_out, const StepCoef<float> &cf, double *status,
                          cudaStream_t st) {
    using namespace tile;
    LoadMaps m;
    if (!encode_step_maps<float>(N, s, &m)) return false;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_leapfrog_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    const int tiles = (N / R) * (N / Cn);
    // imag = 4: the byte offset of a link's imaginary part
    k_leapfrog_tile<<<tiles < sms ? tiles : sms, 256, SMEM, st>>>(m, N, cf, status, 4u, s, ux_out,
                                                                  uy_out, phi_out);
    return true;
}

// The FP64 form's step kernel: the TMA-staged tile kernel unless
// IPG_FP64_KERNEL=site selects the plain-load kernel (same per-site code).
bool use_tile64_kernel() {
    static const bool tile = [] {
        const char *e = std::getenv("IPG_FP64_KERNEL");
        return !(e && std::strcmp(e, "site") == 0);
    }();
    return tile;
}

bool launch_leapfrog_tile64(int N, const State<double> &s, C<double> *ux_out, C<double> *uy_out,
                            double *phi_out, const StepCoef<double> &cf, double *status,
                            cudaStream_t st) {
    using namespace tile64;
    LoadMaps m;
    if (!encode_step_maps<double>(N, s, &m)) return false;
    cudaFuncSetAttribute(k_leapfrog_tile64, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    k_leapfrog_tile64<<<(N / R) * (N / Cn), 128, SMEM, st>>>(m, N, cf, status, s, ux_out, uy_out,
                                                               phi_out);
    return true;
}

}  // namespace

template <typename T>
void launch_leapfrog(const EventGeom *d_ev, int N, const State<T> &s,
                     C<T> *ux_out, C<T> *uy_out, T *phi_out,
                     const StepCoef<T> &cf, bool reunit, cudaStream_t st, double *status) {
    // FP64 runs one thread per site: at 512^2 it takes 97 us a step against
    // 108 us for the direction split (both FP64-pipe and latency bound at one
    // 256-thread block per SM). FP32 runs both directions of a site in the
    // two lanes of packed FP32 instructions, from shared-memory tiles filled
    // by TMA (k_leapfrog_tile) or from plain loads (k_leapfrog_pair).
    if constexpr (sizeof(T) == 4) {
        if (N >= 32) {
            // N is a power of two >= 32: the tiles cover the lattice exactly
            (void)reunit;
            if (use_tile_kernel() &&
                launch_leapfrog_tile(N, s, ux_out, uy_out, phi_out, cf, status, st))
                return;
            k_leapfrog_pair<<<dim3(N / 32, N / 8), 256, 0, st>>>(d_ev, s, ux_out, uy_out, phi_out,
                                                                 cf);
            return;
        }
    }
    if constexpr (sizeof(T) == 8) {
        if (N >= 32 && !reunit && use_tile64_kernel() &&
            launch_leapfrog_tile64(N, s, ux_out, uy_out, phi_out, cf, status, st))
            return;
    }
    launch_leapfrog_site(d_ev, N, s, ux_out, uy_out, phi_out, cf, reunit, st);
}

void launch_leapfrog_into(const EventGeom *d_ev, int N, const State<double> &in,
                          const State<double> &out, const StepCoef<double> &cf, cudaStream_t st) {
    const size_t n = (size_t)N * N;
    // the step writes E and pi only when it updates them
    const bool copy_e = !cf.do_pe || N < 32 || !use_tile64_kernel();
    if (copy_e) {
        cudaMemcpyAsync(out.e1, in.e1, 8 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(out.e2, in.e2, 8 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(out.pi, in.pi, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    // links and phi from `in`; E and pi read from `in` (TMA) or, after the
    // copy, updated in place in `out`
    State<double> s = in;
    s.e1 = out.e1;
    s.e2 = out.e2;
    s.pi = out.pi;
    if (!copy_e) {
        using namespace tile64;
        const uint64_t nn = (uint64_t)N;
        const auto U64 = CU_TENSOR_MAP_DATA_TYPE_UINT64;
        LoadMaps m;
        const bool ok =
            encode_tiled_3d(&m.ux, in.ux, U64, 8, 2 * nn, nn, 9, 2 * UC, UR, 9) &&
            encode_tiled_3d(&m.uy, in.uy, U64, 8, 2 * nn, nn, 9, 2 * UC, UR, 9) &&
            encode_tiled_3d(&m.phi, in.phi, U64, 8, nn, nn, 9, PC, PR, 9) &&
            encode_tiled_3d(&m.e1, in.e1, U64, 8, nn, nn, 8, Cn, R, 8) &&
            encode_tiled_3d(&m.e2, in.e2, U64, 8, nn, nn, 8, Cn, R, 8) &&
            encode_tiled_3d(&m.pi, in.pi, U64, 8, nn, nn, 9, Cn, R, 9);
        if (ok) {
            cudaFuncSetAttribute(k_leapfrog_tile64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SMEM);
            k_leapfrog_tile64<<<(N / R) * (N / Cn), 128, SMEM, st>>>(m, N, cf, nullptr, s, out.ux,
                                                                       out.uy, out.phi);
            return;
        }
        cudaMemcpyAsync(out.e1, in.e1, 8 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(out.e2, in.e2, 8 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(out.pi, in.pi, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    }
    launch_leapfrog_site<double>(d_ev, N, s, out.ux, out.uy, out.phi, cf, false, st);
}

// one thread per site (lattices smaller than 32 sites per side)
template <typename T>
void launch_leapfrog_site(const EventGeom *d_ev, int N, const State<T> &s,
                          C<T> *ux_out, C<T> *uy_out, T *phi_out,
                          const StepCoef<T> &cf, bool reunit, cudaStream_t st) {
    dim3 block(32, 4);
    dim3 grid((N + 31) / 32, (N + 3) / 4);
    if constexpr (sizeof(T) == 4) {
        // FP32 bulk form: deviation storage, reunitarised every step
        (void)reunit;
        k_leapfrog_dev<T><<<grid, block, 0, st>>>(d_ev, s, ux_out, uy_out,
                                                  phi_out, cf);
    } else {
        if (reunit)
            k_leapfrog<T, true><<<grid, block, 0, st>>>(d_ev, s, ux_out, uy_out,
                                                       phi_out, cf);
        else
            k_leapfrog<T, false><<<grid, block, 0, st>>>(d_ev, s, ux_out, uy_out,
                                                        phi_out, cf);
    }
}

// The E and pi half of a step reversed. S_e with dt_pe negated (cst and cdt
// change sign) gives E = TL(E' - cst t - cdt i[U phi(+d) U^dag, phi]) and
// pi = pi' - cdt br, the inverse of the forward update up to rounding, and
// the step's TMA tile kernel computes exactly that with the U and phi update
// switched off: links and phi from `cur` (already recovered), E' and pi' from
// `nxt`, E and pi written to `cur`. Without tiles, k_inv_se.
template <typename T>
void launch_inverse_se(int N, const State<T> &nxt, const State<T> &cur, const StepCoef<double> &cf,
                       cudaStream_t st) {
    const size_t n = (size_t)N * N;
    if constexpr (sizeof(T) == 8) {
        if (cf.do_pe && N >= 32 && use_tile64_kernel()) {
            using namespace tile64;
            const uint64_t nn = (uint64_t)N;
            const auto U64 = CU_TENSOR_MAP_DATA_TYPE_UINT64;
            LoadMaps m;
            const bool ok =
                encode_tiled_3d(&m.ux, cur.ux, U64, 8, 2 * nn, nn, 9, 2 * UC, UR, 9) &&
                encode_tiled_3d(&m.uy, cur.uy, U64, 8, 2 * nn, nn, 9, 2 * UC, UR, 9) &&
                encode_tiled_3d(&m.phi, cur.phi, U64, 8, nn, nn, 9, PC, PR, 9) &&
                encode_tiled_3d(&m.e1, nxt.e1, U64, 8, nn, nn, 8, Cn, R, 8) &&
                encode_tiled_3d(&m.e2, nxt.e2, U64, 8, nn, nn, 8, Cn, R, 8) &&
                encode_tiled_3d(&m.pi, nxt.pi, U64, 8, nn, nn, 9, Cn, R, 9);
            if (ok) {
                StepCoef<double> rc = cf;
                rc.dt_pe = -cf.dt_pe;
                rc.do_pu = 0;
                set_derived(rc);
                cudaFuncSetAttribute(k_leapfrog_tile64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     SMEM);
                k_leapfrog_tile64<<<(N / R) * (N / Cn), 128, SMEM, st>>>(m, N, rc, nullptr, cur,
                                                                           nullptr, nullptr, nullptr);
                return;
            }
        }
    }
    k_inv_se<T><<<dim3((unsigned)((n + 127) / 128), 3), 128, 0, st>>>(N, nxt, cur, cf);
}
template void launch_inverse_se<double>(int, const State<double> &, const State<double> &,
                                        const StepCoef<double> &, cudaStream_t);

template void launch_leapfrog<double>(const EventGeom *, int, const State<double> &,
                                      C<double> *, C<double> *, double *,
                                      const StepCoef<double> &, bool, cudaStream_t, double *);
template void launch_leapfrog<float>(const EventGeom *, int, const State<float> &, C<float> *,
                                     C<float> *, float *, const StepCoef<float> &, bool,
                                     cudaStream_t, double *);

}  // namespace ipg
