// Stencil helpers shared by the leapfrog step (evolve.cu) and its reverse
// sweep (adjoint.cu): full-matrix neighbour loads from the global planes with
// the reference's clamped edges, and the time reversal of the E and pi
// update.
#pragma once

#include "fields.cuh"

namespace ipg {

template <typename T>
__device__ __forceinline__ H3<T> i_antiherm_mul(const M3<T> &p,
                                                const M3<T> &q) {
    M3<T> x = mul(p, q);
    return i_antiherm(x);
}

// Field selectors of the link loaders: a link (or lane of a packed link
// pair) comes from Ux (kLx) or Uy (kLy) at a neighbour offset (dx, dy).
constexpr int kLx = 0, kLy = 1;

// Full-matrix loads from the global planes, neighbours clamped at the lattice
// edge (Lattice.cpp:19-28); E and pi are site-local and written back in place.
template <typename T>
struct FullLoadGlobal {
    const State<T> &s;
    size_t pos, n;
    long ox[3], oy[3];  // index offsets of dx (dy) = -1, 0, +1, clamped
    __device__ __forceinline__ FullLoadGlobal(const State<T> &s_, int N, int ix, int iy)
        : s(s_), pos((size_t)ix * N + iy), n((size_t)N * N) {
        ox[0] = ix > 0 ? -(long)N : 0;
        ox[1] = 0;
        ox[2] = ix + 1 < N ? N : 0;
        oy[0] = iy > 0 ? -1 : 0;
        oy[1] = 0;
        oy[2] = iy + 1 < N ? 1 : 0;
    }
    template <int F, int DX, int DY>
    __device__ __forceinline__ M3<T> link() const {
        return ld_m3(F == kLy ? s.uy : s.ux, pos + ox[DX + 1] + oy[DY + 1], n);
    }
    template <int DX, int DY>
    __device__ __forceinline__ H3<T> phi() const {
        return ld_h(s.phi, pos + ox[DX + 1] + oy[DY + 1], n);
    }
    __device__ __forceinline__ H3<T> pi() const { return ld_h(s.pi, pos, n); }
    __device__ __forceinline__ H3<T> e1() const { return ld_h8(s.e1, pos, n); }
    __device__ __forceinline__ H3<T> e2() const { return ld_h8(s.e2, pos, n); }
    __device__ __forceinline__ void put_e(const H3<T> &a, const H3<T> &b) const {
        st_h8(s.e1, pos, n, a);
        st_h8(s.e2, pos, n, b);
    }
    __device__ __forceinline__ void put_pi(const H3<T> &h) const { st_h(s.pi, pos, n, h); }
};

// Time reversal of the E and pi half of a step (the inverse of S_e) at one
// site, for one of three thread roles (0: E1, 1: E2, 2: pi): with U and phi
// of the step's input already recovered in `cur`,
//   pi = pi' - cdt br(U, phi),   E_d = E_d' - TL(cst t_d + cdt i[U_d phi(+d) U_d^dag, phi])
// with the forward step's staple and transport expressions
// (Evolution.cpp:117-293), each role loading only the links and phi its own
// field needs.
template <typename T>
__device__ __forceinline__ void inverse_se_role(int N, int role, size_t p, const State<T> &nxt,
                                                const State<T> &cur, T cst, T cdt) {
    const FullLoadGlobal<T> ld(cur, N, (int)(p / N), (int)(p % N));
    const size_t pos = ld.pos, n = ld.n;
    if (role == 2) {
        H3<T> pi = ld_h(nxt.pi, pos, n);
        H3<T> br = conj_h(ld.template link<kLx, 0, 0>(), ld.template phi<1, 0>());
        h_add(br, conj_h(ld.template link<kLy, 0, 0>(), ld.template phi<0, 1>()));
        h_add(br, conj_h_dag(ld.template link<kLx, -1, 0>(), ld.template phi<-1, 0>()));
        h_add(br, conj_h_dag(ld.template link<kLy, 0, -1>(), ld.template phi<0, -1>()));
        h_axpy(br, T(-4.), ld.template phi<0, 0>());
        h_axpy(pi, -cdt, br);
        st_h(cur.pi, pos, n, pi);
        return;
    }
    H3<T> e = ld_h8(role == 0 ? nxt.e1 : nxt.e2, pos, n);
    // plaquette U12 = Ux Uy(x+1) Ux(y+1)^dag Uy^dag (Evolution.cpp:228-232)
    H3<T> h12;
    {
        M3<T> a = mul(ld.template link<kLx, 0, 0>(), ld.template link<kLy, 1, 0>());
        M3<T> b = mul(ld.template link<kLy, 0, 0>(), ld.template link<kLx, 0, 1>());
        h12 = i_antiherm(mul_nd(a, b));
    }
    H3<T> t, ph;
    if (role == 0) {
        // E1: U12 + U1m2 - h.c. (234-257)
        M3<T> pp = mul_nd(ld.template link<kLx, 0, 0>(), ld.template link<kLy, 1, -1>());
        M3<T> q = mul_dn(ld.template link<kLx, 0, -1>(), ld.template link<kLy, 0, -1>());
        t = h12;
        h_add(t, i_antiherm_mul(pp, q));
        ph = conj_h(ld.template link<kLx, 0, 0>(), ld.template phi<1, 0>());
    } else {
        // E2: U12^dag + U2m1 - h.c. (240-244, 266-275)
        M3<T> pp = mul_nd(ld.template link<kLy, 0, 0>(), ld.template link<kLx, -1, 1>());
        M3<T> q = mul_dn(ld.template link<kLy, -1, 0>(), ld.template link<kLx, -1, 0>());
        t = i_antiherm_mul(pp, q);
        h_axpy(t, T(-1), h12);
        ph = conj_h(ld.template link<kLy, 0, 0>(), ld.template phi<0, 1>());
    }
    h_traceless(t);
    H3<T> d = {};
    h_axpy(d, cst, t);
    h_axpy(d, cdt, i_commutator(ph, ld.template phi<0, 0>()));
    h_traceless(d);
    h_axpy(e, T(-1.), d);
    h_traceless(e);
    st_h8(role == 0 ? cur.e1 : cur.e2, pos, n, e);
}

}  // namespace ipg
