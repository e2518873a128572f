// Reverse mode (adjoint) of the FP64 leapfrog evolution and of T^tautau.
//
// The reference has no derivative code; these kernels give the gradient of a
// loss built from T^tautau at the final time (total transverse energy E_T and
// a T^tautau-weighted eccentricity) with respect to the tau = 0 fields.
//
// Conventions. A complex field A has the adjoint A_bar = dL/dRe A + i dL/dIm A,
// so dL = Re tr(A_bar^dag dA). Products C = A B pass A_bar += C_bar B^dag and
// B_bar += A^dag C_bar. Hermitian fields (phi, pi) and traceless Hermitian
// ones (E1, E2) keep full-matrix adjoint buffers; only their Hermitian
// (traceless) part is meaningful and it is taken where an adjoint is
// consumed. Adjoint buffers hold 18 real planes per field (real and imaginary
// parts of the 9 entries apart; see adj_planes).
//
// One leapfrog step (evolve.cu, Evolution.cpp:35-293) is S = S_u o S_e:
//   S_e: E_d' = TL(E_d + cst (AH-plaquette + AH-staple)_d + cdt i[U_d phi(+d) U_d^dag, phi])
//        pi'  = pi + cdt sum_d (U_d phi(+d) U_d^dag + U_d(-d)^dag phi(-d) U_d(-d) - 2 phi)
//   S_u: phi' = phi + c2 pi',   U_d' = T2(i c E_d') U_d,  T2(X) = 1 + X + X^2/2
// with cst = tau dtau / (2 g^2), cdt = dtau / tau, c = g^2 dtau / (tau + dtau/2),
// c2 = (tau + dtau/2) dtau. Its vector-Jacobian product is k_adj_su (local)
// followed by k_adj_se (it scatters into neighbouring links and phi with
// FP64 atomics, so the summation order, not the result, varies between runs).
// The step is inverted exactly in exact arithmetic: U and phi by k_inv_su
// (or k_inv_adj_su, fused with the S_u adjoint), then E and pi by S_e with
// dtau negated (launch_inverse_se in evolve.cu: the forward step's tile
// kernel with the U/phi update off). This is the time reversal used to walk
// back between checkpoints.
#include <cstdint>

#include "expm.cuh"
#include "fields.cuh"
#include "ipg_internal.h"
#include "philox.cuh"

namespace ipg {

namespace {

using Md = M3<double>;

__device__ __forceinline__ size_t at(int N, int i, int j) { return (size_t)i * N + j; }

template <typename T>
__device__ __forceinline__ M3<T> herm(const M3<T> &a) {
    M3<T> r;
#pragma unroll
    for (int x = 0; x < 3; x++)
#pragma unroll
        for (int y = 0; y < 3; y++)
            r.m[3 * x + y] = {T(0.5) * (a.m[3 * x + y].r + a.m[3 * y + x].r),
                              T(0.5) * (a.m[3 * x + y].i - a.m[3 * y + x].i)};
    return r;
}

// s * i * a
template <typename T>
__device__ __forceinline__ M3<T> times_i(const M3<T> &a, T s) {
    M3<T> r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = {-s * a.m[k].i, s * a.m[k].r};
    return r;
}

template <typename T>
__device__ __forceinline__ M3<T> sc(const M3<T> &a, T s) { return scaled(a, s); }

template <typename T>
__device__ __forceinline__ M3<T> addm(const M3<T> &a, const M3<T> &b) {
    M3<T> r = a;
    add_to(r, b);
    return r;
}

// i [A, B]
template <typename T>
__device__ __forceinline__ M3<T> icomm(const M3<T> &a, const M3<T> &b) {
    return times_i(minus(mul(a, b), mul(b, a)), T(1.));
}

template <typename T>
__device__ __forceinline__ M3<T> ld_herm(const T *p, size_t pos, size_t n) {
    return from_h(ld_h(p, pos, n));
}
template <typename T>
__device__ __forceinline__ M3<T> ld_herm8(const T *p, size_t pos, size_t n) {
    return from_h(ld_h8(p, pos, n));
}

// A link of a stored state: full matrices in FP64; the FP32 adjoint works on
// the FP32 bulk form's states, which hold the deviation W = U - 1, so the
// identity is added back (its products with adjoints need no deviation form)
template <typename T>
__device__ __forceinline__ M3<T> ld_link(const C<T> *p, size_t pos, size_t n) {
    M3<T> u = ld_m3(p, pos, n);
    if constexpr (sizeof(T) == 4) {
        u.m[0].r += T(1);
        u.m[4].r += T(1);
        u.m[8].r += T(1);
    }
    return u;
}

// Adjoint buffers hold 9 complex entries a site as 18 planes of n doubles:
// the real part of entry k in plane 2k, its imaginary part in plane 2k+1
// (the buffer is typed as 9 complex planes and has the same size). A warp's
// FP64 atomics on one plane then fill whole 32-byte sectors.
template <typename T>
__device__ __forceinline__ T *adj_planes(C<T> *buf) {
    return reinterpret_cast<T *>(buf);
}
template <typename T>
__device__ __forceinline__ const T *adj_planes(const C<T> *buf) {
    return reinterpret_cast<const T *>(buf);
}

template <typename T>
__device__ __forceinline__ void atomic_add_m(C<T> *buf, size_t pos, size_t n,
                                             const M3<T> &a) {
    T *b = adj_planes(buf);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        atomicAdd(&b[(2 * k) * n + pos], a.m[k].r);
        atomicAdd(&b[(2 * k + 1) * n + pos], a.m[k].i);
    }
}

template <typename T>
__device__ __forceinline__ M3<T> ld_adj(const C<T> *buf, size_t pos, size_t n) {
    const T *b = adj_planes(buf);
    M3<T> m;
#pragma unroll
    for (int k = 0; k < 9; k++) m.m[k] = {b[(2 * k) * n + pos], b[(2 * k + 1) * n + pos]};
    return m;
}

template <typename T>
__device__ __forceinline__ void st_adj(C<T> *buf, size_t pos, size_t n, const M3<T> &m) {
    T *b = adj_planes(buf);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        b[(2 * k) * n + pos] = m.m[k].r;
        b[(2 * k + 1) * n + pos] = m.m[k].i;
    }
}

// During the reverse sweep the adjoints of the Hermitian fields keep only
// their Hermitian part, the part the loss sees: phi and pi as 9 planes (d0 d1
// d2, re/im of the 01, 02, 12 entries), E1 and E2 as their traceless part in
// 8 planes (d0 d1 and the off-diagonals; d2 = -d0 - d1). A contribution M is
// added as its (traceless) Hermitian part. k_adj_project expands them to full
// matrices (split planes) at the end of the sweep.
template <typename T>
__device__ __forceinline__ H3<T> ld_h9a(const C<T> *buf, size_t pos, size_t n) {
    const T *b = adj_planes(buf);
    H3<T> h;
    h.d0 = b[pos];
    h.d1 = b[n + pos];
    h.d2 = b[2 * n + pos];
    h.o01 = {b[3 * n + pos], b[4 * n + pos]};
    h.o02 = {b[5 * n + pos], b[6 * n + pos]};
    h.o12 = {b[7 * n + pos], b[8 * n + pos]};
    return h;
}

template <typename T>
__device__ __forceinline__ void st_h9a(C<T> *buf, size_t pos, size_t n, const H3<T> &h) {
    T *b = adj_planes(buf);
    b[pos] = h.d0;
    b[n + pos] = h.d1;
    b[2 * n + pos] = h.d2;
    b[3 * n + pos] = h.o01.r;
    b[4 * n + pos] = h.o01.i;
    b[5 * n + pos] = h.o02.r;
    b[6 * n + pos] = h.o02.i;
    b[7 * n + pos] = h.o12.r;
    b[8 * n + pos] = h.o12.i;
}

template <typename T>
__device__ __forceinline__ H3<T> ld_h8a(const C<T> *buf, size_t pos, size_t n) {
    const T *b = adj_planes(buf);
    H3<T> h;
    h.d0 = b[pos];
    h.d1 = b[n + pos];
    h.d2 = -(h.d0 + h.d1);
    h.o01 = {b[2 * n + pos], b[3 * n + pos]};
    h.o02 = {b[4 * n + pos], b[5 * n + pos]};
    h.o12 = {b[6 * n + pos], b[7 * n + pos]};
    return h;
}

template <typename T>
__device__ __forceinline__ void st_h8a(C<T> *buf, size_t pos, size_t n, const H3<T> &h) {
    T *b = adj_planes(buf);
    b[pos] = h.d0;
    b[n + pos] = h.d1;
    b[2 * n + pos] = h.o01.r;
    b[3 * n + pos] = h.o01.i;
    b[4 * n + pos] = h.o02.r;
    b[5 * n + pos] = h.o02.i;
    b[6 * n + pos] = h.o12.r;
    b[7 * n + pos] = h.o12.i;
}

// Hermitian part (M + M^dag) / 2
template <typename T>
__device__ __forceinline__ H3<T> herm_part(const M3<T> &m) {
    H3<T> h;
    h.d0 = m.m[0].r;
    h.d1 = m.m[4].r;
    h.d2 = m.m[8].r;
    h.o01 = {T(0.5) * (m.m[1].r + m.m[3].r), T(0.5) * (m.m[1].i - m.m[3].i)};
    h.o02 = {T(0.5) * (m.m[2].r + m.m[6].r), T(0.5) * (m.m[2].i - m.m[6].i)};
    h.o12 = {T(0.5) * (m.m[5].r + m.m[7].r), T(0.5) * (m.m[5].i - m.m[7].i)};
    return h;
}

template <typename T>
__device__ __forceinline__ void atomic_add_h9a(C<T> *buf, size_t pos, size_t n,
                                               const M3<T> &m) {
    const H3<T> h = herm_part(m);
    T *b = adj_planes(buf);
    atomicAdd(&b[pos], h.d0);
    atomicAdd(&b[n + pos], h.d1);
    atomicAdd(&b[2 * n + pos], h.d2);
    atomicAdd(&b[3 * n + pos], h.o01.r);
    atomicAdd(&b[4 * n + pos], h.o01.i);
    atomicAdd(&b[5 * n + pos], h.o02.r);
    atomicAdd(&b[6 * n + pos], h.o02.i);
    atomicAdd(&b[7 * n + pos], h.o12.r);
    atomicAdd(&b[8 * n + pos], h.o12.i);
}

template <typename T>
__device__ __forceinline__ void atomic_add_h8a(C<T> *buf, size_t pos, size_t n,
                                               const M3<T> &m) {
    const H3<T> h = herm_part(m);
    const T t = (h.d0 + h.d1 + h.d2) / T(3.);
    T *b = adj_planes(buf);
    atomicAdd(&b[pos], h.d0 - t);
    atomicAdd(&b[n + pos], h.d1 - t);
    atomicAdd(&b[2 * n + pos], h.o01.r);
    atomicAdd(&b[3 * n + pos], h.o01.i);
    atomicAdd(&b[4 * n + pos], h.o02.r);
    atomicAdd(&b[5 * n + pos], h.o02.i);
    atomicAdd(&b[6 * n + pos], h.o12.r);
    atomicAdd(&b[7 * n + pos], h.o12.i);
}

// T2(X) = 1 + X + X^2 / 2
template <typename T>
__device__ __forceinline__ M3<T> taylor2(const M3<T> &x) {
    M3<T> r = mul(x, x);
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = {T(0.5) * r.m[k].r + x.m[k].r, T(0.5) * r.m[k].i + x.m[k].i};
    r.m[0].r += T(1.);
    r.m[4].r += T(1.);
    r.m[8].r += T(1.);
    return r;
}

// inverse of a 3x3 complex matrix (adjugate / determinant)
template <typename T>
__device__ __forceinline__ M3<T> inverse3(const M3<T> &a) {
    auto e = [&](int r, int c) { return a.m[3 * r + c]; };
    auto sub = [](C<T> x, C<T> y) { return C<T>{x.r - y.r, x.i - y.i}; };
    M3<T> adj;
    adj.m[0] = sub(cmul(e(1, 1), e(2, 2)), cmul(e(1, 2), e(2, 1)));
    adj.m[1] = sub(cmul(e(0, 2), e(2, 1)), cmul(e(0, 1), e(2, 2)));
    adj.m[2] = sub(cmul(e(0, 1), e(1, 2)), cmul(e(0, 2), e(1, 1)));
    adj.m[3] = sub(cmul(e(1, 2), e(2, 0)), cmul(e(1, 0), e(2, 2)));
    adj.m[4] = sub(cmul(e(0, 0), e(2, 2)), cmul(e(0, 2), e(2, 0)));
    adj.m[5] = sub(cmul(e(0, 2), e(1, 0)), cmul(e(0, 0), e(1, 2)));
    adj.m[6] = sub(cmul(e(1, 0), e(2, 1)), cmul(e(1, 1), e(2, 0)));
    adj.m[7] = sub(cmul(e(0, 1), e(2, 0)), cmul(e(0, 0), e(2, 1)));
    adj.m[8] = sub(cmul(e(0, 0), e(1, 1)), cmul(e(0, 1), e(1, 0)));
    C<T> det = {T(0.), T(0.)};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const C<T> t = cmul(e(0, k), adj.m[3 * k]);
        det.r += t.r;
        det.i += t.i;
    }
    const T d2 = det.r * det.r + det.i * det.i;
    const C<T> inv = {det.r / d2, -det.i / d2};
#pragma unroll
    for (int k = 0; k < 9; k++) adj.m[k] = cmul(adj.m[k], inv);
    return adj;
}

struct StepGeom {
    int N;
    size_t pos, pX, pY, mX, mY, pXmY, mXpY;
};

__device__ __forceinline__ StepGeom step_geom(int N, int ix, int iy) {
    StepGeom g;
    g.N = N;
    const int ixp = min(N - 1, ix + 1), ixm = max(0, ix - 1);
    const int iyp = min(N - 1, iy + 1), iym = max(0, iy - 1);
    g.pos = at(N, ix, iy);
    g.pX = at(N, ixp, iy);
    g.pY = at(N, ix, iyp);
    g.mX = at(N, ixm, iy);
    g.mY = at(N, ix, iym);
    g.pXmY = at(N, ixp, iym);
    g.mXpY = at(N, ixm, iyp);
    return g;
}

}  // namespace

// ---------------------------------------------------------------------------
// time reversal of one step
// ---------------------------------------------------------------------------

// U_d = T2(i c E_d')^{-1} U_d',  phi = phi' - c2 pi'
template <typename T>
__global__ void k_inv_su(int N, State<T> nxt, State<T> cur, T c, T c2) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    for (int d = 0; d < 2; d++) {
        const M3<T> E = ld_herm8(d ? nxt.e2 : nxt.e1, pos, n);
        const M3<T> M = taylor2(times_i(E, c));
        st_m3(d ? cur.uy : cur.ux, pos, n, mul(inverse3(M), ld_m3(d ? nxt.uy : nxt.ux, pos, n)));
    }
    H3<T> phi = ld_h(nxt.phi, pos, n);
    h_axpy(phi, -c2, ld_h(nxt.pi, pos, n));
    st_h(cur.phi, pos, n, phi);
}

// ---------------------------------------------------------------------------
// vector-Jacobian products
// ---------------------------------------------------------------------------

// S_u: reads the adjoints of the step's outputs, leaves the adjoints of its
// inputs (U before the update, phi before, pi' and E' after S_e). `cur` holds
// U, phi of the step's input, `nxt` E' of its output. One thread per site and
// link direction (blockIdx.y): twice the warps of one thread per site, at
// three blocks an SM.
template <typename T>
__global__ void __launch_bounds__(128, 3) k_adj_su(int N, State<T> cur, State<T> nxt, AdjStateT<T> a, T c,
                         T c2) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int d = blockIdx.y;  // the link direction of this thread
    if (d == 0) {
        // pi_bar += c2 phi_bar (phi_bar itself passes through unchanged)
        H3<T> pib = ld_h9a(a.pi, pos, n);
        h_axpy(pib, c2, ld_h9a(a.phi, pos, n));
        st_h9a(a.pi, pos, n, pib);
    }
    {
        C<T> *Ub = d ? a.uy : a.ux;
        C<T> *Eb = d ? a.e2 : a.e1;
        const M3<T> Ubar = ld_adj(Ub, pos, n);
        const M3<T> U = ld_link(d ? cur.uy : cur.ux, pos, n);
        const M3<T> X = times_i(ld_herm8(d ? nxt.e2 : nxt.e1, pos, n), c);
        const M3<T> M = taylor2(X);
        st_adj(Ub, pos, n, mul_dn(M, Ubar));
        const M3<T> Mb = mul_nd(Ubar, U);
        // X_bar = M_bar + (M_bar X^dag + X^dag M_bar) / 2
        M3<T> Xb = Mb;
        add_to(Xb, sc(addm(mul_nd(Mb, X), mul_dn(X, Mb)), T(0.5)));
        // X = i c E  ->  E_bar += Herm(-i c X_bar); stored traceless Hermitian,
        // which is also the adjoint of E before S_e (E' = TL(E + ...))
        H3<T> Eb_ = herm_part(times_i(Xb, -c));
        h_traceless(Eb_);
        h_add(Eb_, ld_h8a(Eb, pos, n));
        st_h8a(Eb, pos, n, Eb_);
    }
}

// The time reversal of S_u fused with its adjoint, for steps reached by
// reversal: U_d = M_d^{-1} U_d' with M_d = T2(i c E_d'), phi = phi' - c2 pi'
// are written to `cur` (as k_inv_su), then the adjoint of S_u runs with that
// M_d and U_d (as k_adj_su, which would recompute M_d and reload U_d). One
// thread per site and link direction, as k_adj_su; phi goes with direction 1.
template <typename T>
__global__ void __launch_bounds__(128, 3) k_inv_adj_su(int N, State<T> nxt, State<T> cur, AdjStateT<T> a, T c,
                             T c2) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int d = blockIdx.y;  // the link direction of this thread
    if (d == 1) {
        H3<T> phi = ld_h(nxt.phi, pos, n);
        h_axpy(phi, -c2, ld_h(nxt.pi, pos, n));
        st_h(cur.phi, pos, n, phi);
    } else {
        // pi_bar += c2 phi_bar (phi_bar itself passes through unchanged)
        H3<T> pib = ld_h9a(a.pi, pos, n);
        h_axpy(pib, c2, ld_h9a(a.phi, pos, n));
        st_h9a(a.pi, pos, n, pib);
    }
    {
        C<T> *Ub = d ? a.uy : a.ux;
        C<T> *Eb = d ? a.e2 : a.e1;
        const M3<T> X = times_i(ld_herm8(d ? nxt.e2 : nxt.e1, pos, n), c);
        const M3<T> M = taylor2(X);
        const M3<T> U = mul(inverse3(M), ld_m3(d ? nxt.uy : nxt.ux, pos, n));
        st_m3(d ? cur.uy : cur.ux, pos, n, U);
        const M3<T> Ubar = ld_adj(Ub, pos, n);
        st_adj(Ub, pos, n, mul_dn(M, Ubar));
        const M3<T> Mb = mul_nd(Ubar, U);
        M3<T> Xb = Mb;
        add_to(Xb, sc(addm(mul_nd(Mb, X), mul_dn(X, Mb)), T(0.5)));
        H3<T> Eb_ = herm_part(times_i(Xb, -c));
        h_traceless(Eb_);
        h_add(Eb_, ld_h8a(Eb, pos, n));
        st_h8a(Eb, pos, n, Eb_);
    }
}

// S_e: the adjoints G_d of E_d' (traceless Hermitian, from k_adj_su) and of
// pi' through the plaquette, the two staples, the commutator terms of E and
// the pi bracket into the link and phi adjoints of the site and its
// neighbours (FP64 atomics). Three thread roles (blockIdx.y) split the work
// by target so that a thread sums every term landing on one link before its
// atomic update, and phi adjoints take their 9 Hermitian components:
// 225 atomics a site. With Mb_0 = -2i cst (G_1 - G_2), Mb_1 = -2i cst G_1,
// Mb_2 = -2i cst G_2, Cb_d = cdt G_d and brb = cdt pi_bar:
//   plaquette Ux Uy(+x) (Uy Ux(+y))^dag:   A = Ux Uy(+x), B = Uy Ux(+y),
//       Ab = Mb_0 B, Bb = Mb_0^dag A
//   E1 staple Ux Uy(+x-y)^dag Ux(-y)^dag Uy(-y):  P = Ux Uy(+x-y)^dag,
//       Q = Ux(-y)^dag Uy(-y), Pb = Mb_1 Q^dag, Qb = P^dag Mb_1
//   E2 staple Uy Ux(-x+y)^dag Uy(-x)^dag Ux(-x):  P2, Q2, Pb2, Qb2 likewise
//   transport: phb_d = i[phi, Cb_d] + brb, ph_d = U_d phi(+d) U_d^dag
// role 0: Ux += Ab Uy(+x)^dag + Pb Uy(+x-y) + 2 phb_x Ux phi(+x);
//         Uy(+x) += Ux^dag Ab; Uy(+x-y) += Pb^dag Ux; phi(+x) += Ux^dag phb_x Ux
// role 1: Uy += Bb Ux(+y)^dag + Pb2 Ux(-x+y) + 2 phb_y Uy phi(+y);
//         Ux(+y) += Uy^dag Bb; Ux(-x+y) += Pb2^dag Uy; phi(+y) += Uy^dag phb_y Uy;
//         phi += -4 brb + i[Cb_1, ph_x] + i[Cb_2, ph_y]
// role 2: Ux(-x) += Uy(-x) Qb2 + 2 phi(-x) Ux(-x) brb; Uy(-x) += Ux(-x) Qb2^dag;
//         phi(-x) += Ux(-x) brb Ux(-x)^dag; and the same along y with Qb
template <typename T>
__global__ void __launch_bounds__(128) k_adj_se(int N, State<T> cur, AdjStateT<T> a, T cst,
                                                T cdt) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const StepGeom G = step_geom(N, (int)(pos / N), (int)(pos % N));
    const int role = blockIdx.y;
    if (role == 0) {
        const H3<T> h1 = ld_h8a(a.e1, pos, n);
        const M3<T> ux = ld_link(cur.ux, pos, n);
        M3<T> acc;
        {
            const M3<T> uy_px = ld_link(cur.uy, G.pX, n);
            const M3<T> B = mul(ld_link(cur.uy, pos, n), ld_link(cur.ux, G.pY, n));
            const M3<T> Mb = times_i(minus(sc(from_h(h1), cst), sc(from_h(ld_h8a(a.e2, pos, n)), cst)), -T(2.));
            const M3<T> Ab = mul(Mb, B);
            acc = mul_nd(Ab, uy_px);
            atomic_add_m(a.uy, G.pX, n, mul_dn(ux, Ab));
        }
        {
            const M3<T> uy_pxmy = ld_link(cur.uy, G.pXmY, n);
            const M3<T> Q = mul_dn(ld_link(cur.ux, G.mY, n), ld_link(cur.uy, G.mY, n));
            const M3<T> Pb = mul_nd(times_i(sc(from_h(h1), cst), -T(2.)), Q);
            add_to(acc, mul(Pb, uy_pxmy));
            atomic_add_m(a.uy, G.pXmY, n, mul_dn(Pb, ux));
        }
        {
            M3<T> phb = icomm(ld_herm(cur.phi, pos, n), sc(from_h(h1), cdt));
            add_to(phb, sc(from_h(ld_h9a(a.pi, pos, n)), cdt));
            add_to(acc, sc(mul(mul(phb, ux), ld_herm(cur.phi, G.pX, n)), T(2.)));
            atomic_add_m(a.ux, pos, n, acc);
            atomic_add_h9a(a.phi, G.pX, n, mul(mul_dn(ux, phb), ux));
        }
    } else if (role == 1) {
        const H3<T> h2 = ld_h8a(a.e2, pos, n);
        const M3<T> uy = ld_link(cur.uy, pos, n);
        M3<T> acc;
        {
            const M3<T> ux_py = ld_link(cur.ux, G.pY, n);
            const M3<T> A = mul(ld_link(cur.ux, pos, n), ld_link(cur.uy, G.pX, n));
            const M3<T> Mb = times_i(minus(sc(from_h(ld_h8a(a.e1, pos, n)), cst), sc(from_h(h2), cst)), -T(2.));
            const M3<T> Bb = mul_dn(Mb, A);
            acc = mul_nd(Bb, ux_py);
            atomic_add_m(a.ux, G.pY, n, mul_dn(uy, Bb));
        }
        {
            const M3<T> ux_mxpy = ld_link(cur.ux, G.mXpY, n);
            const M3<T> Q = mul_dn(ld_link(cur.uy, G.mX, n), ld_link(cur.ux, G.mX, n));
            const M3<T> Pb = mul_nd(times_i(sc(from_h(h2), cst), -T(2.)), Q);
            add_to(acc, mul(Pb, ux_mxpy));
            atomic_add_m(a.ux, G.mXpY, n, mul_dn(Pb, uy));
        }
        {
            M3<T> phb = icomm(ld_herm(cur.phi, pos, n), sc(from_h(h2), cdt));
            add_to(phb, sc(from_h(ld_h9a(a.pi, pos, n)), cdt));
            add_to(acc, sc(mul(mul(phb, uy), ld_herm(cur.phi, G.pY, n)), T(2.)));
            atomic_add_m(a.uy, pos, n, acc);
            atomic_add_h9a(a.phi, G.pY, n, mul(mul_dn(uy, phb), uy));
        }
        {
            // phi += -4 brb + i[Cb_1, ph_x] + i[Cb_2, ph_y]
            M3<T> phib = icomm(sc(from_h(h2), cdt), mul_nd(mul(uy, ld_herm(cur.phi, G.pY, n)), uy));
            const M3<T> ux = ld_link(cur.ux, pos, n);
            add_to(phib, icomm(sc(from_h(ld_h8a(a.e1, pos, n)), cdt),
                               mul_nd(mul(ux, ld_herm(cur.phi, G.pX, n)), ux)));
            add_to(phib, sc(from_h(ld_h9a(a.pi, pos, n)), -T(4.) * cdt));
            atomic_add_h9a(a.phi, pos, n, phib);
        }
    } else {
        const M3<T> brb = sc(from_h(ld_h9a(a.pi, pos, n)), cdt);
        {
            // E2 staple's Q side and the -x transport
            const M3<T> uy = ld_link(cur.uy, pos, n), ux_mxpy = ld_link(cur.ux, G.mXpY, n);
            const M3<T> P = mul_nd(uy, ux_mxpy);
            const M3<T> Qb = mul_dn(P, times_i(sc(from_h(ld_h8a(a.e2, pos, n)), cst), -T(2.)));
            const M3<T> ux_mx = ld_link(cur.ux, G.mX, n), uy_mx = ld_link(cur.uy, G.mX, n);
            const M3<T> f = ld_herm(cur.phi, G.mX, n);
            atomic_add_m(a.uy, G.mX, n, mul_nd(ux_mx, Qb));
            M3<T> acc = mul(uy_mx, Qb);
            add_to(acc, sc(mul(mul(f, ux_mx), brb), T(2.)));
            atomic_add_m(a.ux, G.mX, n, acc);
            atomic_add_h9a(a.phi, G.mX, n, mul_nd(mul(ux_mx, brb), ux_mx));
        }
        {
            // E1 staple's Q side and the -y transport
            const M3<T> ux = ld_link(cur.ux, pos, n), uy_pxmy = ld_link(cur.uy, G.pXmY, n);
            const M3<T> P = mul_nd(ux, uy_pxmy);
            const M3<T> Qb = mul_dn(P, times_i(sc(from_h(ld_h8a(a.e1, pos, n)), cst), -T(2.)));
            const M3<T> ux_my = ld_link(cur.ux, G.mY, n), uy_my = ld_link(cur.uy, G.mY, n);
            const M3<T> f = ld_herm(cur.phi, G.mY, n);
            atomic_add_m(a.ux, G.mY, n, mul_nd(uy_my, Qb));
            M3<T> acc = mul(ux_my, Qb);
            add_to(acc, sc(mul(mul(f, uy_my), brb), T(2.)));
            atomic_add_m(a.uy, G.mY, n, acc);
            atomic_add_h9a(a.phi, G.mY, n, mul_nd(mul(uy_my, brb), uy_my));
        }
    }
}

// adjoint of T^tautau (k_tmunu_diag, Evolution.cpp:759-900) in lattice units,
// tbar[pos] = dL/dTtt_lat(pos)
template <typename T>
__global__ void k_adj_ttt(int N, State<T> s, const T *tbar, AdjStateT<T> a, T g,
                          T tau) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const T tb = tbar[pos];
    if (tb == T(0.)) return;
    const int i = (int)(pos / N), j = (int)(pos % N);
    const size_t pX = at(N, min(N - 1, i + 1), j), pY = at(N, i, min(N - 1, j + 1));
    const size_t pXY = at(N, min(N - 1, i + 1), min(N - 1, j + 1));
    const T ge = g * g / tau / tau, ht = T(0.5) / tau / tau;
    // electric: ge/2 (|E1|^2 + |E1(+y)|^2 + |E2|^2 + |E2(+x)|^2)
    atomic_add_h8a(a.e1, pos, n, sc(ld_herm8(s.e1, pos, n), tb * ge));
    atomic_add_h8a(a.e1, pY, n, sc(ld_herm8(s.e1, pY, n), tb * ge));
    atomic_add_h8a(a.e2, pos, n, sc(ld_herm8(s.e2, pos, n), tb * ge));
    atomic_add_h8a(a.e2, pX, n, sc(ld_herm8(s.e2, pX, n), tb * ge));
    // longitudinal electric: tr pi^2 / 4 over four cells
    const size_t cells[4] = {pos, pX, pY, pXY};
    for (int k = 0; k < 4; k++)
        atomic_add_h9a(a.pi, cells[k], n, sc(ld_herm(s.pi, cells[k], n), T(0.5) * tb));
    const M3<T> ux = ld_link(s.ux, pos, n), uy = ld_link(s.uy, pos, n);
    // magnetic: 2/g^2 (3 - Re tr(Ux Uy(+x) Ux(+y)^dag Uy^dag)), zero on the last row
    if (i != N - 1) {
        const T cb = -T(2.) / (g * g) * tb;
        const M3<T> uy_px = ld_link(s.uy, pX, n), ux_py = ld_link(s.ux, pY, n);
        const M3<T> A12 = mul(ux, uy_px);
        // plaq = A1 A2 A3 A4 with A1 = Ux, A2 = Uy(+x), A3 = Ux(+y)^dag, A4 = Uy^dag
        const M3<T> R = mul_nd(mul_nd(uy_px, ux_py), uy);  // A2 A3 A4
        atomic_add_m(a.ux, pos, n, sc(dagger(R), cb));
        atomic_add_m(a.uy, pX, n, sc(mul_dn(ux, mul(uy, ux_py)), cb));
        atomic_add_m(a.ux, pY, n, sc(mul_dn(uy, A12), cb));
        atomic_add_m(a.uy, pos, n, sc(mul_nd(A12, ux_py), cb));
    }
    // longitudinal magnetic: ht tr(d^2), d = phi_a - U phi_b U^dag
    struct Term {
        size_t pa, pb;
        const C<T> *u;
        C<T> *ub;
        size_t pu;
    };
    const Term terms[4] = {{pos, pX, s.ux, a.ux, pos},
                           {pos, pY, s.uy, a.uy, pos},
                           {pY, pXY, s.ux, a.ux, pY},
                           {pX, pXY, s.uy, a.uy, pX}};
    for (int k = 0; k < 4; k++) {
        const Term &tm = terms[k];
        const M3<T> u = ld_link(tm.u, tm.pu, n), fb = ld_herm(s.phi, tm.pb, n);
        const M3<T> C = mul_nd(mul(u, fb), u);
        const M3<T> d = minus(ld_herm(s.phi, tm.pa, n), C);
        const M3<T> db = sc(d, T(2.) * ht * tb);
        atomic_add_h9a(a.phi, tm.pa, n, db);
        const M3<T> Cb = sc(db, -T(1.));
        atomic_add_m(tm.ub, tm.pu, n, sc(mul(mul(Cb, u), fb), T(2.)));
        atomic_add_h9a(a.phi, tm.pb, n, mul(mul_dn(u, Cb), u));
    }
}

// Hermitian (and, for E, traceless) parts of the adjoints
template <typename T>
__global__ void k_adj_project(size_t n, AdjStateT<T> a) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    // the sweep's Hermitian storage expanded to full matrices in place (each
    // thread reads its site's planes before it writes them)
    const H3<T> e1 = ld_h8a(a.e1, pos, n), e2 = ld_h8a(a.e2, pos, n);
    const H3<T> phi = ld_h9a(a.phi, pos, n), pi = ld_h9a(a.pi, pos, n);
    st_adj(a.e1, pos, n, from_h(e1));
    st_adj(a.e2, pos, n, from_h(e2));
    st_adj(a.phi, pos, n, from_h(phi));
    st_adj(a.pi, pos, n, from_h(pi));
}

// ---------------------------------------------------------------------------
// adjoint of the initial conditions (Init.cpp:1678-1849, 2437-2691)
// ---------------------------------------------------------------------------
namespace {

// Gaussian elimination with partial pivoting for the 8 x 8 transposed Newton
// Jacobian (row-major a, solution into x)
__device__ void solve8(double a[64], double b[8], double x[8]) {
    for (int col = 0; col < 8; col++) {
        int piv = col;
        for (int r = col + 1; r < 8; r++)
            if (fabs(a[r * 8 + col]) > fabs(a[piv * 8 + col])) piv = r;
        if (piv != col) {
            for (int k = 0; k < 8; k++) {
                const double t = a[col * 8 + k];
                a[col * 8 + k] = a[piv * 8 + k];
                a[piv * 8 + k] = t;
            }
            const double t = b[col];
            b[col] = b[piv];
            b[piv] = t;
        }
        const double d = a[col * 8 + col];
        for (int r = col + 1; r < 8; r++) {
            const double l = d != 0. ? a[r * 8 + col] / d : 0.;
            for (int k = col; k < 8; k++) a[r * 8 + k] -= l * a[col * 8 + k];
            b[r] -= l * b[col];
        }
    }
    for (int r = 7; r >= 0; r--) {
        double acc = b[r];
        for (int k = r + 1; k < 8; k++) acc -= a[r * 8 + k] * x[k];
        x[r] = a[r * 8 + r] != 0. ? acc / a[r * 8 + r] : 0.;
    }
}

// Re tr(A^dag B)
__device__ __forceinline__ double re_dot(const Md &a, const Md &b) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 9; k++) s += a.m[k].r * b.m[k].r + a.m[k].i * b.m[k].i;
    return s;
}

// central difference of the closed-form exponential exp(i q.t) along q_b
__device__ __forceinline__ Md dexp(double q[8], int b, double h) {
    const double q0 = q[b];
    q[b] = q0 + h;
    const Md ep = exp_from_coeff(q);
    q[b] = q0 - h;
    const Md em = exp_from_coeff(q);
    q[b] = q0;
    return sc(minus(ep, em), 0.5 / h);
}

constexpr double kDexpStep = 1e-5;  // truncation ~1e-10, rounding ~1e-11

// Q = q.t with t^a = lambda_a / 2 (the matrix exp_from_coeff exponentiates)
__device__ __forceinline__ Md q_matrix(const double q[8]) {
    const double c8 = IPG_C8, s3 = IPG_INV_SQRT3;
    Md Q;
    Q.m[0] = {0.5 * q[2] + c8 * q[7], 0.};
    Q.m[4] = {-0.5 * q[2] + c8 * q[7], 0.};
    Q.m[8] = {-s3 * q[7], 0.};
    Q.m[1] = {0.5 * q[0], -0.5 * q[1]};
    Q.m[3] = {0.5 * q[0], 0.5 * q[1]};
    Q.m[2] = {0.5 * q[3], -0.5 * q[4]};
    Q.m[6] = {0.5 * q[3], 0.5 * q[4]};
    Q.m[5] = {0.5 * q[5], -0.5 * q[6]};
    Q.m[7] = {0.5 * q[5], 0.5 * q[6]};
    return Q;
}

// tr(a^dag b)
__device__ __forceinline__ C<double> dot_c(const Md &a, const Md &b) {
    C<double> s = {0., 0.};
#pragma unroll
    for (int k = 0; k < 9; k++) {
        s.r += a.m[k].r * b.m[k].r + a.m[k].i * b.m[k].i;
        s.i += a.m[k].r * b.m[k].i - a.m[k].i * b.m[k].r;
    }
    return s;
}

__device__ __forceinline__ Md cscale(const Md &a, C<double> s) {
    Md r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = cmul(a.m[k], s);
    return r;
}

__device__ __forceinline__ C<double> cadd(C<double> a, C<double> b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ C<double> csub(C<double> a, C<double> b) { return {a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ C<double> crs(C<double> a, double s) { return {a.r * s, a.i * s}; }
__device__ __forceinline__ C<double> cis(C<double> a, double s) { return {-a.i * s, a.r * s}; }  // i s a

// qb_b = Re tr(eb^dag dE/dq_b), b = 0..7, for E = exp(i q.t): the
// vector-Jacobian product of the exponential without differencing.
// With Q = q.t, c0 = det Q, c1 = tr(Q^2)/2 and E = f0 + f1 Q + f2 Q^2
// (Cayley-Hamilton, the f_j of expm_coeff as functions of u and w):
//   qb_b = Re(P0) tr(Q^2 t^b) + Re(P1) q_b / 2 + Re tr((f1 eb^dag + f2 (Q eb^dag + eb^dag Q)) t^b)
// where P_i = sum_j (df_j/dc_i) tr(eb^dag Q^j), since dc0/dq_b = tr(Q^2 t^b)
// (the adjugate of a traceless Q is Q^2 - c1) and dc1/dq_b = q_b / 2. The
// df_j/dc_i follow from f_j = h_j(u, w) / (9u^2 - w^2) and the derivatives
// of u, w by c0, c1 (c0 = 2u^3 - 2u w^2, c1 = 3u^2 + w^2 differentiated
// implicitly: du/dc0 = 1/(2D), du/dc1 = u/D, dw/dc0 = -3u/(2wD), dw/dc1 = (3u^2-w^2)/(2wD)
// with D = 9u^2 - w^2). For c1 < 1e-7 the Taylor series to third order is
// used (error below 1e-11). Returns false where two eigenvalues of Q nearly
// coincide (w or D small against c1) or where exp_from_coeff returns the
// identity; the caller then differences instead.
__device__ bool exp_vjp(const double q[8], const Md &eb, double qb[8]) {
    const Md Q = q_matrix(q);
    const Md Q2 = mul(Q, Q);
    const Md ebd = dagger(eb);
    const Md Qe = mul(Q, ebd), eQ = mul(ebd, Q);
    double c1 = 0.;
#pragma unroll
    for (int a = 0; a < 8; a++) c1 += q[a] * q[a];
    c1 *= 0.25;
    Md M;
    double s1 = 0.;
    if (c1 < 1e-7) {
        // d/dq_b of 1 + iQ - Q^2/2 - iQ^3/6:
        // M = i eb^dag - (Q eb^dag + eb^dag Q)/2 - i (Q^2 eb^dag + Q eb^dag Q + eb^dag Q^2)/6
        M = times_i(ebd, 1.);
        sub_from(M, sc(addm(Qe, eQ), 0.5));
        Md t3 = mul(Q, Qe);
        add_to(t3, mul(Qe, Q));
        add_to(t3, mul(ebd, Q2));
        sub_from(M, times_i(t3, 1. / 6.));
    } else {
        const double c0 = re_trace_mul(Q2, Q) / 3.;  // det Q = tr(Q^3)/3
        const double t3 = c1 / 3., st3 = sqrt(t3);
        const double c0max = fmax(1e-15, 2. * (t3 * st3));
        const double theta3 = acos(c0 / c0max) / 3.;
        double sth, cth;
        sincos(theta3, &sth, &cth);
        const double u = st3 * cth, w = sqrt(c1) * sth;
        const double D = 9. * u * u - w * w;
        if (!(w >= 1e-3 * sqrt(c1)) || !(fabs(D) >= 1e-3 * c1)) return false;
        double su, cu, sw, cw;
        sincos(u, &su, &cu);
        sincos(w, &sw, &cw);
        const C<double> E2 = {(cu - su) * (cu + su), 2. * su * cu};  // e^{2iu}
        const C<double> Em = {cu, -su};                              // e^{-iu}
        const double xi0 = sw / w, xi0p = (cw - xi0) / w;            // sin w / w, its w-derivative
        const double uu = u * u, ww = w * w;
        const C<double> B0 = {8. * uu * cw, 2. * u * (3. * uu + ww) * xi0};
        const C<double> B1 = {2. * u * cw, -(3. * uu - ww) * xi0};
        const C<double> B2 = {cw, 3. * u * xi0};
        const C<double> EB0 = cmul(Em, B0), EB1 = cmul(Em, B1), EB2 = cmul(Em, B2);
        C<double> h[3], hu[3], hw[3];
        h[0] = cadd(crs(E2, uu - ww), EB0);
        h[1] = csub(crs(E2, 2. * u), EB1);
        h[2] = csub(E2, EB2);
        hu[0] = cadd(cadd(crs(E2, 2. * u), cis(E2, 2. * (uu - ww))),
                     csub(cmul(Em, {16. * u * cw, 2. * (9. * uu + ww) * xi0}), cis(EB0, 1.)));
        hu[1] = cadd(cadd(crs(E2, 2.), cis(E2, 4. * u)),
                     csub(cis(EB1, 1.), cmul(Em, {2. * cw, -6. * u * xi0})));
        hu[2] = cadd(cis(E2, 2.), csub(cis(EB2, 1.), cmul(Em, {0., 3. * xi0})));
        hw[0] = cadd(crs(E2, -2. * w),
                     cmul(Em, {-8. * uu * sw, 2. * u * (2. * w * xi0 + (3. * uu + ww) * xi0p)}));
        hw[1] = cmul(Em, {2. * u * sw, -2. * w * xi0 + (3. * uu - ww) * xi0p});
        hw[2] = cmul(Em, {sw, -3. * u * xi0p});
        const double rD = 1. / D;
        const double du0 = 0.5 * rD, du1 = u * rD;
        const double dw0 = -1.5 * u * rD / w, dw1 = 0.5 * (3. * uu - ww) * rD / w;
        const C<double> tau[3] = {{trace(eb).r, -trace(eb).i}, dot_c(eb, Q), dot_c(eb, Q2)};
        C<double> f[3], P0 = {0., 0.}, P1 = {0., 0.};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            f[j] = crs(h[j], rD);
            const C<double> fu = crs(csub(hu[j], crs(f[j], 18. * u)), rD);
            const C<double> fw = crs(cadd(hw[j], crs(f[j], 2. * w)), rD);
            P0 = cadd(P0, cmul(cadd(crs(fu, du0), crs(fw, dw0)), tau[j]));
            P1 = cadd(P1, cmul(cadd(crs(fu, du1), crs(fw, dw1)), tau[j]));
        }
        // exp_from_coeff returns the identity when |Re u0| < 1e-15
        if (!(fabs(f[0].r + 2. / 3. * c1 * f[2].r) >= 1e-15)) return false;
        M = sc(Q2, P0.r);
        add_to(M, cscale(ebd, f[1]));
        add_to(M, cscale(addm(Qe, eQ), f[2]));
        s1 = 0.5 * P1.r;
    }
    C<double> tr[8];
    trace_ta(M, tr);
    bool ok = true;
#pragma unroll
    for (int b = 0; b < 8; b++) {
        qb[b] = tr[b].r + s1 * q[b];
        ok = ok && isfinite(qb[b]);
    }
    return ok;
}

}  // namespace

// pi(tau=0) = -i t / (4 g), t the "minus" stencil (init.cu k_initial_pi):
// pi_bar -> adjoints of U1, U2 (both directions) and of the tau = 0 links
__global__ void k_adj_initial_pi(int N, double g, const C<double> *u1x, const C<double> *u2x,
                                 const C<double> *u1y, const C<double> *u2y,
                                 const C<double> *ux, const C<double> *uy, AdjState a,
                                 C<double> *b1x, C<double> *b2x, C<double> *b1y,
                                 C<double> *b2y) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / N), iy = (int)(pos % N);
    const size_t mX = at(N, max(0, ix - 1), iy), mY = at(N, ix, max(0, iy - 1));
    const Md tb = times_i(herm(ld_adj(a.pi, pos, n)), 1. / (4. * g));
    const Md tbd = dagger(tb);
    for (int dir = 0; dir < 2; dir++) {
        const C<double> *u1 = dir ? u1y : u1x, *u2 = dir ? u2y : u2x, *u = dir ? uy : ux;
        C<double> *b1 = dir ? b1y : b1x, *b2 = dir ? b2y : b2x, *ub = dir ? a.uy : a.ux;
        {
            // here: D U^dag - D - U D^dag + D^dag
            const Md U = ld_m3(u, pos, n), D = minus(ld_m3(u1, pos, n), ld_m3(u2, pos, n));
            Md Db = mul(tb, U);
            sub_from(Db, tb);
            sub_from(Db, mul(tbd, U));
            add_to(Db, tbd);
            const Md Ub = minus(mul(tbd, D), mul(tb, D));
            atomic_add_m(b1, pos, n, Db);
            atomic_add_m(b2, pos, n, sc(Db, -1.));
            atomic_add_m(ub, pos, n, Ub);
        }
        {
            // minus (at the -dir neighbour): -U^dag D + D + D^dag U - D^dag
            const size_t q = dir ? mY : mX;
            const Md U = ld_m3(u, q, n), D = minus(ld_m3(u1, q, n), ld_m3(u2, q, n));
            Md Db = sc(mul(U, tb), -1.);
            add_to(Db, tb);
            add_to(Db, mul(U, tbd));
            sub_from(Db, tbd);
            const Md Ub = minus(mul(D, tb), mul(D, tbd));
            atomic_add_m(b1, q, n, Db);
            atomic_add_m(b2, q, n, sc(Db, -1.));
            atomic_add_m(ub, q, n, Ub);
        }
    }
}

// Newton links U = exp(i alpha.t) U1 U2 with F(alpha; U1, U2) = 0 (k_newton):
// implicit-function adjoint. With alpha_bar_b = Re tr(U_bar^dag dU/dalpha_b)
// and J^T lambda = alpha_bar, U1 and U2 receive the direct part through
// U1 U2 minus the adjoint of sum_a lambda_a F_a at fixed alpha.
__global__ void __launch_bounds__(128)
    k_adj_newton(int N, const C<double> *u1x, const C<double> *u2x, const C<double> *u1y,
                 const C<double> *u2y, const double *alpha, AdjState a, C<double> *b1x,
                 C<double> *b2x, C<double> *b1y, C<double> *b2y) {
    const size_t n = (size_t)N * N;
    const size_t lid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lid >= 2 * n) return;
    const size_t pos = lid >> 1;
    const int dir = (int)(lid & 1);
    const Md U1 = ld_m3(dir ? u1y : u1x, pos, n), U2 = ld_m3(dir ? u2y : u2x, pos, n);
    const Md S = addm(U1, U2), U0 = mul(U1, U2);
    double q[8];
    for (int k = 0; k < 8; k++) q[k] = alpha[(size_t)k * 2 * n + lid];
    const Md E = exp_from_coeff(q);
    const Md Ub = ld_adj(dir ? a.uy : a.ux, pos, n);
    double J[64], abar[8], lam[8];
    for (int b = 0; b < 8; b++) {
        const Md dU = mul(dexp(q, b, kDexpStep), U0);
        abar[b] = re_dot(Ub, dU);
        // dF_a = -Im tr(t^a (S dU^dag - dU S^dag)); stored transposed
        C<double> tr[8];
        trace_ta(minus(mul_nd(S, dU), mul_nd(dU, S)), tr);
        for (int r = 0; r < 8; r++) J[b * 8 + r] = -tr[r].i;
    }
    solve8(J, abar, lam);
    // Lambda = sum lambda_a t^a, M_bar = -i Lambda
    Md one, Lam = {};
    set_identity(one);
    for (int r = 0; r < 8; r++) add_to(Lam, sc(ta_mul(r, one), lam[r]));
    const Md Mb = times_i(Lam, -1.), Mbd = dagger(Mb);
    const Md U = mul(E, U0);
    // M = S - S^dag + S U^dag - U S^dag
    Md Sb = minus(Mb, Mbd);
    add_to(Sb, mul(Mb, U));
    sub_from(Sb, mul(Mbd, U));
    const Md Udir = minus(mul(Mbd, S), mul(Mb, S));
    const Md U0psi = mul_dn(E, Udir);
    const Md U0d = mul_dn(E, Ub);
    const Md G0 = minus(U0d, U0psi);  // adjoint of U1 U2 in total
    Md g1 = mul_nd(G0, U2), g2 = mul_dn(U1, G0);
    sub_from(g1, Sb);
    sub_from(g2, Sb);
    C<double> *B1 = dir ? b1y : b1x, *B2 = dir ? b2y : b2x;
    atomic_add_m(B1, pos, n, g1);
    atomic_add_m(B2, pos, n, g2);
}

// link products U1 = V_A V_A(+i)^dag, U2 = V_B V_B(+i)^dag (k_link_products)
__global__ void k_adj_link_products(int N, const C<double> *VA, const C<double> *VB,
                                    const C<double> *b1x, const C<double> *b2x,
                                    const C<double> *b1y, const C<double> *b2y, C<double> *vbA,
                                    C<double> *vbB) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / N), iy = (int)(pos % N);
    const size_t pX = at(N, min(N - 1, ix + 1), iy), pY = at(N, ix, min(N - 1, iy + 1));
    for (int nuc = 0; nuc < 2; nuc++) {
        const C<double> *V = nuc ? VB : VA;
        C<double> *vb = nuc ? vbB : vbA;
        const Md v = ld_m3(V, pos, n);
        const Md bx = ld_adj(nuc ? b2x : b1x, pos, n), by = ld_adj(nuc ? b2y : b1y, pos, n);
        atomic_add_m(vb, pos, n, addm(mul(bx, ld_m3(V, pX, n)), mul(by, ld_m3(V, pY, n))));
        atomic_add_m(vb, pX, n, mul_dn(bx, v));
        atomic_add_m(vb, pY, n, mul_dn(by, v));
    }
}

// one sheet of V_k = exp(-i A_k.t) V_{k-1}, backwards: V <- V_{k-1} (time
// reversal by the unitary inverse), V_bar <- V_bar_{k-1}, and the packed A
// of the sheet in work is replaced by its adjoint A_bar
__global__ void __launch_bounds__(128) k_adj_wilson_sheet(int N, double2 *work, C<double> *V,
                                                          C<double> *Vb) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    double q[8];
    for (int c = 0; c < 4; c++) {
        const double2 v = work[(size_t)c * n + pos];
        q[2 * c] = -v.x;
        q[2 * c + 1] = -v.y;
    }
    const Md e = exp_from_coeff(q);
    const Md Vk = ld_m3(V, pos, n), Vbk = ld_adj(Vb, pos, n);
    const Md Vprev = mul_dn(e, Vk);
    const Md eb = mul_nd(Vbk, Vprev);
    st_m3(V, pos, n, Vprev);
    st_adj(Vb, pos, n, mul_dn(e, Vbk));
    double qb[8];
    if (!exp_vjp(q, eb, qb))
        for (int b = 0; b < 8; b++) qb[b] = re_dot(eb, dexp(q, b, kDexpStep));
    for (int c = 0; c < 4; c++) work[(size_t)c * n + pos] = make_double2(-qb[2 * c], -qb[2 * c + 1]);
}

// rho = g sqrt(g2mu2 / Ny) xi: the packed rho_bar of one sheet in work ->
// g2mu2_bar (accumulated) and, if rho_out is set, rho_bar as [n][8]
__global__ void k_adj_rho(int N, int Ny, double g, const double *g2mu2, const double *xi,
                          uint64_t key, uint32_t nucleus, int k, const double2 *work,
                          double *g2mu_bar, double *rho_out) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    double z[8];
    if (xi) {
        for (int a = 0; a < 8; a++) z[a] = xi[((size_t)k * n + pos) * 8 + a];
    } else {
        for (int h = 0; h < 2; h++)
            for (int p = 0; p < 2; p++)
                normal2({(uint32_t)pos, (uint32_t)k, (nucleus << 1) | (uint32_t)h, 0u}, key, p,
                        z + 4 * h + 2 * p);
    }
    double acc = 0.;
    for (int c = 0; c < 4; c++) {
        const double2 v = work[(size_t)c * n + pos];
        acc += v.x * z[2 * c] + v.y * z[2 * c + 1];
        if (rho_out) {
            rho_out[pos * 8 + 2 * c] = v.x;
            rho_out[pos * 8 + 2 * c + 1] = v.y;
        }
    }
    const double m = g2mu2[pos];
    if (m > 0.) g2mu_bar[pos] += acc * g / (2. * sqrt(m * Ny));
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
namespace {
inline unsigned blocks(size_t n) { return (unsigned)((n + 127) / 128); }
}  // namespace

void launch_inverse_step(int N, const State<double> &nxt, const State<double> &cur,
                         const StepCoef<double> &cf, cudaStream_t st) {
    const size_t n = (size_t)N * N;
    const double c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / 2.);
    const double c2 = (cf.tau + cf.dt_pu / 2.) * cf.dt_pu;
    k_inv_su<<<blocks(n), 128, 0, st>>>(N, nxt, cur, c, c2);
    launch_inverse_se(N, nxt, cur, cf, st);
}

// the step coefficients in T, from the FP64 ones (one rounding each)
template <typename T>
struct AdjCoef {
    T c, c2, cst, cdt;
    explicit AdjCoef(const StepCoef<double> &cf)
        : c((T)(cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / 2.))),
          c2((T)((cf.tau + cf.dt_pu / 2.) * cf.dt_pu)),
          cst((T)(cf.tau * cf.dt_pe / (2. * cf.g * cf.g))),
          cdt((T)(cf.tau > 0 ? cf.dt_pe / cf.tau : 0.)) {}
};

template <typename T>
void launch_inverse_adjoint_step(int N, const State<T> &nxt, const State<T> &cur,
                                 const AdjStateT<T> &a, const StepCoef<double> &cf,
                                 cudaStream_t st) {
    const size_t n = (size_t)N * N;
    const AdjCoef<T> k(cf);
    k_inv_adj_su<<<dim3(blocks(n), 2), 128, 0, st>>>(N, nxt, cur, a, k.c, k.c2);
    // E and pi of the recovered state (written to cur.e1, e2, pi, which the
    // S_e adjoint does not read). Fusing this into k_adj_se's three roles, or
    // running it beside k_adj_se on a second stream, was not faster: both
    // kernels are held to two or three blocks an SM by their registers.
    launch_inverse_se<T>(N, nxt, cur, cf, st);
    if (cf.do_pe) k_adj_se<<<dim3(blocks(n), 3), 128, 0, st>>>(N, cur, a, k.cst, k.cdt);
}

template <typename T>
void launch_adjoint_step(int N, const State<T> &cur, const State<T> &nxt, const AdjStateT<T> &a,
                         const StepCoef<double> &cf, cudaStream_t st) {
    const size_t n = (size_t)N * N;
    const AdjCoef<T> k(cf);
    k_adj_su<<<dim3(blocks(n), 2), 128, 0, st>>>(N, cur, nxt, a, k.c, k.c2);
    if (cf.do_pe) k_adj_se<<<dim3(blocks(n), 3), 128, 0, st>>>(N, cur, a, k.cst, k.cdt);
}

template <typename T>
void launch_adjoint_ttt(int N, const State<T> &s, const T *tbar, const AdjStateT<T> &a, double g,
                        double tau, cudaStream_t st) {
    const size_t n = (size_t)N * N;
    k_adj_ttt<<<blocks(n), 128, 0, st>>>(N, s, tbar, a, (T)g, (T)tau);
}

template <typename T>
void launch_adjoint_project(size_t n, const AdjStateT<T> &a, cudaStream_t st) {
    k_adj_project<<<blocks(n), 128, 0, st>>>(n, a);
}

template void launch_inverse_adjoint_step<double>(int, const State<double> &,
                                                  const State<double> &, const AdjState &,
                                                  const StepCoef<double> &, cudaStream_t);
template void launch_adjoint_step<double>(int, const State<double> &, const State<double> &,
                                          const AdjState &, const StepCoef<double> &,
                                          cudaStream_t);
template void launch_adjoint_step<float>(int, const State<float> &, const State<float> &,
                                         const AdjStateT<float> &, const StepCoef<double> &,
                                         cudaStream_t);
template void launch_adjoint_ttt<double>(int, const State<double> &, const double *,
                                         const AdjState &, double, double, cudaStream_t);
template void launch_adjoint_ttt<float>(int, const State<float> &, const float *,
                                        const AdjStateT<float> &, double, double, cudaStream_t);
template void launch_adjoint_project<double>(size_t, const AdjState &, cudaStream_t);
template void launch_adjoint_project<float>(size_t, const AdjStateT<float> &, cudaStream_t);

// FP32 adjoint buffers (18 real planes a field) -> FP64 adjoint buffers
__global__ void k_adj_widen(size_t count, const float *src, double *dst) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = (double)src[i];
}

void launch_adjoint_widen(size_t n, const AdjStateT<float> &src, const AdjState &dst,
                          cudaStream_t st) {
    const C<float> *s[6] = {src.ux, src.uy, src.e1, src.e2, src.phi, src.pi};
    C<double> *d[6] = {dst.ux, dst.uy, dst.e1, dst.e2, dst.phi, dst.pi};
    for (int f = 0; f < 6; f++)
        k_adj_widen<<<blocks(18 * n), 128, 0, st>>>(18 * n, reinterpret_cast<const float *>(s[f]),
                                                    reinterpret_cast<double *>(d[f]));
}

// [9 complex planes][n] -> per site 18 doubles, for the host copy
__global__ void k_planes_to_sites(size_t n, const C<double> *src, double *dst) {
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const Md m = ld_adj(src, pos, n);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        dst[18 * pos + 2 * k] = m.m[k].r;
        dst[18 * pos + 2 * k + 1] = m.m[k].i;
    }
}

void launch_planes_to_sites(size_t n, const C<double> *src, double *dst, cudaStream_t st) {
    k_planes_to_sites<<<blocks(n), 128, 0, st>>>(n, src, dst);
}

void launch_adjoint_init_links(const AdjInitArgs &A, cudaStream_t st) {
    const size_t n = (size_t)A.N * A.N;
    k_adj_initial_pi<<<blocks(n), 128, 0, st>>>(A.N, A.g, A.u1x, A.u2x, A.u1y, A.u2y, A.ux, A.uy,
                                                A.adj, A.b1x, A.b2x, A.b1y, A.b2y);
    k_adj_newton<<<blocks(2 * n), 128, 0, st>>>(A.N, A.u1x, A.u2x, A.u1y, A.u2y, A.alpha, A.adj,
                                                A.b1x, A.b2x, A.b1y, A.b2y);
    k_adj_link_products<<<blocks(n), 128, 0, st>>>(A.N, A.VA, A.VB, A.b1x, A.b2x, A.b1y, A.b2y,
                                                   A.vbA, A.vbB);
}

void launch_adjoint_wilson_sheet(int N, double2 *work, C<double> *V, C<double> *Vb,
                                 cudaStream_t st) {
    const size_t n = (size_t)N * N;
    k_adj_wilson_sheet<<<blocks(n), 128, 0, st>>>(N, work, V, Vb);
}

void launch_adjoint_rho(const WilsonArgs &w, int k, double *g2mu_bar, double *rho_out,
                        cudaStream_t st) {
    const size_t n = (size_t)w.N * w.N;
    k_adj_rho<<<blocks(n), 128, 0, st>>>(w.N, w.Ny, w.g, w.g2mu2, w.xi, w.philox_key, w.nucleus,
                                         k, w.work, g2mu_bar, rho_out);
}

}  // namespace ipg
