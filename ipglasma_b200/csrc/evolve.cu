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
#include <cstdint>

#include "fields.cuh"
#include "ipg_internal.h"

namespace ipg {

// i * (P Q - (P Q)^dag) without forming P Q.
template <typename T>
__device__ __forceinline__ H3<T> i_antiherm_mul(const M3<T> &p,
                                                const M3<T> &q) {
    M3<T> x = mul(p, q);
    return i_antiherm(x);
}

template <typename T>
__device__ __forceinline__ void reunitarize(M3<T> &u) {
    // Gram-Schmidt on the first two rows, third row = conj(row0 x row1),
    // the SU(3) completion used by the reference's Matrix::reu (Matrix.h:67-109).
    T n0 = u.m[0].r * u.m[0].r + u.m[0].i * u.m[0].i + u.m[1].r * u.m[1].r +
           u.m[1].i * u.m[1].i + u.m[2].r * u.m[2].r + u.m[2].i * u.m[2].i;
    T inv0 = rsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        u.m[k].r *= inv0;
        u.m[k].i *= inv0;
    }
    // proj = <row0, row1> = sum conj(row0_k) row1_k
    C<T> pr = {T(0), T(0)};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        pr.r += u.m[k].r * u.m[3 + k].r + u.m[k].i * u.m[3 + k].i;
        pr.i += u.m[k].r * u.m[3 + k].i - u.m[k].i * u.m[3 + k].r;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        C<T> t = cmul(pr, u.m[k]);
        u.m[3 + k].r -= t.r;
        u.m[3 + k].i -= t.i;
    }
    T n1 = u.m[3].r * u.m[3].r + u.m[3].i * u.m[3].i + u.m[4].r * u.m[4].r +
           u.m[4].i * u.m[4].i + u.m[5].r * u.m[5].r + u.m[5].i * u.m[5].i;
    T inv1 = rsqrt(n1);
#pragma unroll
    for (int k = 3; k < 6; k++) {
        u.m[k].r *= inv1;
        u.m[k].i *= inv1;
    }
    // row2 = conj(row0 x row1)
    C<T> a0 = u.m[0], a1 = u.m[1], a2 = u.m[2], b0 = u.m[3], b1 = u.m[4],
         b2 = u.m[5];
    C<T> c0 = cmul(a1, b2), c0b = cmul(a2, b1);
    C<T> c1 = cmul(a2, b0), c1b = cmul(a0, b2);
    C<T> c2 = cmul(a0, b1), c2b = cmul(a1, b0);
    u.m[6] = {c0.r - c0b.r, -(c0.i - c0b.i)};
    u.m[7] = {c1.r - c1b.r, -(c1.i - c1b.i)};
    u.m[8] = {c2.r - c2b.r, -(c2.i - c2b.i)};
}

// U_new = (1 + X + X^2/2) U with X = i c E, E Hermitian:
// (1 + X + X^2/2) = (1 - c^2 E^2 / 2) + i c E.
template <typename T>
__device__ __forceinline__ M3<T> taylor2_update(const H3<T> &e, T c,
                                                const M3<T> &u) {
    M3<T> em = from_h(e);
    M3<T> e2 = mul(em, em);
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

template <typename T, bool REUNIT>
__global__ void __launch_bounds__(128)
    k_leapfrog(const EventGeom *__restrict__ ev, State<T> s, C<T> *ux_out,
               C<T> *uy_out, T *phi_out, StepCoef<T> cf) {
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

        const M3<T> ux = ld_m3(s.ux, pos, n);
        const M3<T> uy = ld_m3(s.uy, pos, n);

        // plaquette U12 = Ux Uy(x+1) Ux(y+1)^dag Uy^dag  (Evolution.cpp:228-232)
        H3<T> h12;
        {
            M3<T> a = mul(ux, ld_m3(s.uy, pX, n));
            M3<T> b = mul(uy, ld_m3(s.ux, pY, n));
            M3<T> u12 = mul_nd(a, b);
            h12 = i_antiherm(u12);
        }
        // E1 staple sum: U12 + U1m2 - h.c.  (234-257)
        H3<T> t1 = h12;
        {
            M3<T> p = mul_nd(ux, ld_m3(s.uy, pXmY, n));
            M3<T> q = mul_dn(ld_m3(s.ux, mY, n), ld_m3(s.uy, mY, n));
            h_add(t1, i_antiherm_mul(p, q));
        }
        // E2 staple sum: U12^dag + U2m1 - h.c.  (240-244, 266-275)
        H3<T> t2;
        {
            M3<T> p = mul_nd(uy, ld_m3(s.ux, mXpY, n));
            M3<T> q = mul_dn(ld_m3(s.uy, mX, n), ld_m3(s.ux, mX, n));
            t2 = i_antiherm_mul(p, q);
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

        // parallel transports of phi (evolvePi 139-157, evolveE 221-223, 278-279)
        H3<T> br;
        {
            H3<T> phx = conj_h(ux, ld_h(s.phi, pX, n));
            h_axpy(e1, cdt, i_commutator(phx, phi));
            br = phx;
        }
        {
            H3<T> phy = conj_h(uy, ld_h(s.phi, pY, n));
            h_axpy(e2, cdt, i_commutator(phy, phi));
            h_add(br, phy);
        }
        h_add(br, conj_h_dag(ld_m3(s.ux, mX, n), ld_h(s.phi, mX, n)));
        h_add(br, conj_h_dag(ld_m3(s.uy, mY, n), ld_h(s.phi, mY, n)));
        h_axpy(br, T(-4), phi);
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
            M3<T> nx = taylor2_update(e1, c, ux);
            if (REUNIT) reunitarize(nx);
            st_m3(ux_out, pos, n, nx);
            M3<T> ny = taylor2_update(e2, c, uy);
            if (REUNIT) reunitarize(ny);
            st_m3(uy_out, pos, n, ny);
        }
    } else if (cf.do_pu) {
        // phi and U only (the tau = 0 half step, Evolution.cpp:393-394)
        H3<T> phin = ld_h(s.phi, pos, n);
        const H3<T> pi = ld_h(s.pi, pos, n);
        h_axpy(phin, (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu, pi);
        st_h(phi_out, pos, n, phin);
        const T c = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
        M3<T> nx = taylor2_update(ld_h8(s.e1, pos, n), c, ld_m3(s.ux, pos, n));
        if (REUNIT) reunitarize(nx);
        st_m3(ux_out, pos, n, nx);
        M3<T> ny = taylor2_update(ld_h8(s.e2, pos, n), c, ld_m3(s.uy, pos, n));
        if (REUNIT) reunitarize(ny);
        st_m3(uy_out, pos, n, ny);
    }
}

template <typename T>
void launch_leapfrog(const EventGeom *d_ev, int N, const State<T> &s,
                     C<T> *ux_out, C<T> *uy_out, T *phi_out,
                     const StepCoef<T> &cf, bool reunit, cudaStream_t st) {
    dim3 block(32, 4);
    dim3 grid((N + 31) / 32, (N + 3) / 4);
    if (reunit)
        k_leapfrog<T, true><<<grid, block, 0, st>>>(d_ev, s, ux_out, uy_out,
                                                   phi_out, cf);
    else
        k_leapfrog<T, false><<<grid, block, 0, st>>>(d_ev, s, ux_out, uy_out,
                                                    phi_out, cf);
}

template void launch_leapfrog<double>(const EventGeom *, int,
                                      const State<double> &, C<double> *,
                                      C<double> *, double *,
                                      const StepCoef<double> &, bool,
                                      cudaStream_t);
template void launch_leapfrog<float>(const EventGeom *, int,
                                     const State<float> &, C<float> *,
                                     C<float> *, float *,
                                     const StepCoef<float> &, bool,
                                     cudaStream_t);

}  // namespace ipg
