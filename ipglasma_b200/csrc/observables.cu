// Energy-momentum tensor, Landau matching and the per-event reductions.
//
// T^{mu nu}: Evolution::Tmunu (Evolution.cpp:659-1246), evaluated with U,
// phi at tau and E, pi at tau - dtau/2 like the reference schedule
// (Evolution.cpp:406-410). The four-link products of the reference come in
// Hermitian-conjugate pairs (e.g. Uy UxpY UDypX UDx = (Ux UypX UDxpY UDy)^dag),
// so each pair is formed once and its traceless anti-Hermitian part
// AH(X) = TL(X - X^dag) is reused across T^taux, T^tauy, T^xeta and T^yeta.
//
// Landau matching: MyEigen::flowVelocity4D (MyEigen.cpp:25-314) per cell,
// including its thresholds, border exclusions and its sequential carry of
// (eps, u) from one cell to the next when a cell finds no time-like
// eigenvector (those values enter pi^{mu nu}).
#include <cstdint>

#include "fields.cuh"
#include "ipg_internal.h"

namespace ipg {

namespace {

__device__ __forceinline__ size_t idx2(int N, int i, int j) {
    return (size_t)i * N + j;
}

// traceless anti-Hermitian part TL(X - X^dag)
__device__ __forceinline__ M3<double> ah(const M3<double> &x) {
    M3<double> r;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
            r.m[3 * a + b] = {x.m[3 * a + b].r - x.m[3 * b + a].r,
                              x.m[3 * a + b].i + x.m[3 * b + a].i};
    const double t = (r.m[0].i + r.m[4].i + r.m[8].i) / 3.;
    r.m[0].i -= t;
    r.m[4].i -= t;
    r.m[8].i -= t;
    return r;
}

__device__ __forceinline__ M3<double> hm(const double *p, size_t pos, size_t n) {
    return from_h(ld_h(p, pos, n));
}
__device__ __forceinline__ M3<double> hm8(const double *p, size_t pos,
                                          size_t n) {
    return from_h(ld_h8(p, pos, n));
}
// the FP32 form's fields, widened to FP64 on load (fields.cuh)
__device__ __forceinline__ M3<double> hm(const float *p, size_t pos, size_t n) {
    return from_h(h64(p, pos, n));
}
__device__ __forceinline__ M3<double> hm8(const float *p, size_t pos, size_t n) {
    return from_h(h8_64(p, pos, n));
}
template <typename L>
__device__ __forceinline__ M3<double> lnk(const L *p, size_t pos, size_t n) {
    return link64(p, pos, n);
}
template <typename S>
__device__ __forceinline__ const State<S> &state_of(const TmunuArgs &A);
template <>
__device__ __forceinline__ const State<double> &state_of<double>(const TmunuArgs &A) {
    return A.s;
}
template <>
__device__ __forceinline__ const State<float> &state_of<float>(const TmunuArgs &A) {
    return A.s32;
}
// U A U^dag
__device__ __forceinline__ M3<double> tr_fwd(const M3<double> &u,
                                             const M3<double> &a) {
    return mul_nd(mul(u, a), u);
}
// U^dag A U
__device__ __forceinline__ M3<double> tr_bwd(const M3<double> &u,
                                             const M3<double> &a) {
    return mul(mul_dn(u, a), u);
}

}  // namespace

// diagonal components: T^tautau, T^xx, T^yy, T^etaeta (Evolution.cpp:735-899)
template <typename S>
__global__ void k_tmunu_diag(TmunuArgs A) {
    const int N = A.N;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int i = (int)(pos / N), j = (int)(pos % N);
    const size_t pX = idx2(N, min(N - 1, i + 1), j);
    const size_t pY = idx2(N, i, min(N - 1, j + 1));
    const size_t pXY = idx2(N, min(N - 1, i + 1), min(N - 1, j + 1));
    const State<S> &s = state_of<S>(A);
    const double g = A.g, tau = A.tau;

    double trE = 0., trEx = 0., trEy = 0.;
    {
        const M3<double> E1 = hm8(s.e1, pos, n), E1p = hm8(s.e1, pY, n);
        const M3<double> E2 = hm8(s.e2, pos, n), E2p = hm8(s.e2, pX, n);
        const double a1 = re_trace_mul(E1, E1), a2 = re_trace_mul(E1p, E1p);
        const double b1 = re_trace_mul(E2, E2), b2 = re_trace_mul(E2p, E2p);
        trE = a1 + a2 + b1 + b2;
        trEx = -a1 - a2 + b1 + b2;
        trEy = a1 + a2 - b1 - b2;
    }
    double trP;
    {
        const M3<double> p0 = hm(s.pi, pos, n), p1 = hm(s.pi, pX, n);
        const M3<double> p2 = hm(s.pi, pY, n), p3 = hm(s.pi, pXY, n);
        trP = re_trace_mul(p0, p0) + re_trace_mul(p1, p1) +
              re_trace_mul(p2, p2) + re_trace_mul(p3, p3);
    }
    const double ge = g * g / tau / tau;
    double Ttt = ge * trE / 2. + trP / 4.;
    double Txx = ge * trEx / 2. + trP / 4.;
    double Tyy = ge * trEy / 2. + trP / 4.;
    double Tee = 1. / tau / tau * (ge * trE / 2. - trP / 4.);

    // magnetic and longitudinal-gradient part
    const M3<double> Ux = lnk(s.ux, pos, n), Uy = lnk(s.uy, pos, n);
    double B;
    if (i == N - 1) {
        B = 0.;  // Uplaq = 1 on the last row (Evolution.cpp:748)
    } else {
        const M3<double> pl =
            mul(Ux, mul(lnk(s.uy, pX, n), mul_nd(dagger(lnk(s.ux, pY, n)), Uy)));
        B = 2. / (g * g) * (3. - trace(pl).r);
    }
    const M3<double> phi = hm(s.phi, pos, n), phiX = hm(s.phi, pX, n);
    const M3<double> phiY = hm(s.phi, pY, n), phiXY = hm(s.phi, pXY, n);
    const M3<double> d1 = minus(phi, tr_fwd(Ux, phiX));
    const M3<double> d3 = minus(phi, tr_fwd(Uy, phiY));
    const M3<double> d2 = minus(phiY, tr_fwd(lnk(s.ux, pY, n), phiXY));
    const M3<double> d4 = minus(phiX, tr_fwd(lnk(s.uy, pX, n), phiXY));
    const double P1 = re_trace_mul(d1, d1), P2 = re_trace_mul(d2, d2);
    const double P3 = re_trace_mul(d3, d3), P4 = re_trace_mul(d4, d4);
    const double ht = 0.5 / tau / tau;
    Ttt += B + ht * (P1 + P2 + P3 + P4);
    Txx += B + ht * (P1 + P2 - P3 - P4);
    Tyy += B + ht * (-P1 - P2 + P3 + P4);
    Tee += 1. / tau / tau * (-B + ht * (P1 + P2 + P3 + P4));

    const double a4 = pow(A.a, 4.), a6 = pow(A.a, 6.);
    A.T10[0 * n + pos] = Ttt / a4;
    A.T10[1 * n + pos] = Txx / a4;
    A.T10[2 * n + pos] = Tyy / a4;
    A.T10[3 * n + pos] = Tee / a6;
}

// T^taux, T^tauy, T^taueta, T^xy, T^xeta, T^yeta (Evolution.cpp:902-1238),
// in six launches (one kernel for all six keeps too many FP64 3x3 matrices
// live and spills). For direction D (0 = x, 1 = y):
//   PART 2D     the plaquette sums K, K' (Kx, Kxp or Ky, Kyp) and from them
//               the magnetic traces of T^taud and T^deta, parked in their
//               output planes;
//   PART 2D+1   the electric/transport traces, combined with the parked
//               values into T^taud and T^deta;
//   PART 4, 5   T^taueta and T^xy.
struct OffdiagGeom {
    size_t pos, pX, pY, pXY, mX, mY, mXpY, pXmY, p2X, p2Y, p2XY, pX2Y;
};

__device__ __forceinline__ OffdiagGeom offdiag_geom(int N, size_t pos) {
    const int i = (int)(pos / N), j = (int)(pos % N);
    const int ip = min(N - 1, i + 1), im = max(0, i - 1), i2 = min(N - 1, i + 2);
    const int jp = min(N - 1, j + 1), jm = max(0, j - 1), j2 = min(N - 1, j + 2);
    OffdiagGeom G;
    G.pos = pos;
    G.pX = idx2(N, ip, j);
    G.pY = idx2(N, i, jp);
    G.pXY = idx2(N, ip, jp);
    G.mX = idx2(N, im, j);
    G.mY = idx2(N, i, jm);
    G.mXpY = idx2(N, im, jp);
    G.pXmY = idx2(N, ip, jm);
    G.p2X = idx2(N, i2, j);
    G.p2Y = idx2(N, i, j2);
    G.p2XY = idx2(N, i2, jp);
    G.pX2Y = idx2(N, ip, j2);
    return G;
}

template <int PART, typename S>
__global__ void __launch_bounds__(128) k_tmunu_offdiag(TmunuArgs A) {
    const int N = A.N;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const OffdiagGeom G = offdiag_geom(N, pos);
    const State<S> &s = state_of<S>(A);
    const double g = A.g, tau = A.tau;
    const double a4 = pow(A.a, 4.), a5 = pow(A.a, 5.);

    if constexpr (PART == 0 || PART == 2) {
        const M3<double> Ux = lnk(s.ux, pos, n), Uy = lnk(s.uy, pos, n);
        const M3<double> UxpY = lnk(s.ux, G.pY, n), UypX = lnk(s.uy, G.pX, n);
        // Pb = Ux UypX UxpY^dag Uy^dag   (plaquette at pos)
        const M3<double> ahPb = ah(mul_nd(mul(Ux, UypX), mul(Uy, UxpY)));
        M3<double> K, Kp;
        if constexpr (PART == 0) {
            {
                // Q1 = UxmX^dag UymX UxmXpY Uy^dag
                const M3<double> q1 = mul_nd(
                    mul(mul_dn(lnk(s.ux, G.mX, n), lnk(s.uy, G.mX, n)), lnk(s.ux, G.mXpY, n)),
                    Uy);
                K = ah(q1);
                sub_from(K, ahPb);
            }
            {
                // R1 = UypX UxpXpY Uyp2X^dag UxpX^dag ; S1 = Ux^dag Uy UxpY UypX^dag
                const M3<double> r1 = mul_nd(mul(UypX, lnk(s.ux, G.pXY, n)),
                                             mul(lnk(s.ux, G.pX, n), lnk(s.uy, G.p2X, n)));
                const M3<double> s1 = mul_nd(mul(mul_dn(Ux, Uy), UxpY), UypX);
                Kp = ah(r1);
                add_to(Kp, ah(s1));
            }
        } else {
            {
                // Q3 = UymY^dag UxmY UypXmY Ux^dag
                const M3<double> q3 = mul_nd(
                    mul(mul_dn(lnk(s.uy, G.mY, n), lnk(s.ux, G.mY, n)), lnk(s.uy, G.pXmY, n)),
                    Ux);
                K = ah(q3);
                add_to(K, ahPb);
            }
            {
                // R3 = UxpY UypXpY Uxp2Y^dag UypY^dag ; S3 = Uy^dag Ux UypX UxpY^dag
                const M3<double> r3 = mul_nd(mul(UxpY, lnk(s.uy, G.pXY, n)),
                                             mul(lnk(s.uy, G.pY, n), lnk(s.ux, G.p2Y, n)));
                const M3<double> s3 = mul_nd(mul(mul_dn(Uy, Ux), UypX), UxpY);
                Kp = ah(r3);
                add_to(Kp, ah(s3));
            }
        }
        // magnetic part of T^taud: Im tr(E K + E' K') with E = E2 (x) or E1 (y)
        {
            const S *Ep = PART == 0 ? s.e2 : s.e1;
            M3<double> c = mul(hm8(Ep, pos, n), K);
            add_to(c, mul(hm8(Ep, PART == 0 ? G.pX : G.pY, n), Kp));
            A.T10[(PART == 0 ? 4 : 5) * n + pos] = trace(c).i;
        }
        // magnetic part of T^deta: Im tr(K d + K' d') with the transported phi
        {
            const M3<double> phi = hm(s.phi, pos, n), phiXY = hm(s.phi, G.pXY, n);
            M3<double> m;
            if constexpr (PART == 0) {
                const M3<double> dY = minus(tr_fwd(Uy, hm(s.phi, G.pY, n)), phi);
                const M3<double> dXY2 = minus(tr_fwd(UypX, phiXY), hm(s.phi, G.pX, n));
                m = mul(K, dY);
                add_to(m, mul(Kp, dXY2));
            } else {
                const M3<double> dX = minus(tr_fwd(Ux, hm(s.phi, G.pX, n)), phi);
                const M3<double> dXY1 = minus(tr_fwd(UxpY, phiXY), hm(s.phi, G.pY, n));
                m = mul(K, dX);
                add_to(m, mul(Kp, dXY1));
            }
            A.T10[(PART == 0 ? 8 : 9) * n + pos] = trace(m).i;
        }
    } else if constexpr (PART == 1 || PART == 3) {
        const M3<double> pi = hm(s.pi, pos, n), piX = hm(s.pi, G.pX, n);
        const M3<double> piY = hm(s.pi, G.pY, n), piXY = hm(s.pi, G.pXY, n);
        const M3<double> Ux = lnk(s.ux, pos, n), Uy = lnk(s.uy, pos, n);
        const M3<double> UxpY = lnk(s.ux, G.pY, n), UypX = lnk(s.uy, G.pX, n);
        const M3<double> phi = hm(s.phi, pos, n), phiX = hm(s.phi, G.pX, n);
        const M3<double> phiY = hm(s.phi, G.pY, n), phiXY = hm(s.phi, G.pXY, n);
        if constexpr (PART == 1) {
            // T^taux
            const double mag = A.T10[4 * n + pos];
            M3<double> t = mul(pi, minus(tr_fwd(Ux, phiX),
                                         tr_bwd(lnk(s.ux, G.mX, n), hm(s.phi, G.mX, n))));
            add_to(t, mul(piY, minus(tr_fwd(UxpY, phiXY),
                                     tr_bwd(lnk(s.ux, G.mXpY, n), hm(s.phi, G.mXpY, n)))));
            add_to(t, mul(piX, minus(tr_fwd(lnk(s.ux, G.pX, n), hm(s.phi, G.p2X, n)),
                                     tr_bwd(Ux, phi))));
            add_to(t, mul(piXY, minus(tr_fwd(lnk(s.ux, G.pXY, n), hm(s.phi, G.p2XY, n)),
                                      tr_bwd(UxpY, phiY))));
            const double el = trace(t).r;
            A.T10[4 * n + pos] = (2. / tau / 8. * mag - 2. / 8. / tau * el) / a4;
            // T^xeta
            const double mi = A.T10[8 * n + pos];
            const M3<double> E1 = hm8(s.e1, pos, n), E1p = hm8(s.e1, G.pY, n);
            M3<double> e = mul(E1, pi);
            add_to(e, mul(E1, tr_fwd(Ux, piX)));
            add_to(e, mul(E1p, piY));
            add_to(e, mul(E1p, tr_fwd(UxpY, piXY)));
            const double v = 1. / 4. * g * trace(e).r + 1. / 8. / g * (-mi);
            A.T10[8 * n + pos] = (-2. / tau / tau * v) / a5;
        } else {
            // T^tauy
            const double mag = A.T10[5 * n + pos];
            M3<double> t = mul(pi, minus(tr_fwd(Uy, phiY),
                                         tr_bwd(lnk(s.uy, G.mY, n), hm(s.phi, G.mY, n))));
            add_to(t, mul(piX, minus(tr_fwd(UypX, phiXY),
                                     tr_bwd(lnk(s.uy, G.pXmY, n), hm(s.phi, G.pXmY, n)))));
            add_to(t, mul(piY, minus(tr_fwd(lnk(s.uy, G.pY, n), hm(s.phi, G.p2Y, n)),
                                     tr_bwd(Uy, phi))));
            add_to(t, mul(piXY, minus(tr_fwd(lnk(s.uy, G.pXY, n), hm(s.phi, G.pX2Y, n)),
                                      tr_bwd(UypX, phiX))));
            const double el = trace(t).r;
            A.T10[5 * n + pos] = (2. / tau / 8. * mag - 2. / 8. / tau * el) / a4;
            // T^yeta
            const double mi = A.T10[9 * n + pos];
            const M3<double> E2 = hm8(s.e2, pos, n), E2p = hm8(s.e2, G.pX, n);
            M3<double> e = mul(E2, pi);
            add_to(e, mul(E2, tr_fwd(Uy, piY)));
            add_to(e, mul(E2p, piX));
            add_to(e, mul(E2p, tr_fwd(UypX, piXY)));
            const double v = 1. / 4. * g * trace(e).r + 1. / 8. / g * (-mi);
            A.T10[9 * n + pos] = (-2. / tau / tau * v) / a5;
        }
    } else {
        const M3<double> Ux = lnk(s.ux, pos, n), Uy = lnk(s.uy, pos, n);
        const M3<double> UxpY = lnk(s.ux, G.pY, n), UypX = lnk(s.uy, G.pX, n);
        const M3<double> phi = hm(s.phi, pos, n), phiX = hm(s.phi, G.pX, n);
        const M3<double> phiY = hm(s.phi, G.pY, n), phiXY = hm(s.phi, G.pXY, n);
        const M3<double> dX = minus(tr_fwd(Ux, phiX), phi), dY = minus(tr_fwd(Uy, phiY), phi);
        const M3<double> dXY1 = minus(tr_fwd(UxpY, phiXY), phiY);
        const M3<double> dXY2 = minus(tr_fwd(UypX, phiXY), phiX);
        const M3<double> E1 = hm8(s.e1, pos, n), E1p = hm8(s.e1, G.pY, n);
        const M3<double> E2 = hm8(s.e2, pos, n), E2p = hm8(s.e2, G.pX, n);
        if constexpr (PART == 4) {
            // T^taueta
            M3<double> t = mul(E1, dX);
            add_to(t, mul(E1p, dXY1));
            add_to(t, mul(E2, dY));
            add_to(t, mul(E2p, dXY2));
            A.T10[6 * n + pos] = (g / tau / tau / tau * trace(t).r) / a5;
        } else {
            // T^xy
            M3<double> ea = E1;
            add_to(ea, tr_fwd(Uy, E1p));
            M3<double> eb = E2;
            add_to(eb, tr_fwd(Ux, E2p));
            M3<double> t = scaled(mul(ea, eb), -1. / 4. * g * g);
            const M3<double> wy = tr_fwd(Uy, dXY1);  // Uy (phiTildeXY1 - phiY) Uy^dag
            const M3<double> wx = tr_fwd(Ux, dXY2);  // Ux (phiTildeXY2 - phiX) Ux^dag
            M3<double> q = mul(dX, dY);
            add_to(q, mul(wy, dY));
            add_to(q, mul(dX, wx));
            add_to(q, mul(wy, wx));
            add_to(t, scaled(q, 1. / 4.));
            A.T10[7 * n + pos] = (2. / tau / tau * trace(t).r) / a4;
        }
    }
}

void launch_tmunu_diag(const TmunuArgs &a, cudaStream_t st) {
    const size_t n = (size_t)a.N * a.N;
    if (a.from32)
        k_tmunu_diag<float><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a);
    else
        k_tmunu_diag<double><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a);
}

template <typename S>
static void launch_tmunu_t(const TmunuArgs &a, cudaStream_t st) {
    const size_t n = (size_t)a.N * a.N;
    const unsigned b = (unsigned)((n + 127) / 128);
    k_tmunu_diag<S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<0, S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<1, S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<2, S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<3, S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<4, S><<<b, 128, 0, st>>>(a);
    k_tmunu_offdiag<5, S><<<b, 128, 0, st>>>(a);
}

void launch_tmunu(const TmunuArgs &a, cudaStream_t st) {
    if (a.from32)
        launch_tmunu_t<float>(a, st);
    else
        launch_tmunu_t<double>(a, st);
}

}  // namespace ipg

// ===========================================================================
// Landau matching
// ===========================================================================
#include "eig4.cuh"

namespace ipg {

// carried per-cell results of the eigen-vector scan; bit k of `wrote` marks
// that variable k (eps, utau, ux, uy, ueta) was assigned while this cell was
// processed
struct LandauCell {
    double v[5];
    int wrote;
};

// (128, 4): four blocks an SM. Every index of the eigen-solver is static
// (eig4.cuh), so unbounded it needs 194 registers and no local memory; at
// 128 registers part of it spills, which the extra warps hide (447 against
// 443 events/s at three blocks an SM and 437 at two)
__global__ void __launch_bounds__(128, 4) k_landau(LandauArgs A, double *carry, int *wrote) {
    const int N = A.N;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int si = (int)(pos / N), sj = (int)(pos % N);
    const double *T = A.T10;
    const double Ttt = T[0 * n + pos], Txx = T[1 * n + pos], Tyy = T[2 * n + pos];
    const double Tee = T[3 * n + pos], Ttx = T[4 * n + pos], Tty = T[5 * n + pos];
    const double Tte = T[6 * n + pos], Txy = T[7 * n + pos], Txe = T[8 * n + pos];
    const double Tye = T[9 * n + pos];
    const double t2d = A.tau_fm * A.tau_fm;  // (it*dtau*a)*(it*dtau*a)
    const double data[16] = {Ttt, -Ttx, -Tty, -t2d * Tte,
                             Ttx, -Txx, -Txy, -t2d * Txe,
                             Tty, -Txy, -Tyy, -t2d * Tye,
                             Tte, -Txe, -Tye, -t2d * Tee};
    double er[4], ei[4], vr[16], vi[16];
    eig4(data, er, ei, vr, vi);

    double eps = 0., utau = 0., ux = 0., uy = 0., ueta = 0.;
    int w = 0;
    double cell_eps = Ttt, cu[4] = {1., 0., 0., 0.};
    int found = 0;
    const double tau2 = A.tau2_fm;  // a*it*dtau*a*it*dtau
#pragma unroll
    for (int i = 0; i < 4; i++) {
        // square and Euclidean square of the eigenvector (complex products)
        double sqr = 0., sqi = 0., eur = 0., eui = 0.;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const double zr = vr[4 * i + j], zi = vi[4 * i + j];
            const double z2r = zr * zr - zi * zi, z2i = zr * zi + zi * zr;
            eur += z2r;
            eui += z2i;
            if (j == 0) {
                sqr += z2r;
                sqi += z2i;
            } else if (j < 3) {
                sqr -= z2r;
                sqi -= z2i;
            } else {
                const double ar = tau2 * zr, ai = tau2 * zi;  // z_aux = tau2 z
                sqr -= ar * zr - ai * zi;
                sqi -= ar * zi + ai * zr;
            }
        }
        const double factor = sqrt(fabs(eur / sqr));
        if (sqr > 0) {
            eps = er[i];
            w |= 1;
            if (fabs(ei[i]) > 0.001 && si > 0 && sj > 0 && si < N - 5 && sj < N - 5)
                eps = Ttt;
        }
        double s2 = 0.;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const double zr = vr[4 * i + j] * factor, zi = vi[4 * i + j] * factor;
            const double z2r = zr * zr - zi * zi;
            if (j == 0) {
                s2 += z2r;
            } else if (j < 3) {
                s2 -= z2r;
            } else {
                const double ar = tau2 * zr, ai = tau2 * zi;
                s2 -= ar * zr - ai * zi;
            }
        }
        if (s2 > 0) {
            found += 1;
            int change = 0;
    #pragma unroll
        for (int j = 0; j < 4; j++) {
                double zr = vr[4 * i + j] * factor, zi = vi[4 * i + j] * factor;
                if (j == 0 && zr < 0) {
                    change = 1;
                    zr = -zr;
                    zi = -zi;
                }
                if (j > 0 && change == 1) {
                    zr = -zr;
                    zi = -zi;
                }
                if (j == 0) utau = (eps > 0.1) ? zr : 1.;
                if (j == 1) ux = (eps > 0.1) ? zr : 0.;
                if (j == 2) uy = (eps > 0.1) ? zr : 0.;
                if (j == 3) ueta = (eps > 0.1) ? zr : 0.;
                if (fabs(zi) > 0.001 && eps > 0.001 && si > 10 && sj > 10 &&
                    si < N - 10 && sj < N - 10) {
                    utau = 1.;
                    ux = 0.;
                    uy = 0.;
                    ueta = 0.;
                    eps = Ttt;
                }
            }
            w |= 0x1f;
            cu[0] = utau;
            cu[1] = ux;
            cu[2] = uy;
            cu[3] = ueta;
            cell_eps = eps;
        }
    }
    A.eps[pos] = cell_eps;
#pragma unroll
    for (int k = 0; k < 4; k++) A.u4[k * n + pos] = cu[k];
    A.found[pos] = found;
    carry[0 * n + pos] = eps;
    carry[1 * n + pos] = utau;
    carry[2 * n + pos] = ux;
    carry[3 * n + pos] = uy;
    carry[4 * n + pos] = ueta;
    wrote[pos] = w;
}

// pi^{mu nu} = T^{mu nu} - (4/3) eps u u + (eps/3) g  with the values the
// reference's cell loop holds when it reaches this cell (MyEigen.cpp:259-305)
__global__ void k_landau_pi(LandauArgs A, const double *carry,
                            const int *wrote) {
    const int N = A.N;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    double v[5];
    for (int k = 0; k < 5; k++) {
        long p = (long)pos;
        while (p >= 0 && !(wrote[p] & (1 << k))) p--;
        v[k] = (p >= 0) ? carry[k * n + p] : 0.;
    }
    const double eps = v[0], utau = v[1], ux = v[2], uy = v[3], ueta = v[4];
    const double *T = A.T10;
    double *P = A.pi10;
    if (utau == 1 && ux == 0 && uy == 0 && ueta == 0) {
        for (int k = 0; k < 10; k++) P[k * n + pos] = 0.;
        return;
    }
    const double t = A.tau_fm_parts[0], d = A.tau_fm_parts[1], a = A.tau_fm_parts[2];
    const double c = 4. / 3.;
    // order: tautau xx yy etaeta taux tauy taueta xy xeta yeta
    P[0 * n + pos] = T[0 * n + pos] - c * eps * utau * utau + eps / 3.;
    P[1 * n + pos] = T[1 * n + pos] - c * eps * ux * ux - eps / 3.;
    P[2 * n + pos] = T[2 * n + pos] - c * eps * uy * uy - eps / 3.;
    P[3 * n + pos] = T[3 * n + pos] - c * eps * ueta * ueta - eps / 3. / t / d / a / t / d / a;
    P[4 * n + pos] = T[4 * n + pos] - c * eps * utau * ux;
    P[5 * n + pos] = T[5 * n + pos] - c * eps * utau * uy;
    P[6 * n + pos] = T[6 * n + pos] - c * eps * utau * ueta;
    P[7 * n + pos] = T[7 * n + pos] - c * eps * ux * uy;
    P[8 * n + pos] = T[8 * n + pos] - c * eps * ux * ueta;
    P[9 * n + pos] = T[9 * n + pos] - c * eps * uy * ueta;
}

void launch_landau(const LandauArgs &a, double *carry, int *wrote,
                   cudaStream_t st) {
    const size_t n = (size_t)a.N * a.N;
    k_landau<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a, carry, wrote);
    k_landau_pi<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a, carry, wrote);
}

}  // namespace ipg
