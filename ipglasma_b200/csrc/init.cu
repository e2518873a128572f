// Initial conditions: colour charges -> Poisson solve -> Wilson lines ->
// tau = 0 links (Newton) -> initial longitudinal field.
//
// Reference: Init::setV (Init.cpp:1678-1849) and the tau = 0 block of
// Init::init (Init.cpp:2437-2691).
//
// The Poisson solve and Wilson-line products of Init::setV are in poisson.cu.
#include <cstdint>
#include <cstdio>

#include "expm.cuh"
#include "fields.cuh"
#include "ipg_internal.h"
#include "philox.cuh"

namespace ipg {

// ---------------------------------------------------------------------------
// link products U1 = V_A(x) V_A(x+i)^dag, U2 likewise for V_B, with the NaN
// guard of Init.cpp:2462-2470
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool nan_trace(const M3<double> &v) {
    C<double> t = trace(v);
    return isnan(t.r) || isnan(t.i);
}

__global__ void k_link_products(int N, const C<double> *VA, const C<double> *VB,
                                C<double> *u1x, C<double> *u2x, C<double> *u1y,
                                C<double> *u2y) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / N), iy = (int)(pos % N);
    const size_t pX = (size_t)min(N - 1, ix + 1) * N + iy;
    const size_t pY = (size_t)ix * N + min(N - 1, iy + 1);
    M3<double> one;
    set_identity(one);
    auto get = [&](const C<double> *V, size_t p) {
        M3<double> v = ld_m3(V, p, n);
        return nan_trace(v) ? one : v;
    };
    const M3<double> a = get(VA, pos), b = get(VB, pos);
    st_m3(u1x, pos, n, mul_nd(a, get(VA, pX)));
    st_m3(u1y, pos, n, mul_nd(a, get(VA, pY)));
    st_m3(u2x, pos, n, mul_nd(b, get(VB, pX)));
    st_m3(u2y, pos, n, mul_nd(b, get(VB, pY)));
}

void launch_link_products(int N, C<double> *VA, C<double> *VB, C<double> *u1x,
                          C<double> *u2x, C<double> *u1y, C<double> *u2y,
                          cudaStream_t st) {
    const size_t n = (size_t)N * N;
    k_link_products<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        N, VA, VB, u1x, u2x, u1y, u2y);
}

// ---------------------------------------------------------------------------
// Newton solve of the tau = 0 matching condition per link
// (Init::findUInForwardLightconeChun, Init.cpp:3344-3481)
// ---------------------------------------------------------------------------

// LU with partial pivoting and solve, in the elimination order of the
// GSL 2.5 routines the reference calls (Init.cpp:47-63). Every operand lives
// in the thread's slice of shared memory, element k at base[k * js] (js =
// the block size): entry (r, c) of the 8 x 8 matrix at J[(8 r + c) * js], the
// right-hand side at F, the solution to x. The pivoting indexes all of them
// by data, which would put register arrays in local memory. The row swaps
// are applied to F as they happen, which gives the permuted right-hand side
// that GSL forms from the permutation afterwards; F is overwritten.
__device__ void lu_solve8(double *J, double *F, double *x, int js) {
    for (int col = 0; col < 7; col++) {
        int piv = col;
        double best = fabs(J[(col * 8 + col) * js]);
        for (int row = col + 1; row < 8; row++) {
            double c = fabs(J[(row * 8 + col) * js]);
            if (c > best) {
                best = c;
                piv = row;
            }
        }
        if (piv != col) {
            for (int k = 0; k < 8; k++) {
                double t = J[(col * 8 + k) * js];
                J[(col * 8 + k) * js] = J[(piv * 8 + k) * js];
                J[(piv * 8 + k) * js] = t;
            }
            const double t = F[col * js];
            F[col * js] = F[piv * js];
            F[piv * js] = t;
        }
        const double d = J[(col * 8 + col) * js];
        if (d != 0.0) {
            for (int row = col + 1; row < 8; row++) {
                const double l = J[(row * 8 + col) * js] / d;
                J[(row * 8 + col) * js] = l;
                for (int k = col + 1; k < 8; k++) J[(row * 8 + k) * js] -= l * J[(col * 8 + k) * js];
            }
        }
    }
    for (int i = 1; i < 8; i++) {
        double acc = F[i * js];
        for (int j = 0; j < i; j++) acc -= J[(i * 8 + j) * js] * F[j * js];
        F[i * js] = acc;
    }
    for (int i = 7; i >= 0; i--) {
        double acc = F[i * js];
        for (int j = i + 1; j < 8; j++) acc -= J[(i * 8 + j) * js] * F[j * js];
        F[i * js] = acc / J[(i * 8 + i) * js];
    }
    for (int i = 0; i < 8; i++) x[i * js] = F[i * js];
}

__device__ __forceinline__ void restart_alpha(double alpha[8], uint64_t key,
                                              uint32_t link, uint32_t draw) {
    double z[8];
    normal4({link, draw, 0xA11CEu, 0u}, key, z);
    normal4({link, draw, 0xA11CEu, 1u}, key, z + 4);
#pragma unroll
    for (int a = 0; a < 8; a++) alpha[a] = z[a];
}

constexpr int kNewtonThreads = 128;
// doubles of shared memory per thread: J (64), F, dalpha, alpha, best alpha
constexpr int kNewtonSmem = 64 + 4 * 8;

// the exponent held in shared memory, into registers, entry b replaced by v
__device__ __forceinline__ void load_alpha(const double *al, int js, double out[8], int b = -1,
                                           double v = 0.) {
#pragma unroll
    for (int k = 0; k < 8; k++) out[k] = (k == b) ? v : al[k * js];
}

// Im tr(t^a M) of M = S X^dag - X S^dag ... as the 8 values F_a are formed
__device__ __forceinline__ void im_trace_ta(const M3<double> &m, double out[8]) {
    C<double> t[8];
    trace_ta(m, t);
#pragma unroll
    for (int a = 0; a < 8; a++) out[a] = t[a].i;
}

__global__ void __launch_bounds__(kNewtonThreads) k_newton(NewtonArgs A) {
    // this thread's slice of shared memory, element k at base[k * js]
    extern __shared__ double newton_j[];
    constexpr int js = kNewtonThreads;
    double *J = newton_j + threadIdx.x;
    double *Fa = J + 64 * js, *dalpha = J + 72 * js, *al = J + 80 * js, *best_al = J + 88 * js;
    const size_t n = (size_t)A.N * A.N;
    const size_t lid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lid >= 2 * n) return;
    if (A.redo_only && A.status[lid] != -1) return;
    // link order of the reference loop: per site, x then y (Init.cpp:2498-2516)
    const size_t pos = lid >> 1;
    const int dir = (int)(lid & 1);
    // Daggers of S and of the iterate are taken inside the products
    // (mul_nd: A B^dag), the best iterate is kept as its exponent, and the
    // small arrays the iteration indexes by data sit in shared memory: that
    // keeps the live state in registers. The iterates are bit-identical to
    // forming the daggers and the best matrix.
    M3<double> U0, S;
    {
        const M3<double> U1 = ld_m3(dir ? A.u1y : A.u1x, pos, n);
        const M3<double> U2 = ld_m3(dir ? A.u2y : A.u2x, pos, n);
        U0 = mul(U1, U2);
        S = U1;
        add_to(S, U2);
    }
    double traceCache[8];  // Im tr(t^a (S - S^dag))
    im_trace_ta(minus(S, dagger(S)), traceCache);

    double a8[8];
#pragma unroll
    for (int a = 0; a < 8; a++) {
        al[a * js] = 0.;
        a8[a] = 0.;
    }
    M3<double> Usol = mul(exp_from_coeff(a8), U0);
    bool have_best = false;  // false stands for the identity
    double Fzero = 10., FzeroMin = 1e6;
    int iter = 0, nRestart = 0, total = 0;
    uint32_t draws = 0;
    while (Fzero > 1e-6 && iter < A.max_iter && nRestart < A.max_restart) {
        iter++;
        total++;
        Fzero = 0.;
        {
            M3<double> Mt = mul_nd(S, Usol);
            sub_from(Mt, mul_nd(Usol, S));
            double tl[8];
            im_trace_ta(Mt, tl);
#pragma unroll
            for (int a = 0; a < 8; a++) {
                // -(traceCache + traceLoc), imaginary part
                const double f = -(traceCache[a] + tl[a]);
                Fa[a * js] = f;
                Fzero += fabs(f);
            }
        }
        bool good = true;
        for (int b = 0; b < 8; b++) {
            const double ab = al[b * js];
            const double d = fmax(0.001, fmin(10., 0.01 * fabs(ab)));
            const double ap = ab + d;
            load_alpha(al, js, a8, b, ap);
            const M3<double> Mt = mul_nd(S, minus(mul(exp_from_coeff(a8), U0), Usol));
            double tl[8];
            im_trace_ta(Mt, tl);
            double mcheck = 0.;
#pragma unroll
            for (int a = 0; a < 8; a++) {
                const double j = 2. * tl[a] / d;
                J[(a * 8 + b) * js] = j;
                mcheck += fabs(j);
                if (mcheck < 1e-15) good = false;
            }
            // the reference adds d and subtracts it again (the rounding stays)
            al[b * js] = ap - d;
        }
        if (!good) {
            // analytic approximation (Init.cpp:3419-3431)
            const M3<double> Usold = dagger(Usol);
            for (int b = 0; b < 8; b++) {
                const M3<double> Mt = ta_mul(b, Usold);
                for (int a = 0; a < 8; a++) {
                    const M3<double> Ma = ta_mul(a, S);
                    J[(a * 8 + b) * js] = -2. * re_trace_mul(Ma, Mt);
                }
            }
        }
        lu_solve8(J, Fa, dalpha, js);
        bool ok = true;
        for (int a = 0; a < 8; a++)
            if (fabs(dalpha[a * js]) > 1e5) {
                ok = false;
                break;
            }
        if (ok) {
#pragma unroll
            for (int a = 0; a < 8; a++) al[a * js] = al[a * js] + dalpha[a * js];
        } else {
            restart_alpha(a8, A.philox_key, (uint32_t)lid, draws++);
#pragma unroll
            for (int a = 0; a < 8; a++) al[a * js] = a8[a];
        }
        load_alpha(al, js, a8);
        Usol = mul(exp_from_coeff(a8), U0);
        if (Fzero < FzeroMin) {
            FzeroMin = Fzero;
            have_best = true;
#pragma unroll
            for (int a = 0; a < 8; a++) best_al[a * js] = a8[a];
        }
        if (iter == A.max_iter) {
            restart_alpha(a8, A.philox_key, (uint32_t)lid, draws++);
#pragma unroll
            for (int a = 0; a < 8; a++) al[a * js] = a8[a];
            Usol = mul(exp_from_coeff(a8), U0);
            nRestart++;
            iter = 0;
        }
    }
    int status = draws ? 1 : 0;
    if (nRestart == A.max_restart) {
        if (have_best) {
            load_alpha(best_al, js, a8);
            Usol = mul(exp_from_coeff(a8), U0);
        } else {
            set_identity(Usol);
        }
        status = 2;
    } else if (A.tol < 1e-6) {
        // polish beyond the reference's criterion (for derivatives through the
        // root): Newton steps with a central-difference Jacobian, no restarts,
        // keeping the iterate with the smallest residual
        double bestF = 1e300;
        for (int p = 0; p < 8; p++) {
            double s = 0.;
            {
                M3<double> Mt = mul_nd(S, Usol);
                sub_from(Mt, mul_nd(Usol, S));
                double tl[8];
                im_trace_ta(Mt, tl);
                for (int a = 0; a < 8; a++) {
                    const double f = -(traceCache[a] + tl[a]);
                    Fa[a * js] = f;
                    s += fabs(f);
                }
            }
            if (s < bestF) {
                bestF = s;
                for (int a = 0; a < 8; a++) best_al[a * js] = al[a * js];
            }
            if (s < A.tol) break;
            for (int b = 0; b < 8; b++) {
                const double h = 1e-6, a0 = al[b * js];
                load_alpha(al, js, a8, b, a0 + h);
                const M3<double> Up = mul(exp_from_coeff(a8), U0);
                load_alpha(al, js, a8, b, a0 - h);
                const M3<double> Um = mul(exp_from_coeff(a8), U0);
                const M3<double> dU = scaled(minus(Up, Um), 0.5 / h);
                M3<double> Mt = mul_nd(S, dU);
                sub_from(Mt, mul_nd(dU, S));
                double tl[8];
                im_trace_ta(Mt, tl);
                for (int a = 0; a < 8; a++) J[(a * 8 + b) * js] = -tl[a];
            }
            lu_solve8(J, Fa, dalpha, js);
            for (int a = 0; a < 8; a++) al[a * js] -= dalpha[a * js];
            load_alpha(al, js, a8);
            Usol = mul(exp_from_coeff(a8), U0);
        }
        for (int a = 0; a < 8; a++) al[a * js] = best_al[a * js];
        load_alpha(al, js, a8);
        Usol = mul(exp_from_coeff(a8), U0);
    }
    st_m3(dir ? A.uy : A.ux, pos, n, Usol);
    if (A.alpha)
        for (int a = 0; a < 8; a++) A.alpha[(size_t)a * 2 * n + lid] = al[a * js];
    A.iters[lid] = total;
    A.status[lid] = status;
}

// ---------------------------------------------------------------------------
// Throughput mode: Newton's method on the group. The same matching condition
//   F_a(U) = -Im tr(t^a (S - S^dag + S U^dag - U S^dag)) = 0
// is solved by steps U <- exp(i d.t) U with d = -J^-1 F and the exact
// Jacobian of that left perturbation: with X = S U^dag,
//   dF_a / dd_b = Re tr(t^a X t^b + t^a t^b X^dag) = 2 Re tr(t^b t^a X)
// (checked against central differences), so the convergence is quadratic,
// no exponential is differenced, and the loop stops as soon as
// sum_a |F_a| < tol. A link that is not below tol after kFastSteps steps, or
// that meets a non-finite value, is marked (status -1) for the reference's
// iteration, which the launcher runs after this kernel.
// ---------------------------------------------------------------------------
constexpr int kFastThreads = 128;
constexpr int kFastSmem = 64 + 2 * 8;  // J, then F and the step d
constexpr int kFastSteps = 30;

__global__ void __launch_bounds__(kFastThreads) k_newton_fast(NewtonArgs A) {
    extern __shared__ double newton_f[];
    constexpr int js = kFastThreads;
    double *J = newton_f + threadIdx.x;
    double *Fv = J + 64 * js, *dv = J + 72 * js;
    const size_t n = (size_t)A.N * A.N;
    const size_t lid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lid >= 2 * n) return;
    const size_t pos = lid >> 1;
    const int dir = (int)(lid & 1);
    M3<double> U0, S;
    {
        const M3<double> U1 = ld_m3(dir ? A.u1y : A.u1x, pos, n);
        const M3<double> U2 = ld_m3(dir ? A.u2y : A.u2x, pos, n);
        U0 = mul(U1, U2);
        S = U1;
        add_to(S, U2);
    }
    double traceCache[8];
    im_trace_ta(minus(S, dagger(S)), traceCache);
    M3<double> U = U0;  // exp(i 0.t) U0
    int steps = 0;
    bool done = false;
    for (; steps <= kFastSteps; steps++) {
        const M3<double> X = mul_nd(S, U);
        double tl[8];
        im_trace_ta(minus(X, dagger(X)), tl);
        double s = 0.;
        bool finite = true;
#pragma unroll
        for (int a = 0; a < 8; a++) {
            const double f = -(traceCache[a] + tl[a]);
            Fv[a * js] = -f;  // the right-hand side of J d = -F
            s += fabs(f);
            finite = finite && isfinite(f);
        }
        if (!finite) break;
        if (s < A.tol) {
            done = true;
            break;
        }
        if (steps == kFastSteps) break;
        for (int a = 0; a < 8; a++) {
            C<double> tr[8];
            trace_ta(ta_mul(a, X), tr);  // tr(t^b t^a X)
#pragma unroll
            for (int b = 0; b < 8; b++) J[(a * 8 + b) * js] = 2. * tr[b].r;
        }
        lu_solve8(J, Fv, dv, js);
        double d8[8];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 8; a++) {
            d8[a] = dv[a * js];
            ok = ok && isfinite(d8[a]) && fabs(d8[a]) < 1e3;
        }
        if (!ok) break;
        U = mul(exp_from_coeff(d8), U);
    }
    if (done) {
        st_m3(dir ? A.uy : A.ux, pos, n, U);
        A.iters[lid] = steps + 1;
        A.status[lid] = 0;
        if (A.alpha)
            for (int a = 0; a < 8; a++) A.alpha[(size_t)a * 2 * n + lid] = nan("");
    } else {
        A.status[lid] = -1;  // the reference's iteration takes this link
    }
}

void launch_newton(const NewtonArgs &a, cudaStream_t st) {
    const size_t links = 2 * (size_t)a.N * a.N;
    const size_t smem = sizeof(double) * kNewtonSmem * kNewtonThreads;  // 96 KB
    cudaFuncSetAttribute(k_newton, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    NewtonArgs b = a;
    if (a.mode == 1) {
        const size_t fsmem = sizeof(double) * kFastSmem * kFastThreads;  // 80 KB
        cudaFuncSetAttribute(k_newton_fast, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fsmem);
        k_newton_fast<<<(unsigned)((links + kFastThreads - 1) / kFastThreads), kFastThreads,
                        fsmem, st>>>(a);
        b.redo_only = 1;
    }
    k_newton<<<(unsigned)((links + kNewtonThreads - 1) / kNewtonThreads), kNewtonThreads, smem,
               st>>>(b);
}

// ---------------------------------------------------------------------------
// pi(tau=0) = (-2i/g) E1 with E1 from the "minus" stencil / 8
// (Init.cpp:2521-2584, 2664-2681). The stencil value t is anti-Hermitian, so
// pi = -(i / (4 g)) t is Hermitian.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void stencil_term(M3<double> &t, const M3<double> &D,
                                             const M3<double> &Dd,
                                             const M3<double> &U, bool here) {
    // here:  + D U^dag - D - U D^dag + D^dag
    // minus: - U^dag D + D + D^dag U - D^dag
    if (here) {
        add_to(t, mul_nd(D, U));
        sub_from(t, D);
        sub_from(t, mul(U, Dd));
        add_to(t, Dd);
    } else {
        sub_from(t, mul_dn(U, D));
        add_to(t, D);
        add_to(t, mul(Dd, U));
        sub_from(t, Dd);
    }
}

__global__ void k_initial_pi(int N, double g, const C<double> *u1x,
                             const C<double> *u2x, const C<double> *u1y,
                             const C<double> *u2y, const C<double> *ux,
                             const C<double> *uy, double *pi) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / N), iy = (int)(pos % N);
    const size_t mX = (size_t)max(0, ix - 1) * N + iy;
    const size_t mY = (size_t)ix * N + max(0, iy - 1);
    M3<double> t;
#pragma unroll
    for (int k = 0; k < 9; k++) t.m[k] = {0., 0.};
    {
        M3<double> D = minus(ld_m3(u1x, pos, n), ld_m3(u2x, pos, n));
        stencil_term(t, D, dagger(D), ld_m3(ux, pos, n), true);
    }
    {
        M3<double> D = minus(ld_m3(u1x, mX, n), ld_m3(u2x, mX, n));
        stencil_term(t, D, dagger(D), ld_m3(ux, mX, n), false);
    }
    {
        M3<double> D = minus(ld_m3(u1y, pos, n), ld_m3(u2y, pos, n));
        stencil_term(t, D, dagger(D), ld_m3(uy, pos, n), true);
    }
    {
        M3<double> D = minus(ld_m3(u1y, mY, n), ld_m3(u2y, mY, n));
        stencil_term(t, D, dagger(D), ld_m3(uy, mY, n), false);
    }
    // pi = (-2i/g) * (t / 8): entry (r,s) = (2/(8g)) * (Im t, -Re t)
    const double f = 2. / g;
    M3<double> p;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double er = t.m[k].r / 8., ei = t.m[k].i / 8.;
        p.m[k] = {f * ei, -f * er};
    }
    st_h(pi, pos, n, to_h(p));
}

void launch_initial_pi(int N, double g, const C<double> *u1x,
                       const C<double> *u2x, const C<double> *u1y,
                       const C<double> *u2y, const C<double> *ux,
                       const C<double> *uy, double *pi, cudaStream_t st) {
    const size_t n = (size_t)N * N;
    k_initial_pi<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        N, g, u1x, u2x, u1y, u2y, ux, uy, pi);
}

}  // namespace ipg
