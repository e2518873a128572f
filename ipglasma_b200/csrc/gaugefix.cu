// Transverse Coulomb gauge fixing (GaugeFix::FFTChi, GaugeFix.cpp:17-165, and
// GaugeFix::gaugeTransform, 167-204) and the gluon multiplicity n(k_T)
// (Evolution::multiplicity, Evolution.cpp:2284-3188) on the FP64 fields.
//
// Gauge fixing is Fourier-accelerated steepest descent. One iteration:
//   k_gf_chi        per site: div A = U_x(x) - U_x(x-x) + U_y(x) - U_y(x-y)
//                   (periodic), g = sum_a Im tr(div A t^a) t^a, which for
//                   t^a = lambda^a / 2 is -(i/4) (B - tr B / 3), B = A - A^dag:
//                   Hermitian traceless, packed into 4 complex planes
//                   (g00 + i g11, g01, g02, g12); one partial of
//                   sum tr(g^dag g) / Nc per block
//                   the block that finishes last folds the partials in
//                   order (the residual, divided by N^2) and applies the
//                   reference's stopping rules (residual < 1e-9; residual
//                   above the value recorded at the last multiple of 10
//                   iterations and below 1e-6)
//   FFT convolution chi <- IFFT(-1.5 / (k~^2 + 1e-9) FFT(g)) with the Poisson
//                   kernels of poisson.cu (the multiplier is real and even, so
//                   the packed real components separate again)
//   k_gf_exp        per site: G = reu(expm(i chi)) with the reference's
//                   [6/6] Pade approximant (its own rounded coefficients,
//                   scaling by 2^-s and s squarings, the 3x3 inverse by
//                   cofactors) and its Gram-Schmidt reunitarisation
//                   (Matrix.cpp:428-553, Matrix.h:67-91, Spinor.cpp:52-137)
//   k_gf_transform  per site: U_i(x) <- G(x) U_i(x) G(x+i)^dag,
//                   E_i, phi, pi <- G E_i G^dag (in place: every site writes
//                   only its own fields and reads G from its own buffer)
// Every kernel of an iteration returns at once when the residual pass has
// set `done`, so the host enqueues iterations in chunks and reads the flag
// once per chunk.
//
// The multiplicity transforms E1, E2 and pi (13 packed complex planes) with
// the forward FFT and, per momentum k with k_x, k_y not at the centred grid's
// first row or column, takes Re tr(E(k) E(-k)) = sum_ij |E_ij(k)|^2 (the
// fields are Hermitian). With the reference's weights per field
// (g^2 / ((it - 0.5) dtau) for E1 and E2, (it - 0.5) dtau for pi) the three
// contributions go into dN/dy, dE/dy and the 100 k_T bins of width
// 2.83 / 100 (Evolution.cpp:2508-2545). The lattice momenta use a sine table
// computed on the host with the reference's expression, and the products
// and sums of k~^2 are rounded one by one, so every k lands in the bin the
// reference puts it in.
#include <cstdint>

#include "fft.cuh"
#include "fields.cuh"
#include "ipg_internal.h"

namespace ipg {

namespace {

constexpr int GB = 256;  // threads per block of the per-site kernels
// the exponential (128 registers a thread) and the transformation (168):
// blocks of 128 threads put four and three blocks on an SM
constexpr int GB_HEAVY = 128;
constexpr double kHbarcGf = 0.1973269718;  // GeV fm (Phys_consts.h)

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    return x;
}

// sum of v over the block, valid in thread 0
__device__ __forceinline__ double block_sum1(double v) {
    __shared__ double sh[GB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.;
    if (threadIdx.x == 0)
        for (int w = 0; w < GB / 32; w++) s += sh[w];
    return s;
}

__host__ __device__ __forceinline__ C<double> cadd2(C<double> a, C<double> b) { return {a.r + b.r, a.i + b.i}; }
__host__ __device__ __forceinline__ C<double> csub2(C<double> a, C<double> b) { return {a.r - b.r, a.i - b.i}; }
__host__ __device__ __forceinline__ C<double> cconj(C<double> a) { return {a.r, -a.i}; }
__host__ __device__ __forceinline__ C<double> cscale(C<double> a, double s) { return {a.r * s, a.i * s}; }
// a / b for a complex b (Smith's method, Comm. ACM 5 (1962) 435)
__host__ __device__ __forceinline__ C<double> cdiv(C<double> a, C<double> b) {
    if (fabs(b.r) >= fabs(b.i)) {
        const double r = b.i / b.r, d = b.r + b.i * r;
        return {(a.r + a.i * r) / d, (a.i - a.r * r) / d};
    }
    const double r = b.r / b.i, d = b.r * r + b.i;
    return {(a.r * r + a.i) / d, (a.i * r - a.r) / d};
}

__host__ __device__ __forceinline__ M3<double> madd(const M3<double> &a, const M3<double> &b) {
    M3<double> r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = cadd2(a.m[k], b.m[k]);
    return r;
}
__host__ __device__ __forceinline__ M3<double> mscale(const M3<double> &a, double s) {
    M3<double> r;
#pragma unroll
    for (int k = 0; k < 9; k++) r.m[k] = cscale(a.m[k], s);
    return r;
}
__host__ __device__ __forceinline__ void add_diag(M3<double> &a, double s) {
    a.m[0].r += s;
    a.m[4].r += s;
    a.m[8].r += s;
}

// A B for a product known to be Hermitian (S = 1) or anti-Hermitian
// (S = -1): the diagonal and the upper triangle are formed, the lower
// triangle is their (negated) conjugate and the diagonal's imaginary (real)
// part is zero
template <int S>
__host__ __device__ __forceinline__ M3<double> mul_sym(const M3<double> &a, const M3<double> &b) {
    M3<double> r;
    const int up[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const int i = up[q][0], j = up[q][1];
        C<double> acc = cmul(a.m[3 * i], b.m[j]);
        acc = cadd2(acc, cmul(a.m[3 * i + 1], b.m[3 + j]));
        acc = cadd2(acc, cmul(a.m[3 * i + 2], b.m[6 + j]));
        if (i == j) {
            if (S == 1) acc.i = 0.;
            else acc.r = 0.;
        }
        r.m[3 * i + j] = acc;
        if (i != j) r.m[3 * j + i] = S == 1 ? cconj(acc) : C<double>{-acc.r, acc.i};
    }
    return r;
}

// exp(M) by the [6/6] Pade approximant with scaling and squaring, in the
// steps of Matrix::expm (Matrix.cpp:431-553) for t = 1, p = 6: the
// coefficients are the reference's 10-digit roundings of
// c_k = (2p-k)! p! / ((2p)! k! (p-k)!), the norm is the largest row sum of
// |M_ij|, s = max(0, (int)(log2 |M| + 2)) when |M| > 1/2, and the
// denominator Q - P is inverted by cofactors. A matrix whose norm is zero but
// that is not zero (NaN entries) returns NaN (the reference exits there).
__host__ __device__ M3<double> expm_pade6(const M3<double> &M) {
    const double c[7] = {1., 0.5, 0.1136363636, 0.01515151515, 0.001262626263,
                         6.313131313e-05, 1.503126503e-06};
    double norm = 0.0;
    for (int i = 0; i < 3; i++) {
        double temp = 0.0;
        for (int j = 0; j < 3; j++) temp += hypot(M.m[3 * i + j].r, M.m[3 * i + j].i);
        // std::max(norm, temp): norm unless norm < temp (NaN keeps norm)
        norm = (norm < temp) ? temp : norm;
    }
    M3<double> U;
    if (norm == 0.0) {
        bool zero = true;
        for (int k = 0; k < 9; k++)
            if (M.m[k].r != 0.0 || M.m[k].i != 0.0) zero = false;
        if (zero) {
            set_identity(U);
            return U;
        }
        for (int k = 0; k < 9; k++) U.m[k] = {nan(""), nan("")};
        return U;
    }
    int s = 0;
    if (norm > 0.5) {
        s = (int)(log(norm) / log(2.0) + 2.0);
        if (s < 0) s = 0;
        const double scale = 1.0 / pow(2.0, (double)s);
        U = mscale(M, scale);
    } else {
        U = M;
    }
    // U is anti-Hermitian (a multiple of i chi), so H2 = U^2 and every
    // polynomial in H2 are Hermitian, and P U is anti-Hermitian: those
    // products form only the diagonal and the upper triangle
    const M3<double> H2 = mul_sym<1>(U, U);
    // Horner in H2: Q from c6, c4, c2, c0 and P from c5, c3, c1 (the loop of
    // Matrix.cpp:492-505 unrolled for p = 6; its first products are with
    // multiples of the identity, c I H2 = c H2 exactly), then P <- P U
    M3<double> Q = mscale(H2, c[6]);
    add_diag(Q, c[4]);
    M3<double> P = mscale(H2, c[5]);
    add_diag(P, c[3]);
    Q = mul_sym<1>(Q, H2);
    add_diag(Q, c[2]);
    P = mul_sym<1>(P, H2);
    add_diag(P, c[1]);
    Q = mul_sym<1>(Q, H2);
    add_diag(Q, c[0]);
    P = mul_sym<-1>(P, U);
    sub_from(Q, P);
    // inverse of Q by cofactors (Matrix.cpp:523-541)
    const C<double> *q = Q.m;
    auto m2 = [&](int a, int b, int c2, int d) { return csub2(cmul(q[a], q[b]), cmul(q[c2], q[d])); };
    M3<double> Hi;
    Hi.m[0] = m2(4, 8, 5, 7);
    Hi.m[1] = m2(2, 7, 1, 8);
    Hi.m[2] = m2(1, 5, 2, 4);
    Hi.m[3] = m2(5, 6, 3, 8);
    Hi.m[4] = m2(0, 8, 2, 6);
    Hi.m[5] = m2(2, 3, 0, 5);
    Hi.m[6] = m2(3, 7, 4, 6);
    Hi.m[7] = m2(1, 6, 0, 7);
    Hi.m[8] = m2(0, 4, 1, 3);
    C<double> det = cmul(cmul(q[0], q[4]), q[8]);
    det = cadd2(det, cmul(cmul(q[1], q[5]), q[6]));
    det = cadd2(det, cmul(cmul(q[2], q[3]), q[7]));
    det = csub2(det, cmul(cmul(q[2], q[4]), q[6]));
    det = csub2(det, cmul(cmul(q[1], q[3]), q[8]));
    det = csub2(det, cmul(cmul(q[5], q[7]), q[0]));
    const C<double> inv = cdiv({1.0, 0.0}, det);
    for (int k = 0; k < 9; k++) Hi.m[k] = cmul(Hi.m[k], inv);
    // odd == 0 after the loop: U = 2 H P + 1
    U = mul(mscale(Hi, 2.0), P);
    add_diag(U, 1.0);
    for (int i = 0; i < s; i++) U = mul(U, U);
    return U;
}

__host__ __device__ __forceinline__ double vnorm(const C<double> v[3]) {
    double s = 0.;
    for (int i = 0; i < 3; i++) s += v[i].r * v[i].r + v[i].i * v[i].i;
    return sqrt(s);
}
__host__ __device__ __forceinline__ void vnormalize(C<double> v[3]) {
    const double nv = vnorm(v);
    for (int i = 0; i < 3; i++) v[i] = {v[i].r / nv, v[i].i / nv};
}

// Matrix::reu (Matrix.h:67-91): rows 0 and 1 by Gram-Schmidt (the second
// against the first renormalised once more, as Spinor::GramSchmidt does),
// row 2 the normalised complex conjugate of their cross product.
__host__ __device__ M3<double> reunitarize(const M3<double> &u) {
    C<double> e1[3] = {u.m[0], u.m[1], u.m[2]};
    C<double> a2[3] = {u.m[3], u.m[4], u.m[5]};
    vnormalize(e1);
    C<double> a1n[3] = {e1[0], e1[1], e1[2]};
    vnormalize(a1n);
    C<double> ip = {0., 0.};  // <a1n, a2>
    for (int i = 0; i < 3; i++) ip = cadd2(ip, cmul(cconj(a1n[i]), a2[i]));
    C<double> e2[3];
    for (int i = 0; i < 3; i++) e2[i] = csub2(a2[i], cmul(ip, a1n[i]));
    vnormalize(e2);
    C<double> e3[3] = {cconj(csub2(cmul(e1[1], e2[2]), cmul(e1[2], e2[1]))),
                       cconj(csub2(cmul(e1[2], e2[0]), cmul(e1[0], e2[2]))),
                       cconj(csub2(cmul(e1[0], e2[1]), cmul(e1[1], e2[0])))};
    vnormalize(e3);
    M3<double> r;
    for (int i = 0; i < 3; i++) {
        r.m[i] = e1[i];
        r.m[3 + i] = e2[i];
        r.m[6 + i] = e3[i];
    }
    return r;
}

}  // namespace

// -------------------------------------------------------------------------
// gauge fixing
// -------------------------------------------------------------------------

// the reference's stopping rules on the residual of iteration ctl->iter
__device__ __forceinline__ void gf_decide(double res, GaugeFixCtl *ctl) {
    const int it = ctl->iter;
    if (it % 10 == 0) {
        ctl->prev = res;
        if (it / 10 < kGaugeHistory) ctl->hist[it / 10] = res;
    }
    ctl->last = res;
    ctl->checks = it + 1;
    if (res < 1e-9 || (res > ctl->prev && res < 1e-6)) {
        ctl->done = 1;  // no transform in this iteration
    } else {
        ctl->iter = it + 1;
    }
}

__global__ void __launch_bounds__(GB) k_gf_chi(State<double> s, int N, double2 *chi,
                                               double *partial, GaugeFixCtl *ctl) {
    if (ctl->done) return;
    const size_t n = (size_t)N * N;
    double acc = 0.;
    for (size_t pos = (size_t)blockIdx.x * GB + threadIdx.x; pos < n;
         pos += (size_t)gridDim.x * GB) {
        const int ix = (int)(pos / N), iy = (int)(pos % N);
        const size_t mx = (size_t)((ix + N - 1) % N) * N + iy;
        const size_t my = (size_t)ix * N + (iy + N - 1) % N;
        M3<double> A = ld_m3(s.ux, pos, n);
        sub_from(A, ld_m3(s.ux, mx, n));
        add_to(A, ld_m3(s.uy, pos, n));
        sub_from(A, ld_m3(s.uy, my, n));
        // diagonal: g_jj = (Im A_jj - sum Im A / 3) / 2
        const double t3 = (A.m[0].i + A.m[4].i + A.m[8].i) / 3.;
        const double g00 = 0.5 * (A.m[0].i - t3), g11 = 0.5 * (A.m[4].i - t3);
        const double g22 = 0.5 * (A.m[8].i - t3);
        // upper triangle: g_jk = -(i/4) (A_jk - conj(A_kj))
        auto off = [&](int jk, int kj) {
            const C<double> z = {A.m[jk].r - A.m[kj].r, A.m[jk].i + A.m[kj].i};
            return C<double>{0.25 * z.i, -0.25 * z.r};
        };
        const C<double> g01 = off(1, 3), g02 = off(2, 6), g12 = off(5, 7);
        chi[0 * n + pos] = make_double2(g00, g11);
        chi[1 * n + pos] = make_double2(g01.r, g01.i);
        chi[2 * n + pos] = make_double2(g02.r, g02.i);
        chi[3 * n + pos] = make_double2(g12.r, g12.i);
        acc += (g00 * g00 + g11 * g11 + g22 * g22 +
                2. * (g01.r * g01.r + g01.i * g01.i + g02.r * g02.r + g02.i * g02.i +
                      g12.r * g12.r + g12.i * g12.i)) /
               3.;
    }
    const double b = block_sum1(acc);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = b;
        __threadfence();  // the partial is visible before the arrival counts
        last = atomicAdd(&ctl->arrived, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block: every partial is written; fold them in block order
    __threadfence();
    double v = 0.;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += GB)
        v += *reinterpret_cast<volatile const double *>(partial + k);
    __syncthreads();  // block_sum1's shared slots are reused
    const double sum = block_sum1(v);
    if (threadIdx.x == 0) {
        ctl->arrived = 0;
        gf_decide(sum / (double)(N * N), ctl);
    }
}

// the multiplier of the gauge-fixing step on the DFT grid (GaugeFix.cpp:118-130)
__global__ void k_gf_green(int N, const double *sin_half, double *green) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N * N) return;
    const int i = (p / N + N / 2) % N, j = (p % N + N / 2) % N;  // centred index
    const double kx = sin_half[i], ky = sin_half[j];
    const double kt2 = 4. * __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
    green[p] = -1.5 * (1. / (kt2 + 1e-9));
}

__global__ void __launch_bounds__(GB_HEAVY) k_gf_exp(const double2 *chi, int N, C<double> *G,
                                                     GaugeFixCtl *ctl) {
    if (ctl->done) return;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * GB_HEAVY + threadIdx.x;
    if (pos >= n) return;
    const double2 p0 = chi[pos], p1 = chi[n + pos], p2 = chi[2 * n + pos], p3 = chi[3 * n + pos];
    const double d0 = p0.x, d1 = p0.y, d2 = -(d0 + d1);
    // M = i chi for the Hermitian chi: i (x + i y) = (-y, x)
    M3<double> M;
    M.m[0] = {0., d0};
    M.m[4] = {0., d1};
    M.m[8] = {0., d2};
    M.m[1] = {-p1.y, p1.x};
    M.m[3] = {p1.y, p1.x};  // i conj(chi_01)
    M.m[2] = {-p2.y, p2.x};
    M.m[6] = {p2.y, p2.x};
    M.m[5] = {-p3.y, p3.x};
    M.m[7] = {p3.y, p3.x};
    M3<double> g = reunitarize(expm_pade6(M));
    // GaugeFix.cpp:143-147: a NaN in entry (0, 2) resets the site to 1
    if (isnan(g.m[2].r) || isnan(g.m[2].i)) {
        set_identity(g);
        atomicAdd(&ctl->nan_sites, 1);
    }
    st_m3(G, pos, n, g);
}

__global__ void __launch_bounds__(GB_HEAVY) k_gf_transform(State<double> s, const C<double> *G,
                                                           int N, const GaugeFixCtl *ctl) {
    if (ctl->done) return;
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * GB_HEAVY + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / N), iy = (int)(pos % N);
    const size_t px = (size_t)((ix + 1) % N) * N + iy;
    const size_t py = (size_t)ix * N + (iy + 1) % N;
    const M3<double> g = ld_m3(G, pos, n);
    st_m3(s.ux, pos, n, mul_nd(mul(g, ld_m3(s.ux, pos, n)), ld_m3(G, px, n)));
    st_m3(s.uy, pos, n, mul_nd(mul(g, ld_m3(s.uy, pos, n)), ld_m3(G, py, n)));
    st_h8(s.e1, pos, n, conj_h(g, ld_h8(s.e1, pos, n)));
    st_h8(s.e2, pos, n, conj_h(g, ld_h8(s.e2, pos, n)));
    st_h(s.phi, pos, n, conj_h(g, ld_h(s.phi, pos, n)));
    st_h(s.pi, pos, n, conj_h(g, ld_h(s.pi, pos, n)));
}

int gauge_fix_blocks(int N) {
    const size_t n = (size_t)N * N;
    const size_t b = (n + GB - 1) / GB;
    return (int)(b < (size_t)kGaugeBlocks ? b : (size_t)kGaugeBlocks);
}

void launch_gauge_green(int N, const double *sin_half, double *green, cudaStream_t st) {
    const int n = N * N;
    k_gf_green<<<(n + 255) / 256, 256, 0, st>>>(N, sin_half, green);
}

void launch_gauge_fix_iteration(const GaugeFixArgs &a, cudaStream_t st) {
    const size_t n = (size_t)a.N * a.N;
    const int blocks = gauge_fix_blocks(a.N);
    const unsigned heavy = (unsigned)((n + GB_HEAVY - 1) / GB_HEAVY);
    k_gf_chi<<<blocks, GB, 0, st>>>(a.s, a.N, a.chi, a.partial, a.ctl);
    launch_poisson_sheets(a.fft, 1, st);  // chi -> chi in place, skipped when done
    k_gf_exp<<<heavy, GB_HEAVY, 0, st>>>(a.chi, a.N, a.G, a.ctl);
    k_gf_transform<<<heavy, GB_HEAVY, 0, st>>>(a.s, a.G, a.N, a.ctl);
}

// -------------------------------------------------------------------------
// multiplicity
// -------------------------------------------------------------------------

// planes: 0 E1 (d0 + i d1), 1-3 E1 o01 o02 o12, 4-7 the same for E2, 8 pi
// (d0 + i d1), 9-11 pi's upper triangle, 12 pi d2, 13-15 zero
__global__ void __launch_bounds__(GB) k_mult_pack(State<double> s, int N, double2 *planes) {
    const size_t n = (size_t)N * N;
    const size_t pos = (size_t)blockIdx.x * GB + threadIdx.x;
    if (pos >= n) return;
    const double *e[2] = {s.e1, s.e2};
    for (int f = 0; f < 2; f++) {
        const double *p = e[f];
        planes[(4 * f + 0) * n + pos] = make_double2(p[0 * n + pos], p[1 * n + pos]);
        planes[(4 * f + 1) * n + pos] = make_double2(p[2 * n + pos], p[3 * n + pos]);
        planes[(4 * f + 2) * n + pos] = make_double2(p[4 * n + pos], p[5 * n + pos]);
        planes[(4 * f + 3) * n + pos] = make_double2(p[6 * n + pos], p[7 * n + pos]);
    }
    const double *p = s.pi;
    planes[8 * n + pos] = make_double2(p[0 * n + pos], p[1 * n + pos]);
    planes[9 * n + pos] = make_double2(p[3 * n + pos], p[4 * n + pos]);
    planes[10 * n + pos] = make_double2(p[5 * n + pos], p[6 * n + pos]);
    planes[11 * n + pos] = make_double2(p[7 * n + pos], p[8 * n + pos]);
    planes[12 * n + pos] = make_double2(p[2 * n + pos], 0.);
    planes[13 * n + pos] = make_double2(0., 0.);
    planes[14 * n + pos] = make_double2(0., 0.);
    planes[15 * n + pos] = make_double2(0., 0.);
}

namespace {

__device__ __forceinline__ C<double> ld_c(const double2 *pl, size_t idx) {
    const double2 v = pl[idx];
    return {v.x, v.y};
}
__device__ __forceinline__ double abs2(C<double> z) { return z.r * z.r + z.i * z.i; }

// real fields a, b packed as Z = a + i b: A(k) = (Z(k) + conj Z(-k)) / 2,
// B(k) = (Z(k) - conj Z(-k)) / (2i)
__device__ __forceinline__ void unpack2(C<double> zk, C<double> zm, C<double> &A, C<double> &B) {
    A = {0.5 * (zk.r + zm.r), 0.5 * (zk.i - zm.i)};
    B = {0.5 * (zk.i + zm.i), -0.5 * (zk.r - zm.r)};
}

// sum_ij |F_ij(k)|^2 of a Hermitian field from its four (E) or five (pi)
// planes at k and -k
__device__ __forceinline__ double herm_power(const double2 *pl, int first, size_t n, size_t pk,
                                             size_t pm, bool traceless) {
    C<double> D0, D1, D2;
    unpack2(ld_c(pl, first * n + pk), ld_c(pl, first * n + pm), D0, D1);
    double t;
    if (traceless) {
        D2 = {-(D0.r + D1.r), -(D0.i + D1.i)};
        t = abs2(D0) + abs2(D1) + abs2(D2);
    } else {
        C<double> X;
        unpack2(ld_c(pl, 12 * n + pk), ld_c(pl, 12 * n + pm), D2, X);
        t = abs2(D0) + abs2(D1) + abs2(D2);
    }
    for (int q = 1; q <= 3; q++)
        t += abs2(ld_c(pl, (first + q) * n + pk)) + abs2(ld_c(pl, (first + q) * n + pm));
    return t;
}

}  // namespace

__global__ void __launch_bounds__(GB) k_mult_bins(const double2 *planes, MultArgs m,
                                                  double *partial) {
    __shared__ double sN[kKtBins], sE[kKtBins];
    __shared__ int sC[kKtBins];
    for (int b = threadIdx.x; b < kKtBins; b += GB) {
        sN[b] = 0.;
        sE[b] = 0.;
        sC[b] = 0;
    }
    __syncthreads();
    const int N = m.N;
    const size_t n = (size_t)N * N;
    const double dkt = 2.83 / (double)kKtBins;
    const double NN = (double)(N * N);
    double dN = 0., dE = 0.;
    for (size_t p = (size_t)blockIdx.x * GB + threadIdx.x; p < n; p += (size_t)gridDim.x * GB) {
        const int mx = (int)(p / N), my = (int)(p % N);
        const int i = (mx + N / 2) % N, j = (my + N / 2) % N;  // the reference's loop indices
        if (i == 0 || j == 0) continue;
        const double sx = m.sin_half[i], sy = m.sin_half[j];
        const double kt2 = 4. * __dadd_rn(__dmul_rn(sx, sx), __dmul_rn(sy, sy));
        const double omega2 = kt2;
        double nk[3] = {0., 0., 0.};
        if (omega2 != 0) {
            const size_t pm = (size_t)((N - mx) % N) * N + (N - my) % N;
            const double w = 2. / sqrt(omega2) / NN;
            nk[0] = w * (m.g * m.g / ((m.it - 0.5) * m.dtau) * herm_power(planes, 0, n, p, pm, true));
            nk[1] = w * (m.g * m.g / ((m.it - 0.5) * m.dtau) * herm_power(planes, 4, n, p, pm, true));
            nk[2] = w * (((m.it - 0.5) * m.dtau) * herm_power(planes, 8, n, p, pm, false));
        }
        const double kt = sqrt(kt2);
        int ik = (int)(kt / dkt) - 1;
        int bin = -1;
        for (int q = 0; q < 3; q++, ik++)
            if (ik >= 0 && ik < kKtBins && kt > ik * dkt && kt <= (ik + 1) * dkt) bin = ik;
        for (int f = 0; f < 3; f++) {
            const double nkt = nk[f];
            dN += nkt;
            dE += nkt * sqrt(omega2) * kHbarcGf / m.a;
            if (bin >= 0) {
                atomicAdd(&sN[bin], nkt / dkt / 2 / M_PI / sqrt(kt2) * 2 * M_PI * sqrt(kt2) * dkt *
                                        N * N / M_PI / M_PI / 2. / 2.);
                atomicAdd(&sE[bin], sqrt(omega2) * kHbarcGf / m.a * nkt / dkt / 2 / M_PI /
                                        sqrt(kt2) * 2 * M_PI * sqrt(kt2) * dkt * N * N / M_PI /
                                        M_PI / 2. / 2.);
            }
        }
        if (bin >= 0) atomicAdd(&sC[bin], 1);
    }
    const double bN = block_sum1(dN);
    __syncthreads();
    const double bE = block_sum1(dE);
    double *out = partial + (size_t)blockIdx.x * kMultRow;
    if (threadIdx.x == 0) {
        out[0] = bN;
        out[1] = bE;
    }
    for (int b = threadIdx.x; b < kKtBins; b += GB) {
        out[2 + b] = sN[b];
        out[2 + kKtBins + b] = sE[b];
        out[2 + 2 * kKtBins + b] = (double)sC[b];
    }
}

// fold the blocks' rows in block order
__global__ void k_mult_fold(const double *partial, int blocks, double *out) {
    for (int k = threadIdx.x; k < kMultRow; k += blockDim.x) {
        double s = 0.;
        for (int b = 0; b < blocks; b++) s += partial[(size_t)b * kMultRow + k];
        out[k] = s;
    }
}

void launch_multiplicity(const State<double> &s, const MultArgs &m, double2 *planes,
                         const WilsonArgs &fft, double *partial, double *out, cudaStream_t st) {
    const size_t n = (size_t)m.N * m.N;
    const unsigned sites = (unsigned)((n + GB - 1) / GB);
    k_mult_pack<<<sites, GB, 0, st>>>(s, m.N, planes);
    launch_fft2_forward(fft, 4, st);
    const int blocks = gauge_fix_blocks(m.N);
    k_mult_bins<<<blocks, GB, 0, st>>>(planes, m, partial);
    k_mult_fold<<<1, 256, 0, st>>>(partial, blocks, out);
}

}  // namespace ipg
