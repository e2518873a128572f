// Colour-charge density maps g^2 mu^2(x) of both nuclei from nucleon
// positions, on the device.
//
// The reference builds g^2 mu^2 in Init::setColorChargeDensity
// (Init.cpp:753-1676) from the summed nucleon thicknesses
// T(x) = sum_k exp(-|x - x_k|^2 / (2 B)) / (2 pi B) (Init.cpp:1052-1062, no
// nucleon substructure) and an IP-Sat Q_s(T) table. The table is outside this
// library; the map here is the Q_s ~ sqrt(T) form
//   Q_s^2 = QsMax^2 T / max T,   g^2 mu^2 = Q_s^2 / QsmuRatio^2 a^2 / hbarc^2 / g^2
// in lattice units (the conversion of Init.cpp:1403-1408).
//
// The Gaussian is separable, so T on the N x N grid is a rank-A product:
// per nucleus, tables gx[k][i] = exp(-(x_i - x_k)^2/2B) and gy[k][j] are
// formed once (A N exponentials instead of A N^2), then every site sums A
// products. The maximum is reduced on a fixed grid of blocks (deterministic).
#include <cstdint>

#include "ipg_internal.h"

namespace ipg {

namespace {
constexpr double kHbarcN = 0.1973269718;  // GeV fm
constexpr int kRB = 256, kRG = 296;
}  // namespace

__global__ void k_nucleon_tables(int N, double L, double B, int A, const double *xyz,
                                 double shift, double *gx, double *gy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A * N) return;
    const int k = t / N, i = t - k * N;
    const double a = L / N;
    const double x = -L / 2. + a * i;
    const double dx = x - xyz[3 * k] - shift, dy = x - xyz[3 * k + 1];
    gx[t] = exp(-dx * dx / (2. * B));
    gy[t] = exp(-dy * dy / (2. * B));
}

// T(i, j) = sum_k gx[k][i] gy[k][j] / (2 pi B); per-block maximum into partial
__global__ void __launch_bounds__(kRB) k_thickness(int N, double B, int A, const double *gx,
                                                   const double *gy, double *T, double *partial) {
    const size_t n = (size_t)N * N;
    double m = 0.;
    for (size_t p = (size_t)blockIdx.x * kRB + threadIdx.x; p < n; p += (size_t)kRG * kRB) {
        const int i = (int)(p / N), j = (int)(p % N);
        double s = 0.;
        for (int k = 0; k < A; k++) s += gx[(size_t)k * N + i] * gy[(size_t)k * N + j];
        const double t = s / (2. * M_PI * B);
        T[p] = t;
        m = fmax(m, t);
    }
    __shared__ double sh[kRB / 32];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int w = 0; w < kRB / 32; w++) r = fmax(r, sh[w]);
        partial[blockIdx.x] = r;
    }
}

// every block folds the partial maxima (same order everywhere) and scales
__global__ void __launch_bounds__(kRB) k_g2mu_scale(int N, double factor, const double *partial,
                                                    double *T) {
    __shared__ double tmax;
    if (threadIdx.x == 0) {
        double r = 0.;
        for (int b = 0; b < kRG; b++) r = fmax(r, partial[b]);
        tmax = r;
    }
    __syncthreads();
    const size_t n = (size_t)N * N;
    for (size_t p = (size_t)blockIdx.x * kRB + threadIdx.x; p < n; p += (size_t)kRG * kRB) {
        const double rel = tmax > 0. ? T[p] / tmax : 0.;
        T[p] = factor * rel;
    }
}

void launch_g2mu_from_nucleons(const NucleiArgs &a, cudaStream_t st) {
    const double B = a.BG * kHbarcN * kHbarcN;  // fm^2
    const double lat = a.L / a.N;
    // QsMax^2 / QsmuRatio^2 a^2 / hbarc^2 / g^2 times T / max T
    const double factor = a.QsMax * a.QsMax / (a.QsmuRatio * a.QsmuRatio) * lat * lat /
                          (kHbarcN * kHbarcN) / (a.g * a.g);
    const int t = a.A * a.N;
    k_nucleon_tables<<<(t + 255) / 256, 256, 0, st>>>(a.N, a.L, B, a.A, a.xyz, a.shift, a.gx,
                                                       a.gy);
    k_thickness<<<kRG, kRB, 0, st>>>(a.N, B, a.A, a.gx, a.gy, a.out, a.partial);
    k_g2mu_scale<<<kRG, kRB, 0, st>>>(a.N, factor, a.partial, a.out);
}

}  // namespace ipg

namespace ipg {

// ===========================================================================
// IP-Sat colour-charge maps (Init::setColorChargeDensity, Init.cpp:753-1676,
// with the nucleon Gaussians of Init.cpp:1009-1106, the saturation-scale
// table lookup Init::getNuclearQs2, Init.cpp:686-749, and the
// fluctuating-x fixed point of Init.cpp:1219-1410).
//
// Every product, quotient and sum is rounded on its own, in the reference's
// order (__dmul_rn / __ddiv_rn / __dadd_rn, no contraction), so the maps
// agree with the reference's -O2 build up to its transcendentals.
// ===========================================================================
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }

// Q_s^2(T, y) from the table (Init.cpp:686-749): linear in T and in y
__device__ double table_qs2(const IpsatArgs &A, double T, double y, int *flags) {
    const int ny = A.ny, nT = A.nT;
    int posy = (int)floor(ad(dv(y, A.dy), 0.0000001));
    if (y > mul((double)ny, A.dy)) {
        atomicOr(flags, 1);  // y beyond the table
        return 0.;
    }
    posy = min(max(posy, 0), ny - 2);
    const double fracy = dv(sb(y, mul((double)posy, A.dy)), A.dy);
    const double *Q = A.qs2;
    if (T > A.Tlist[nT - 1]) {
        atomicOr(flags, 2);  // T beyond the table: its last row (a warning in the reference)
        return ad(mul(fracy, Q[(size_t)(nT - 1) * ny + posy + 1]),
                  mul(sb(1., fracy), Q[(size_t)(nT - 1) * ny + posy]));
    }
    if (T < A.Tlist[0]) return 0.;
    // the row iT with Tlist[iT] <= T < Tlist[iT + 1] (the table is increasing)
    int lo = 0, hi = nT - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (A.Tlist[mid] <= T) lo = mid;
        else hi = mid;
    }
    if (!(T >= A.Tlist[lo] && T < A.Tlist[lo + 1])) {
        // no row brackets T (T equal to the last entry): the last row
        return ad(mul(fracy, Q[(size_t)(nT - 1) * ny + posy + 1]),
                  mul(sb(1., fracy), Q[(size_t)(nT - 1) * ny + posy]));
    }
    const double fracT = dv(sb(T, A.Tlist[lo]), sb(A.Tlist[lo + 1], A.Tlist[lo]));
    const double down = ad(mul(fracT, Q[(size_t)(lo + 1) * ny + posy]),
                           mul(sb(1., fracT), Q[(size_t)lo * ny + posy]));
    const double up = ad(mul(fracT, Q[(size_t)(lo + 1) * ny + posy + 1]),
                         mul(sb(1., fracT), Q[(size_t)lo * ny + posy + 1]));
    return ad(mul(fracy, up), mul(sb(1., fracy), down));
}

// g^2 mu^2 in lattice units from Q_s (Init.cpp:1289-1293)
__device__ __forceinline__ double g2mu_of(const IpsatArgs &A, double Qs, double ratio) {
    double v = mul(Qs, Qs);
    v = dv(v, ratio);
    v = dv(v, ratio);
    v = mul(v, A.a);
    v = mul(v, A.a);
    v = dv(v, kHbarcN);
    v = dv(v, kHbarcN);
    v = dv(v, A.g);
    return dv(v, A.g);
}

// The fluctuating-x fixed point of one nucleus at one site from the start
// rapidity y0 and start Q_s (Init.cpp:1263-1311); sign = +1 for A (exp(yIn)),
// -1 for B (exp(-yIn)). Returns g^2 mu^2 and leaves the final rapidity in
// *y_end. The reference loops until |dY| <= 0.001; here at most 1000 times.
__device__ double fluct_x(const IpsatArgs &A, double T, double ratio, double sign, double y0,
                          double Qs, double *y_end, int *flags, double *qs_end = nullptr) {
    const double eyin = exp(mul(sign, A.rapidity));
    const double exponent = 5.6;  // 1212.2974 Eq. (17)
    double yl = y0, ydev = 10000., g2 = 0.;
    int it = 0;
    while (fabs(ydev) > 0.001) {
        if (++it > 1000) {
            atomicOr(flags, 4);
            break;
        }
        if (yl >= 0) {
            Qs = sqrt(table_qs2(A, T, fabs(yl), flags));
        } else {
            const double xv = mul(dv(mul(Qs, A.xfactor), A.roots), eyin);
            if (xv == 0) Qs = 0.;
            else
                Qs = mul(sqrt(table_qs2(A, T, 0., flags)),
                         sqrt(mul(pow(dv(sb(1., xv), sb(1., 0.01)), exponent),
                                  pow(dv(0.01, xv), 0.2))));
        }
        if (Qs == 0) {
            ydev = 0.;
            g2 = 0.;
        } else {
            g2 = g2mu_of(A, Qs, ratio);
            const double ynew = log(dv(0.01, mul(dv(mul(Qs, A.xfactor), A.roots), eyin)));
            ydev = sb(yl, ynew);
            yl = ynew;
        }
    }
    *y_end = yl;
    if (qs_end) *qs_end = Qs;
    return g2 != g2 ? 0. : g2;
}

// distance of the site from the nearest nucleon centre implied by T
// (Init.cpp:1236-1262), fm
__device__ __forceinline__ double nucleon_distance(const IpsatArgs &A, double T) {
    const double l = log(mul(mul(mul(2., M_PI), A.BG), T));
    if (l < 0.) {
        if (isinf(l)) return ad(A.rmax, 1.);
        return mul(sqrt(mul(mul(-2., A.BG), l)), kHbarcN);
    }
    return 0.;
}

}  // namespace

// T_A, T_B: the nucleon Gaussians summed in nucleon order (Init.cpp:1009-1106,
// no constituent quarks): sqrt(1 + xi) exp(-b^2/(2 BG)) / (2 pi BG) g_i with
// b^2 = (dx^2 + dy^2 + xi (dx cos phi + dy sin phi)^2) / hbarc^2
__global__ void k_ipsat_thickness(IpsatArgs A) {
    const size_t n = (size_t)A.N * A.N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int ix = (int)(pos / A.N), iy = (int)(pos % A.N);
    const double x = ad(-A.L / 2., mul(A.a, (double)ix));
    const double y = ad(-A.L / 2., mul(A.a, (double)iy));
    const double h2 = mul(kHbarcN, kHbarcN);
    const double sx = sqrt(ad(1., A.xi));
    const double den = mul(mul(2., M_PI), A.BG);
    for (int nuc = 0; nuc < 2; nuc++) {
        const double *p = nuc ? A.nucB : A.nucA;
        const int cnt = nuc ? A.nB : A.nA;
        double tp = 0.;
        for (int i = 0; i < cnt; i++) {
            const double xm = p[4 * i], ym = p[4 * i + 1], phi = p[4 * i + 2],
                         gn = p[4 * i + 3];
            const double dx = sb(xm, x), dy = sb(ym, y);
            const double pr = ad(mul(dx, cos(phi)), mul(dy, sin(phi)));
            double bp2 = ad(ad(mul(dx, dx), mul(dy, dy)), mul(A.xi, pow(pr, 2.)));
            bp2 = dv(bp2, h2);
            double T = mul(sx, exp(dv(-bp2, mul(2., A.BG))));
            T = mul(dv(T, den), gn);
            tp = ad(tp, dv(T, A.nuclei_in_average));
        }
        (nuc ? A.TB : A.TA)[pos] = tp;
    }
}

// inside flags (both nucleon distances below Rmax, Init.cpp:1263-1270), B's
// fixed point (it starts from the configured rapidity at every site), and
// the non-fluctuating maps
__global__ void k_ipsat_b(IpsatArgs A) {
    const size_t n = (size_t)A.N * A.N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const double TA = A.TA[pos], TB = A.TB[pos];
    const bool in = nucleon_distance(A, TA) < A.rmax && nucleon_distance(A, TB) < A.rmax;
    A.inside[pos] = in;
    A.g2A[pos] = 0.;
    A.g2B[pos] = 0.;
    if (!in) return;
    if (A.fluct_x) {
        if (A.rapidity < 0) atomicOr(A.flags, 8);  // B's first step uses a carried Q_s
        double yend;
        A.g2B[pos] = fluct_x(A, TB, A.ratioB, -1., A.rapidity, 1., &yend, A.flags);
        A.yB[pos] = yend;
    } else {
        A.g2A[pos] = dv(dv(dv(dv(mul(mul(dv(dv(table_qs2(A, TA, A.rapidity, A.flags), A.ratioA),
                                                   A.ratioA),
                                                A.a),
                                            A.a),
                                        kHbarcN),
                                     kHbarcN),
                                  A.g),
                              A.g);
        A.g2B[pos] = dv(dv(dv(dv(mul(mul(dv(dv(table_qs2(A, TB, A.rapidity, A.flags), A.ratioB),
                                                   A.ratioB),
                                                A.a),
                                            A.a),
                                        kHbarcN),
                                     kHbarcN),
                                  A.g),
                              A.g);
    }
}

// previous inside site in raster order, per row (one warp a row): prev[pos]
// = largest inside index < pos within the row, or -1
__global__ void k_ipsat_prev_row(IpsatArgs A) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= A.N) return;
    int carry = -1;
    for (int j0 = 0; j0 < A.N; j0 += 32) {
        const int j = j0 + lane;
        const size_t pos = (size_t)row * A.N + j;
        const int own = (j < A.N && A.inside[pos]) ? (int)pos : -1;
        // inclusive max scan over the lanes
        int v = own;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v = max(v, u);
        }
        int excl = __shfl_up_sync(0xffffffffu, v, 1);
        if (lane == 0) excl = -1;
        excl = max(excl, carry);
        if (j < A.N) A.prev[pos] = excl;
        carry = max(carry, __shfl_sync(0xffffffffu, v, 31));
    }
}

// across rows: a row's first entries see the last inside site of earlier rows
__global__ void k_ipsat_prev_rows(IpsatArgs A) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int last = -1;
    for (int r = 0; r < A.N; r++) {
        const size_t base = (size_t)r * A.N;
        int row_last = -1;
        for (int j = A.N - 1; j >= 0; j--)
            if (A.inside[base + j]) {
                row_last = (int)(base + j);
                break;
            }
        A.row_last[r] = last;
        if (row_last >= 0) last = row_last;
    }
}

// A's fixed point: with the reference's single-threaded loop the rapidity
// variable is not reset before A, so it starts from B's final rapidity at
// the previous inside site (Init.cpp:1219-1312), or the configured rapidity
// at the first one
__global__ void k_ipsat_a(IpsatArgs A) {
    const size_t n = (size_t)A.N * A.N;
    const size_t pos = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n || !A.inside[pos] || !A.fluct_x) return;
    int p = A.prev[pos];
    if (p < 0) p = A.row_last[pos / A.N];
    const double y0 = p >= 0 ? A.yB[p] : A.rapidity;
    if (y0 < 0) {
        atomicOr(A.flags, 8);  // A's first step uses the carried Q_s: sequential pass
        return;
    }
    double yend;
    A.g2A[pos] = fluct_x(A, A.TA[pos], A.ratioA, 1., y0, 1., &yend, A.flags);
}

// Both fixed points in the reference's single-threaded order, carrying the
// rapidity and Q_s of each nucleus from site to site (only needed when a
// start rapidity is negative).
__global__ void k_ipsat_sequential(IpsatArgs A) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const size_t n = (size_t)A.N * A.N;
    double yl = A.rapidity, QsA = 1., QsB = 1.;
    for (size_t pos = 0; pos < n; pos++) {
        if (!A.inside[pos]) continue;
        double yend;
        A.g2A[pos] = fluct_x(A, A.TA[pos], A.ratioA, 1., yl, QsA, &yend, A.flags, &QsA);
        A.g2B[pos] = fluct_x(A, A.TB[pos], A.ratioB, -1., A.rapidity, QsB, &yend, A.flags, &QsB);
        yl = yend;
    }
}

// Event averages of setColorChargeDensity (Init.cpp:1423-1520): over the
// cells within sqrt(0.1 sigma_NN / pi) of a collided nucleon of each nucleus
// the means of max/avg/min of Q_sA^2, Q_sB^2 (and of max Q_s), over all cells
// but the first and last the sum of min(Q_sA^2, Q_sB^2), and T_pp. Each block
// writes 8 partial sums (sum Qs_max, Qs2_max, Qs2_min, Qs2_avg, count,
// Qs2_min over all cells, Tpp, -), folded in order on the host.
__global__ void __launch_bounds__(kRB) k_ipsat_averages(IpsatArgs A, const double *colA,
                                                         const double *colB, double r_cut,
                                                         double *partial) {
    const size_t n = (size_t)A.N * A.N;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t pos = (size_t)blockIdx.x * kRB + threadIdx.x; pos < n;
         pos += (size_t)kRG * kRB) {
        const int ix = (int)(pos / A.N), iy = (int)(pos % A.N);
        const double x = ad(-A.L / 2., mul(A.a, (double)ix));
        const double y = ad(-A.L / 2., mul(A.a, (double)iy));
        const bool in_range = pos > 0 && pos < (size_t)(A.N - 1) * A.N + A.N - 1;
        const double gA = in_range ? A.g2A[pos] : 0., gB = in_range ? A.g2B[pos] : 0.;
        // lattice g^2 mu^2 back to Q_s^2 in GeV^2
        auto qs2 = [&](double g2, double ratio) {
            double v = mul(g2, ratio);
            v = mul(v, ratio);
            v = dv(v, A.a);
            v = dv(v, A.a);
            v = mul(v, kHbarcN);
            v = mul(v, kHbarcN);
            v = mul(v, A.g);
            return mul(v, A.g);
        };
        const double qA = qs2(gA, A.ratioA), qB = qs2(gB, A.ratioB);
        acc[5] += gB >= gA ? qA : qB;
        int check = 0;
        for (int i = 0; i < A.nA && check == 0; i++) {
            if (colA[3 * i + 2] == 0.) continue;
            const double dx = sb(x, colA[3 * i]), dy = sb(y, colA[3 * i + 1]);
            if (sqrt(ad(mul(dx, dx), mul(dy, dy))) < r_cut) check = 1;
        }
        if (check == 1)
            for (int i = 0; i < A.nB; i++) {
                if (colB[3 * i + 2] == 0.) continue;
                const double dx = sb(x, colB[3 * i]), dy = sb(y, colB[3 * i + 1]);
                if (sqrt(ad(mul(dx, dx), mul(dy, dy))) < r_cut) {
                    check = 2;
                    break;
                }
            }
        if (check == 2) {
            const double qmax = gB > gA ? qB : qA, qmin = gB > gA ? qA : qB;
            acc[0] += sqrt(qmax);
            acc[1] += qmax;
            acc[2] += qmin;
            acc[3] += dv(ad(mul(mul(gB, A.ratioB), A.ratioB), mul(mul(gA, A.ratioA), A.ratioA)),
                         2.) / A.a / A.a * kHbarcN * kHbarcN * A.g * A.g;
            acc[4] += 1.;
        }
        acc[6] += A.TB[pos] * A.TA[pos] * A.a * A.a / kHbarcN / kHbarcN / kHbarcN / kHbarcN;
    }
    __shared__ double sh[8][kRB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double v = 0.;
        for (int w = 0; w < kRB / 32; w++) v += sh[threadIdx.x][w];
        partial[(size_t)blockIdx.x * 8 + threadIdx.x] = v;
    }
}

void launch_ipsat_averages(const IpsatArgs &a, const double *colA, const double *colB,
                           double r_cut, double *partial, cudaStream_t st) {
    k_ipsat_averages<<<kRG, kRB, 0, st>>>(a, colA, colB, r_cut, partial);
}

void launch_ipsat(const IpsatArgs &a, bool sequential, cudaStream_t st) {
    const size_t n = (size_t)a.N * a.N;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    if (!sequential) {
        k_ipsat_thickness<<<blocks, 128, 0, st>>>(a);
        k_ipsat_b<<<blocks, 128, 0, st>>>(a);
        if (a.fluct_x) {
            k_ipsat_prev_row<<<(a.N + 7) / 8, 256, 0, st>>>(a);
            k_ipsat_prev_rows<<<1, 32, 0, st>>>(a);
            k_ipsat_a<<<blocks, 128, 0, st>>>(a);
        }
    } else {
        k_ipsat_sequential<<<1, 32, 0, st>>>(a);
    }
}

}  // namespace ipg
