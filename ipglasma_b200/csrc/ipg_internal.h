// Internal declarations shared by the CUDA translation units of the library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fields.cuh"

namespace ipg {

// Per-event constants visible to kernels (one entry per event of a batch).
struct EventGeom {
    int N;         // sites per side
    int Ny;        // longitudinal sheets
    double a;      // lattice spacing, fm
    double g;      // coupling
    double m_lat;  // IR mass in lattice units (m a / hbar c)
    double uvdamp_lat;
};

template <typename T>
struct StepCoef {
    T tau;    // current time (lattice units)
    T dt_pe;  // time step used for the pi and E updates
    T dt_pu;  // time step used for the phi and U updates
    T g;
    int do_pe;
    int do_pu;
    // derived on the host by set_derived, in T arithmetic (the FP32 kernels
    // read these instead of dividing per thread)
    T c_e;    // tau dt_pe / (2 g^2): staple term of E
    T c_pi;   // dt_pe / tau: bracket term of pi and commutator term of E
    T c_u;    // g^2 dt_pu / (tau + dt_pu/2): the U update's X = i c_u E
    T c_phi;  // (tau + dt_pu/2) dt_pu: the phi update
};

template <typename T>
inline void set_derived(StepCoef<T> &cf) {
    cf.c_e = cf.tau * cf.dt_pe / (T(2) * cf.g * cf.g);
    cf.c_pi = cf.dt_pe / cf.tau;
    cf.c_u = cf.g * cf.g * cf.dt_pu / (cf.tau + cf.dt_pu / T(2));
    cf.c_phi = (cf.tau + cf.dt_pu / T(2)) * cf.dt_pu;
}

// status (may be null): set to 1 if a wait of the FP32 tile kernel hit its
// limit (the step is then incomplete)
template <typename T>
void launch_leapfrog(const EventGeom *d_ev, int N, const State<T> &s,
                     C<T> *ux_out, C<T> *uy_out, T *phi_out,
                     const StepCoef<T> &cf, bool reunit, cudaStream_t st,
                     double *status = nullptr);

// One FP64 step from the state `in` into the separate state `out` (all six
// fields written; `in` is left unchanged)
void launch_leapfrog_into(const EventGeom *d_ev, int N, const State<double> &in,
                          const State<double> &out, const StepCoef<double> &cf, cudaStream_t st);

// One event of a batched leapfrog launch: its buffers for this step and its
// step coefficients (inactive events are skipped).
template <typename T>
struct BatchEvent {
    State<T> s;
    C<T> *ux_out, *uy_out;
    T *phi_out;
    StepCoef<T> cf;
    int N;
    int active;
    int map_sel;  // which of the event's two tensor-map sets holds s (U/phi buffer parity)
};

// Tensor maps of the six input fields of one step (the TMA tile kernels)
struct LoadMaps {
    CUtensorMap ux, uy, phi, e1, e2, pi;
};
// the maps of the TMA tile kernels of precision T (FP32: 8 x 32 tiles, FP64:
// 4 x 32 tiles) for a lattice of N x N sites with the given field planes;
// false if the driver rejects them
template <typename T>
bool encode_step_maps(int N, const State<T> &s, LoadMaps *out);
template <>
bool encode_step_maps<float>(int N, const State<float> &s, LoadMaps *out);
template <>
bool encode_step_maps<double>(int N, const State<double> &s, LoadMaps *out);

// Tile-shape variants of the batched kernel: variant v < batch_plain_variants
// advances tiles of 32 x batch_tile_rows(v) sites with plain loads, one
// thread per site; the last variant (v = batch_plain_variants) runs the TMA
// tile kernel of the single-event form over the concatenated tile lists,
// with per-event tensor maps (d_maps[2 e + map_sel]).
template <typename T>
constexpr int batch_plain_variants() {
    return sizeof(T) == 4 ? 3 : 2;
}
template <typename T>
constexpr int batch_variants() {
    return batch_plain_variants<T>() + 1;
}
template <typename T>
int batch_tile_rows(int variant);
template <typename T>
int batch_max_blocks_per_sm(int variant, int n_events);
// tile_begin[n_events + 1]: prefix sums of (N/32) (N/rows) per event;
// status (TMA variant): set to 1 if a bounded wait gave up
template <typename T>
void launch_leapfrog_batch(const BatchEvent<T> *d_evs, int n_events, const int *d_tile_begin,
                           int total_tiles, int variant, int grid, const LoadMaps *d_maps,
                           double *status, cudaStream_t st);

// ---- initial conditions -------------------------------------------------

// Colour-charge sheets -> Wilson lines for one nucleus, sheets [k0, k0+ns).
struct WilsonArgs {
    int N;
    int logN;
    int Ny;
    double g;
    const double *g2mu2;     // [n] lattice units
    double *amp;             // [n] scratch: g sqrt(g2mu2 / Ny) (launch_wilson_amp)
    const double *xi;        // [Ny][n][8] unit normals, or null (Philox)
    uint64_t philox_key;     // used when xi == null
    uint32_t nucleus;        // 0 = A, 1 = B (Philox stream selector)
    const double2 *twiddle;  // [N] exp(-2 pi i k / N)
    const double *green;     // [N*N] Poisson multiplier on the DFT grid
    double2 *work;           // [ns][4][n] complex scratch
    C<double> *V;            // [9][n] Wilson line, updated in place
    // when set, the row transform reads this packed field ([ns][4][n], colour
    // 2c in the real and 2c+1 in the imaginary part of channel c) instead of
    // generating rho (the adjoint runs the self-adjoint Poisson map on it)
    const double2 *rho_in = nullptr;
    int no_product = 0;  // transform only, leave V alone
    // when set and nonzero on the device, the transform kernels return at
    // once (the gauge-fixing loop's stop flag)
    const int *skip = nullptr;
    // the FP32 form's Poisson transforms: work holds float2 values
    // ([ns][4][n]), with twiddle32 and green32 in place of twiddle and green;
    // the exponentials and the Wilson-line products stay FP64
    int fp32 = 0;
    const float2 *twiddle32 = nullptr;
    const float *green32 = nullptr;
};
// Poisson map only (no Wilson-line product) of w.rho_in -> w.work, sheets [0, ns)
void launch_poisson_sheets(const WilsonArgs &w, int ns, cudaStream_t st);
void launch_wilson_sheets(const WilsonArgs &w, int k0, int ns,
                          cudaStream_t st);
// k_wilson alone: V <- exp(-i A_k.t) V for the ns sheets whose A is in w.work
void launch_wilson_product(const WilsonArgs &w, int ns, cudaStream_t st);
// charge amplitude of every site, once per nucleus before its sheets
void launch_wilson_amp(const WilsonArgs &w, cudaStream_t st);
// out[p] = (float)in[p], p < n
void launch_round_to_float(size_t n, const double *in, float *out, cudaStream_t st);

// the device noise of sheets [k0, k0+ns) of one nucleus, as the unit normals
// xi[ns][N*N][8] that k_rows_fwd draws for them
void launch_draw_noise(int N, int k0, int ns, uint64_t key, uint32_t nucleus, double *out,
                       cudaStream_t st);

void launch_green(int N, double m_lat, double uvdamp_lat, double *green,
                  cudaStream_t st);
// unnormalised forward 2-D DFT of the packed planes w.rho_in ([ns][4][n]
// complex) into w.work (the same array may be passed for both)
void launch_fft2_forward(const WilsonArgs &w, int ns, cudaStream_t st);

// ---- Coulomb gauge fixing and gluon multiplicity (gaugefix.cu) ----------

constexpr int kGaugeHistory = 401;  // residuals at iterations 0, 10, ..., 4000
constexpr int kGaugeBlocks = 592;   // reduction blocks (4 per SM)
constexpr int kKtBins = 100;        // k_T bins of Evolution::multiplicity
constexpr int kMultRow = 2 + 3 * kKtBins;  // dN, dE, n[100], E[100], count[100]

// device state of one gauge fixing (the host sets done = iter = nan_sites =
// arrived = 0, prev = 10000 and hist = NaN before the first iteration)
struct GaugeFixCtl {
    int done;       // a stopping rule fired: later iterations do nothing
    int iter;       // gauge transformations applied
    int checks;     // residuals computed
    int nan_sites;  // sites whose transformation was NaN and was reset to 1
    unsigned arrived;  // blocks of the residual pass done (the last one decides)
    double prev;    // residual at the last multiple of 10 iterations
    double last;    // the latest residual
    double hist[kGaugeHistory];
};
struct GaugeFixArgs {
    State<double> s;     // fields, transformed in place
    int N;
    double2 *chi;        // [4][n] packed g, then chi
    C<double> *G;        // [9][n] the transformation of every site
    double *partial;     // [kGaugeBlocks]
    GaugeFixCtl *ctl;
    WilsonArgs fft;      // rho_in = work = chi, green = the gauge multiplier, skip = &ctl->done
};
int gauge_fix_blocks(int N);
// the multiplier -1.5 / (k~^2 + 1e-9) on the DFT grid from sin_half[i] =
// sin(pi (-0.5 + i / N)) (the reference's centred index i)
void launch_gauge_green(int N, const double *sin_half, double *green, cudaStream_t st);
void launch_gauge_fix_iteration(const GaugeFixArgs &a, cudaStream_t st);

struct MultArgs {
    int N;
    int it;            // the step whose fields these are
    double dtau, g, a;  // lattice dtau, coupling, spacing (fm)
    const double *sin_half;  // [N] sin(kx / 2), kx = 2 pi (-0.5 + i / N)
};
// n(k_T) of the fields s: out[kMultRow] = dN, dE, the bin sums of n and E,
// the bin counts (planes: [16][n] complex scratch; partial:
// [kGaugeBlocks][kMultRow])
void launch_multiplicity(const State<double> &s, const MultArgs &m, double2 *planes,
                         const WilsonArgs &fft, double *partial, double *out, cudaStream_t st);

// V_A, V_B -> link products U1, U2 for both directions (Init.cpp:2462-2491)
void launch_link_products(int N, C<double> *VA, C<double> *VB,
                          C<double> *u1x, C<double> *u2x, C<double> *u1y,
                          C<double> *u2y, cudaStream_t st);

struct NewtonArgs {
    int N;
    int max_iter;
    int max_restart;
    uint64_t philox_key;
    const C<double> *u1x, *u2x, *u1y, *u2y;
    C<double> *ux, *uy;  // solutions
    int *iters;          // [2n] iterations used (total over restarts)
    int *status;         // [2n] 0 ok, 1 restarted then converged, 2 failed
    double tol;          // stop when sum_a |F_a| < tol (reference: 1e-6)
    double *alpha;       // [8][2n] the solution's exponent (may be null)
    int mode = 0;        // 0: the reference's iteration; 1: Newton on the group
    int redo_only = 0;   // (internal) run only the links whose status is -1
};
void launch_newton(const NewtonArgs &a, cudaStream_t st);

// Initial longitudinal field pi from the "minus" stencil (Init.cpp:2521-2584,
// 2664-2681).
void launch_initial_pi(int N, double g, const C<double> *u1x,
                       const C<double> *u2x, const C<double> *u1y,
                       const C<double> *u2y, const C<double> *ux,
                       const C<double> *uy, double *pi, cudaStream_t st);

// g2mu2 of one nucleus from its nucleon positions (nuclei.cu)
struct NucleiArgs {
    int N;
    double L, BG, QsMax, QsmuRatio, g;
    int A;               // nucleons
    const double *xyz;   // [A][3] fm, device
    double shift;        // added to x (fm)
    double *gx, *gy;     // [A][N] scratch
    double *partial;     // [296] scratch
    double *out;         // [N*N] g2mu2, lattice units
};
void launch_g2mu_from_nucleons(const NucleiArgs &a, cudaStream_t st);

// IP-Sat maps of both nuclei (nuclei.cu): nucleon thickness, saturation-scale
// table, fluctuating-x fixed point
struct IpsatArgs {
    int N;
    double L, a, g;
    double BG;                 // nucleon width, GeV^-2
    double xi;                 // proton anisotropy
    double nuclei_in_average;  // averageOverNuclei
    double ratioA, ratioB;     // QsmuRatio of A and B
    double rapidity, roots, xfactor, rmax;
    int fluct_x;               // useFluctuatingx
    int nA, nB;
    const double *nucA, *nucB;  // [n][4]: x, y (shifted by -+b/2), phi, Q_s normalisation
    int nT, ny;
    double dy;
    const double *Tlist;  // [nT]
    const double *qs2;    // [nT][ny]
    double *TA, *TB;      // [N*N] thickness, GeV^2
    double *g2A, *g2B;    // [N*N] g^2 mu^2, lattice units
    double *yB;           // [N*N] B's final rapidity
    int *inside, *prev;   // [N*N]
    int *row_last;        // [N]
    int *flags;           // bit 0: y beyond table, 1: T beyond table, 2: no convergence,
                          // 3: a start rapidity < 0 (run the sequential pass)
};
// sequential = false: the parallel passes; true: both fixed points again in
// the single-threaded site order (after the parallel passes flagged bit 3)
void launch_ipsat(const IpsatArgs &a, bool sequential, cudaStream_t st);
// partial[296][8] sums of the event averages; colA/colB: [n][3] x, y (shifted),
// collided flag of each nucleon; r_cut = sqrt(0.1 sigma_NN / pi) fm
void launch_ipsat_averages(const IpsatArgs &a, const double *colA, const double *colB,
                           double r_cut, double *partial, cudaStream_t st);

// ---- observables ----------------------------------------------------------

struct TmunuArgs {
    int N;
    double g;
    double tau;  // lattice units (it * dtau)
    double a;
    State<double> s;
    double *T10;  // [10][n]: tautau xx yy etaeta taux tauy taueta xy xeta yeta
    // from32: read the FP32 form's state s32 instead (links stored as U - 1),
    // widened to FP64 on load; the arithmetic stays FP64
    State<float> s32{};
    int from32 = 0;
};
void launch_tmunu(const TmunuArgs &a, cudaStream_t st);
// T^tautau, T^xx, T^yy, T^etaeta only
void launch_tmunu_diag(const TmunuArgs &a, cudaStream_t st);

// ---- adjoint ---------------------------------------------------------------
// Adjoint buffers of the six fields, each sized as 9 complex planes and
// holding 18 real planes (entry k: real part in plane 2k, imaginary in 2k+1).
template <typename T>
struct AdjStateT {
    C<T> *ux, *uy, *e1, *e2, *phi, *pi;
};
using AdjState = AdjStateT<double>;
// time reversal of one FP64 step: state after (nxt) -> state before (cur)
void launch_inverse_step(int N, const State<double> &nxt, const State<double> &cur,
                         const StepCoef<double> &cf, cudaStream_t st);
// E and pi of the step's input from its output nxt and the recovered U, phi
// in cur (evolve.cu; FP64, full links)
template <typename T>
void launch_inverse_se(int N, const State<T> &nxt, const State<T> &cur,
                       const StepCoef<double> &cf, cudaStream_t st);
// the time reversal nxt -> cur and the adjoint step together (the U/phi
// reversal fused with the S_u adjoint, then the E/pi reversal and the S_e
// adjoint; same results as launch_inverse_step then launch_adjoint_step; FP64)
template <typename T>
void launch_inverse_adjoint_step(int N, const State<T> &nxt, const State<T> &cur,
                                 const AdjStateT<T> &a, const StepCoef<double> &cf,
                                 cudaStream_t st);
// adjoints of a step's outputs -> adjoints of its inputs (in place); cur is the
// state before the step, nxt the state after it. T = double, or float for the
// FP32 adjoint (the FP32 bulk form's states, links as W = U - 1; adjoints in
// FP32; the step differentiated is the plain form's, without the
// reunitarisation)
template <typename T>
void launch_adjoint_step(int N, const State<T> &cur, const State<T> &nxt, const AdjStateT<T> &a,
                         const StepCoef<double> &cf, cudaStream_t st);
// tbar[n] = dL/dTtt (lattice units) -> field adjoints (accumulated)
template <typename T>
void launch_adjoint_ttt(int N, const State<T> &s, const T *tbar, const AdjStateT<T> &a, double g,
                        double tau, cudaStream_t st);
template <typename T>
void launch_adjoint_project(size_t n, const AdjStateT<T> &a, cudaStream_t st);
// FP32 adjoint buffers -> FP64 ones (for the initial-condition adjoint)
void launch_adjoint_widen(size_t n, const AdjStateT<float> &src, const AdjState &dst,
                          cudaStream_t st);
// adjoint buffer (18 real planes) -> [n][18] doubles, (re, im) per entry
void launch_planes_to_sites(size_t n, const C<double> *src, double *dst, cudaStream_t st);
// adjoint of the tau = 0 links and pi: pi_bar, U_bar(tau=0) (in adj) ->
// U1/U2 adjoints b* (initial-pi stencil, then the Newton solve) -> V_A, V_B
// adjoints vbA, vbB (link products); b* and vb* must start at zero
struct AdjInitArgs {
    int N;
    double g;
    const C<double> *u1x, *u2x, *u1y, *u2y, *ux, *uy, *VA, *VB;
    const double *alpha;  // [8][2n] Newton exponents
    AdjState adj;
    C<double> *b1x, *b2x, *b1y, *b2y, *vbA, *vbB;
};
void launch_adjoint_init_links(const AdjInitArgs &a, cudaStream_t st);
// one sheet backwards through V_k = exp(-i A_k.t) V_{k-1}; work holds the
// packed A_k on entry and A_bar_k on return
void launch_adjoint_wilson_sheet(int N, double2 *work, C<double> *V, C<double> *Vb,
                                 cudaStream_t st);
// packed rho_bar of sheet k in w.work -> g2mu2_bar (+=) and rho_bar [n][8]
void launch_adjoint_rho(const WilsonArgs &w, int k, double *g2mu_bar, double *rho_out,
                        cudaStream_t st);

struct LandauArgs {
    int N;
    double tau_fm;        // it * dtau * a
    double tau2_fm;       // a * it * dtau * a * it * dtau (MyEigen.cpp:101)
    double tau_fm_parts[3];  // it, dtau, a (for eps/3/it/dtau/a/it/dtau/a)
    const double *T10;
    double *eps;     // [n]
    double *u4;      // [4][n]
    double *pi10;    // [10][n]
    int *found;      // [n]
};
void launch_landau(const LandauArgs &a, double *carry, int *wrote,
                   cudaStream_t st);

// reductions; out receives the per-event scalars
struct Reductions {
    double gauss_max;
    double unitarity_max;
    double etot;
};
// d_partial needs ceil(N*N/256) * 18 doubles
// (S = float: the FP32 form's state read directly, links as 1 + W, in FP64)
template <typename S>
void launch_gauss_law(int N, const State<S> &s, double *d_partial, double *d_out,
                      cudaStream_t st);
template <typename S>
void launch_unitarity(int N, const C<S> *ux, const C<S> *uy, double *d_partial,
                      double *d_out, cudaStream_t st);
// sums1[5] = {sum x w, sum y w, sum w, sum T^tautau, sum eps},
// sums2[18] = radial moments (see reduce.cu)
void launch_eccentricity(int N, double L, double a, const double *eps,
                         const double *utau, const double *Ttt,
                         double *d_partial, double *d_sums1, double *d_sums2,
                         cudaStream_t st);

// out[8] = {sum x^2 w, sum y^2 w, sum w (all cells), cells with eps >= 0,
// their sum eps, their sum g2mu2A g2mu2B, the largest ix + 1 with w > 0 on
// the centroid's row, the largest iy + 1 on its column} (see reduce.cu)
void launch_eccentricity_extras(int N, double L, double a, const double *eps,
                                const double *utau, const double *g2A, const double *g2B,
                                const double *d_sums1, double *d_partial, double *d_out,
                                cudaStream_t st);

// out[4] = {max iterations, sum of iterations, restarted links, failed links};
// d_partial needs 4 * ceil(links/256) doubles
void launch_newton_stats(size_t links, const int *iters, const int *status,
                         double *d_partial, double *d_out, cudaStream_t st);
// out[2] = {cells without a time-like eigenvector, cells with non-finite e}
void launch_cell_flags(size_t n, const int *found, const double *eps,
                       double *d_partial, double *d_out, cudaStream_t st);

// ---- output files formatted on the GPU (writers_gpu.cu) -------------------
// resampling grid of writers.cpp: lattice N, L, a = L/N; output hx = sizeOutput
// points over hL = LOutput (spacing ha), heta eta slices of deta; proper time
// tau0 = it dtau a
struct OutputGrid {
    int N;
    double L, a;
    int hx, heta;
    double hL, ha, deta;
    int it;
    double dtau, gfactor, tau0;
};
struct OutputFields {
    const double *eps, *u4, *pi10, *T10;  // device, as ipg_get_observables
};
// bytes of the chunk buffer and of the text image for `lines` output lines
size_t output_text_capacity(long long lines);
int output_text_chunks(long long lines);
// kind 0: hydro file lines (heta hx hx, term[line] = the Etot term), kind 1:
// KoMPoST lines (hx hx); text receives the file body, chunk_off[chunks] its
// length; *bad is set when a number needs the host formatter
void launch_output_text(int kind, const OutputGrid &g, const OutputFields &f, long long lines,
                        char *chunks, int *chunk_len, long long *chunk_off, char *text,
                        double *term, int *bad, cudaStream_t st);

template <typename T>
void launch_convert_state(size_t n, const State<T> &src, State<double> &dst,
                          cudaStream_t st);
template <typename T>
void launch_convert_state_down(size_t n, const State<double> &src,
                               State<T> &dst, cudaStream_t st);

}  // namespace ipg
