/*
 * ipglasma_b200 -- C ABI of the B200 implementation of IP-Glasma's per-event
 * hot path: colour-charge sampling -> Poisson solve -> Wilson lines -> tau=0
 * Newton link solve -> boost-invariant leapfrog -> T^{mu nu} and Landau
 * matching.
 *
 * The reference has no plugin or FFI layer; its hot path is entered through
 * two calls in the event loop (main.cpp:347-359):
 *     init.init(&lat, &group, param, random, &glauber, READFROMFILE);
 *     evolution.run(&lat, &group, param);
 * with all state in a Lattice of heap Cells (Lattice.h, Cell.h) and every
 * error ending the process (exit(1)). The entry points below replace those
 * two calls and the Cell getters their callers use; each cites what it
 * replaces.
 *
 * Conventions
 *   - Opaque context, one CUDA stream per context; a context is not
 *     re-entrant, separate contexts may be driven from separate host threads.
 *   - The caller owns host buffers, the library owns device memory.
 *   - Lattice site index pos = ix * N + iy (Lattice.cpp:15-28).
 *   - 3x3 matrices cross the ABI as 9 complex numbers, row-major, (re, im)
 *     pairs: 18 doubles per site, sites in pos order.
 *   - Lattice units as in the reference: g2mu2 is g^2 mu^2 a^2, tau and dtau
 *     are in units of a.
 *   - Every function returns an ipg_status; nothing calls exit().
 */
#ifndef IPGLASMA_B200_H
#define IPGLASMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    IPG_OK = 0,
    IPG_ERR_BAD_CONFIG = 1,        /* invalid configuration or argument */
    IPG_ERR_CUDA = 2,              /* CUDA runtime error (message kept) */
    IPG_ERR_NEWTON_NONCONVERGED = 3, /* some tau=0 links used their best estimate */
    IPG_ERR_NAN = 4,               /* NaN/Inf detected in the fields */
    IPG_ERR_STATE = 5,             /* call out of order */
    IPG_ERR_NOMEM = 6,             /* device allocation failed */
    IPG_ERR_TIMEOUT = 7,           /* a device wait hit its limit */
    IPG_NO_COLLISION = 8           /* the gluon spectrum at it = 1 is zero: the
                                      evolution stopped there, as the reference's
                                      does (Evolution.cpp:655, 3111-3122) */
} ipg_status;

typedef enum {
    IPG_FP64 = 0, /* plain form: FP64 everywhere, no reunitarisation */
    IPG_FP32 = 1  /* bulk form: FP32 leapfrog with per-step reunitarisation,
                     FP64 initial conditions, observables and reductions */
} ipg_precision;

typedef struct ipg_ctx ipg_ctx;

/* Per-event configuration; the keys of the reference input file that the
 * hot path reads (main.cpp:448-578). */
typedef struct {
    int size;          /* N, sites per side: power of two, 8 <= N <= 4096 */
    int Nc;            /* colours, must be 3 */
    int Ny;            /* longitudinal sheets per nucleus */
    double L;          /* transverse box, fm */
    double g;          /* coupling */
    double m;          /* IR regulator, GeV */
    double UVdamp;     /* UV damping, GeV^-1 */
    double maxtime;    /* final proper time, fm */
    double dtau;       /* lattice units; <= 0 derives it like main.cpp:531-534 */
    int precision;     /* ipg_precision */
    int newton_max_iterations; /* 0 -> 2000 (Init.cpp:3345) */
    int newton_max_restarts;   /* 0 -> 200  (Init.cpp:3346) */
    uint64_t seed;     /* key of the device random streams (noise, restarts) */
    int device;        /* CUDA device ordinal */
    double newton_tolerance; /* stop when sum_a |F_a| < this; <= 0 -> 1e-6, the
                                reference's criterion (Init.cpp:3372). The
                                adjoint needs a converged root: use ~1e-12 */
    int newton_mode;   /* 0: the reference's iteration (Init.cpp:3344-3481),
                          bit for bit; 1: Newton on the group, U <- exp(i d.t) U
                          with the exact Jacobian of that step (no numeric
                          differences, stops as soon as sum_a |F_a| < the
                          tolerance), for throughput: the same root to the
                          tolerance, not the same bits; a link it does not
                          converge in 30 steps takes the reference's
                          iteration. The adjoint through the initial
                          conditions needs mode 0. */
} ipg_config;

/* Summary of the initial-condition stage. */
typedef struct {
    int newton_links;         /* 2 N^2 */
    int newton_restarted;     /* links that drew a random restart */
    int newton_failed;        /* links left at their best estimate */
    int newton_max_iterations;
    double newton_mean_iterations;
    double ms_wilson;         /* rho -> V_A, V_B */
    double ms_newton;         /* link products + Newton */
    double ms_fields;         /* initial pi */
} ipg_init_report;

/* Scalars of a finished event. */
typedef struct {
    int itmax;                /* leapfrog steps (Evolution.cpp:396) */
    double dtau;              /* lattice units */
    double tau_final;         /* fm, it*dtau*a at the observables */
    double gauss_violation;   /* Evolution.cpp:295-364 */
    double unitarity_max;     /* max |U^dag U - 1| over links, entrywise */
    double sum_Ttautau;       /* sum over cells of T^tautau (fm^-4) */
    double sum_eps;           /* sum over cells of e (fm^-4) */
    double E_T;               /* tau a^2 hbarc sum T^tautau, GeV */
    double eccentricity[6];   /* epsilon_1 .. epsilon_6 (Evolution.cpp:1660-1672) */
    double psi[6];            /* Psi_1 .. Psi_6 */
    int cells_without_u;      /* cells with no time-like eigenvector */
    double ms_evolution;
    double ms_observables;
} ipg_result;

/* Error text of the last failing call on ctx (never NULL). */
const char *ipg_last_error(const ipg_ctx *ctx);

/* Replaces the per-event construction of Parameters, Lattice, Init and
 * Evolution (main.cpp:66-336) and the derived time step (main.cpp:531-534). */
ipg_status ipg_create(const ipg_config *cfg, ipg_ctx **out);
ipg_status ipg_destroy(ipg_ctx *ctx);

/* New key for the device random streams of the next ipg_init_fields (a new
 * event on the same context, no reallocation). */
ipg_status ipg_reseed(ipg_ctx *ctx, uint64_t seed);

/* Effective dtau (lattice units) and leapfrog step count of ctx. */
ipg_status ipg_time_grid(const ipg_ctx *ctx, double *dtau, int *itmax);

/* g^2 mu^2 maps of both nuclei, lattice units, [N*N] host arrays; replaces
 * Cell::setg2mu2A/B as filled by Init::setColorChargeDensity
 * (Init.cpp:753-1676). The copies are queued on the context's stream: from
 * page-locked memory they are read after the call returns, so keep the
 * arrays unchanged until the next call that waits (ipg_init_fields). */
ipg_status ipg_set_g2mu(ipg_ctx *ctx, const double *g2mu2A,
                        const double *g2mu2B);
/* same, device pointers (no host copy) */
ipg_status ipg_set_g2mu_device(ipg_ctx *ctx, const double *d_g2mu2A,
                               const double *d_g2mu2B);

/* g^2 mu^2 maps of both nuclei computed on the device from nucleon
 * positions: xyz[3*nA], xyz[3*nB] in fm (x, y, z), nucleus A shifted by
 * -b/2 and B by +b/2 along x. T(x) = sum_k exp(-|x - x_k|^2/(2B))/(2 pi B)
 * with B = BG hbarc^2 (Init.cpp:1052-1062, no substructure), then
 * Q_s^2 = QsMax^2 T / max T and g2mu2 = Q_s^2/QsmuRatio^2 a^2/hbarc^2/g^2
 * (Init.cpp:1403-1408). The reference's IP-Sat Q_s(T) table is not part of
 * this library; this is the Q_s ~ sqrt(T) map. Replaces the g2mu part of
 * Init::setColorChargeDensity (Init.cpp:753-1676) for that map. */
ipg_status ipg_set_nuclei(ipg_ctx *ctx, const double *xyzA, int nA, const double *xyzB, int nB,
                          double b, double BG, double QsMax, double QsmuRatio);
/* IP-Sat colour-charge maps: the parameters of Init::setColorChargeDensity
 * (Init.cpp:753-1676) that this path reads (the reference's input keys in
 * brackets). */
typedef struct {
    double BG;                /* nucleon width B_G, GeV^-2 (BG) */
    double QsmuRatio;         /* Q_s / g^2 mu of nucleus A (QsmuRatio) */
    double QsmuRatioB;        /* of nucleus B; the reference sets it to QsmuRatio */
    double proton_anisotropy; /* xi of the elliptic nucleon (protonAnisotropy); 0: round */
    double rapidity;          /* y (Rapidity) */
    double roots;             /* sqrt(s), GeV (roots) */
    double x_factor;          /* x = factor Q_s / sqrt(s) e^{-y} (xFromThisFactorTimesQs) */
    double rmax;              /* nucleon cut-off radius, fm (rmax) */
    double sigmaNN;           /* inelastic NN cross section, mb (SigmaNN) */
    int use_fluctuating_x;    /* 1: Q_s at the x of the site's own Q_s (useFluctuatingx) */
    int average_over_nuclei;  /* T divided by this (averageOverNuclei), >= 1 */
} ipg_ipsat_params;

/* What setColorChargeDensity reports about the event (Init.cpp:1117-1217,
 * 1423-1530). */
typedef struct {
    int Npart, Ncoll;       /* hard-sphere wounding with d^2 < sigma_NN / (10 pi) */
    double Tpp;             /* sum of T_A T_B a^2, fm^-2 */
    double average_Qs;      /* GeV, over the cells near collided nucleons of both nuclei:
                               sqrt of the mean of max(Q_sA^2, Q_sB^2) */
    double average_Qs_avg;  /* sqrt of the mean of (Q_sA^2 + Q_sB^2) / 2 */
    double average_Qs_min;  /* sqrt of the mean of min(Q_sA^2, Q_sB^2) */
    double Qs2min_ST;       /* sum over all cells of min(Q_sA^2, Q_sB^2) a^2 / hbarc^2 */
    int overlap_cells;      /* cells counted in the means */
    int flags;              /* bit 0: y beyond the table, 1: T beyond the table (its
                               last row used), 2: a fixed point did not converge in
                               1000 steps, 3: the single-threaded order was needed */
} ipg_ipsat_report;

/* g^2 mu^2 of both nuclei from nucleon positions with the reference's IP-Sat
 * construction, on the device: T_A, T_B as sums of nucleon Gaussians
 * (Init.cpp:1009-1106; optional per-nucleon angle phi and Q_s normalisation,
 * NULL for 0 and 1), then at cells within rmax of both nuclei Q_s^2 from
 * the table Q_s^2(T, y) (Init::getNuclearQs2, Init.cpp:686-749: Tlist[nT]
 * increasing, qs2[nT][ny] at y = k dy) with the fluctuating-x fixed point
 * (Init.cpp:1219-1410), and g^2 mu^2 = Q_s^2 / QsmuRatio^2 a^2/hbarc^2/g^2.
 * xyz[3 n] in fm (z unused), nucleus A shifted by -b/2 and B by +b/2 along x.
 * The fixed point of nucleus A starts from the rapidity nucleus B ended on
 * at the previous cell, as in the reference's loop run on one thread. The
 * table is the reference's qs2Adj_vs_Tp_vs_Y_200.in (readNuclearQs,
 * Init.cpp:441-480: nT = 200, ny = 44, dy = 0.25). rep may be NULL. */
ipg_status ipg_set_nuclei_ipsat(ipg_ctx *ctx, const double *xyzA, int nA, const double *xyzB,
                                int nB, const double *phiA, const double *phiB,
                                const double *normA, const double *normB, double b,
                                const ipg_ipsat_params *params, const double *Tlist,
                                const double *qs2, int nT, int ny, double dy,
                                ipg_ipsat_report *rep);
/* The nucleon thickness maps T_A, T_B ([N*N], GeV^2) of the last
 * ipg_set_nuclei_ipsat. */
ipg_status ipg_get_thickness(ipg_ctx *ctx, double *TA, double *TB);

/* Copy the current g^2 mu^2 maps ([N*N] each, lattice units) to the host. */
ipg_status ipg_get_g2mu(ipg_ctx *ctx, double *g2mu2A, double *g2mu2B);

/* Unit Gaussian noise xi[k][pos][a] (k < Ny, a < 8) of both nuclei in the
 * draw order of Init::setV, so rho = g sqrt(g2mu2/Ny) xi reproduces
 * Init.cpp:1695-1705 and 1773-1783. Host arrays of Ny*N*N*8 doubles. */
ipg_status ipg_set_noise(ipg_ctx *ctx, const double *xiA, const double *xiB);
/* same, device pointers, 16-byte aligned; they must stay valid until
 * ipg_init_fields returns */
ipg_status ipg_set_noise_device(ipg_ctx *ctx, const double *d_xiA,
                                const double *d_xiB);
/* Draw the noise on the device (Philox4x32-10 keyed by cfg.seed) instead of
 * reading it; replaces the serial Random::Gauss stream (Random.cpp:178-204). */
ipg_status ipg_use_device_noise(ipg_ctx *ctx);

/* The unit normals ipg_use_device_noise draws for nucleus (0 = A, 1 = B),
 * sheets [sheet_first, sheet_first + sheet_count), under the context's
 * current key, written to the host array xi[sheet_count][N*N][8] in the
 * layout of ipg_set_noise. Feeding them back through ipg_set_noise gives the
 * same Wilson lines as the device draw; for statistical checks of the
 * generator that replaces Random::Gauss (Random.cpp:178-204). */
ipg_status ipg_draw_device_noise(ipg_ctx *ctx, int nucleus, int sheet_first, int sheet_count,
                                 double *xi);

/* Wilson lines, tau=0 Newton link solve and initial fields; replaces
 * Init::setV (Init.cpp:1678-1849) and the tau=0 block of Init::init
 * (Init.cpp:2437-2691). report may be NULL. Returns
 * IPG_ERR_NEWTON_NONCONVERGED (fields still set) if any link failed. */
ipg_status ipg_init_fields(ipg_ctx *ctx, ipg_init_report *report);

/* tau=0 link solve and initial fields from Wilson lines loaded with
 * ipg_set_field(IPG_VA / IPG_VB); replaces the READFROMFILE > 0 path of
 * Init::init (readV then the tau=0 block, Init.cpp:2377-2381, 2437-2691). */
ipg_status ipg_init_from_wilson_lines(ipg_ctx *ctx, ipg_init_report *report);

/* The whole schedule of Evolution::run (Evolution.cpp:366-657): tau=0 half
 * step, itmax-1 full steps, T^{mu nu} + Landau matching at it = itmax
 * before the final half step of pi and E, then Gauss law and
 * eccentricities. result may be NULL. */
ipg_status ipg_run(ipg_ctx *ctx, ipg_result *result);

/* Leapfrog only: the tau=0 half step (evolvePhi/evolveU at tau=0,
 * Evolution.cpp:393-394) when the context is fresh from ipg_init_fields,
 * then `steps` full steps it = 1..steps (Evolution.cpp:416-421). */
ipg_status ipg_evolve(ipg_ctx *ctx, int steps);

/* Per-cell observables after ipg_run, [N*N] (eps, fm^-4) and component-major
 * [k][N*N] arrays: u4 = (u^tau, u^x, u^y, u^eta); pi10 and T10 in the order
 * tautau xx yy etaeta taux tauy taueta xy xeta yeta (Cell.h getters,
 * MyEigen.cpp:259-305, Evolution.cpp:759-1238). Any pointer may be NULL. */
ipg_status ipg_get_observables(ipg_ctx *ctx, double *eps, double *u4,
                               double *pi10, double *T10);
/* The same copies started on a second stream, returning at once: they run
 * while the caller starts the next event on this context, whose observables
 * stage waits for them before it rewrites the device arrays. The host arrays
 * are complete after ipg_wait_observables; they should be page-locked for
 * the copies to overlap. */
ipg_status ipg_get_observables_async(ipg_ctx *ctx, double *eps, double *u4, double *pi10,
                                     double *T10);
ipg_status ipg_wait_observables(ipg_ctx *ctx);

/* Field access for stage-wise checks; which = IPG_UX, IPG_UY, IPG_E1, IPG_E2,
 * IPG_PHI, IPG_PI, IPG_VA, IPG_VB: N*N*18 doubles (Cell::getUx ...,
 * Cell.h:141-166). ipg_set_field loads a state, e.g. a tau=0 state written
 * by the reference. */
enum { IPG_UX = 0, IPG_UY, IPG_E1, IPG_E2, IPG_PHI, IPG_PI, IPG_VA, IPG_VB };
ipg_status ipg_get_field(ipg_ctx *ctx, int which, double *out);
ipg_status ipg_set_field(ipg_ctx *ctx, int which, const double *in);

/* Mark a state loaded with ipg_set_field as the tau=0 state (as if
 * ipg_init_fields had run). */
ipg_status ipg_mark_initialized(ipg_ctx *ctx);

/* Newton iteration counts [2*N*N] (link 2*pos + dir) after ipg_init_fields. */
ipg_status ipg_get_newton_iterations(ipg_ctx *ctx, int *iters, int *status);

/* Device time of the last leapfrog launch sequence run by ipg_evolve or
 * ipg_run, and the number of leapfrog launches it contained. */
ipg_status ipg_last_leapfrog_ms(ipg_ctx *ctx, double *ms, int *launches);

/* Number of kernels this library launched on ctx since creation. */
ipg_status ipg_kernel_launches(const ipg_ctx *ctx, long long *count);

/* Output files in the reference's formats from host observables (as returned
 * by ipg_get_observables); replace the writer part of
 * MyEigen::flowVelocity4D: the hydro file epsilon-u-Hydro-... (MyEigen.cpp:
 * 380-797, writeOutputs odd) and the KoMPoST file Tmunu-t... (MyEigen.cpp:
 * 801-1045, writeOutputs/4 == 1). it and dtau give the proper time
 * it*dtau*a of the observables; gfactor is 1 for a fixed coupling. Etot (may
 * be NULL) receives the energy the reference prints as "Etot". */
ipg_status ipg_write_hydro(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *eps,
                           const double *u4, const double *pi10, double gfactor,
                           double *Etot);
ipg_status ipg_write_tmunu(const char *path, int N, double L, int sizeOutput,
                           double LOutput, int etaSizeOutput, double detaOutput,
                           int it, double dtau, const double *T10, double gfactor);
/* The same two files from the context's observables after ipg_run, with the
 * resampling and the number formatting on the GPU: byte-identical to
 * ipg_write_hydro / ipg_write_tmunu on the ipg_get_observables arrays (same
 * operation order and rounding, correctly rounded "%.6g"), for L and N of
 * the context. Either path may be NULL. A file holding a number outside
 * [1e-130, 1e6) in magnitude (or a NaN) is written by the host writer
 * instead, with the same result. */
ipg_status ipg_write_outputs(ipg_ctx *ctx, const char *hydro_path, const char *tmunu_path,
                             int sizeOutput, double LOutput, int etaSizeOutput,
                             double detaOutput, int it, double dtau, double gfactor,
                             double *Etot);
/* The reference's output file names for an event id (MyEigen.cpp:376-383,
 * 804-807); buffers of at least 64 bytes. */
ipg_status ipg_output_names(int event_id, int it, double dtau, double a,
                            char *hydro, size_t hydro_len, char *tmunu,
                            size_t tmunu_len);

/* The remaining figures of the eccentricities<id>.dat line that
 * Evolution::eccentricity writes (Evolution.cpp:1280-1810, cutoff 0) for the
 * observables of the last ipg_run: sqrt(<r^2>) (the r^2 moment over
 * [2, N-2)^2 divided by the weight of all cells), the outermost cells with
 * weight on the centroid's row and column, the area and mean e of the cells
 * with e >= 0, Rbar = 1/sqrt(1/<x^2> + 1/<y^2>), and the mean of
 * Q_sA^2 Q_sB^2 over the same cells times hbarc (QsmuRatio, QsmuRatioB: the
 * ratios the g2mu maps were made with). The eccentricities and angles are in
 * ipg_result. */
typedef struct {
    double tau;            /* fm */
    double r_rms;          /* fm */
    double max_x, max_y;   /* fm, from the centroid; 0 when no cell has weight */
    double area;           /* fm^2 */
    double Rbar;           /* fm */
    double avg_eps;        /* GeV/fm^3 */
    double avg_qs2a_qs2b;  /* as printed by the reference (times hbarc) */
} ipg_ecc_report;
ipg_status ipg_eccentricity_report(ipg_ctx *ctx, double QsmuRatio, double QsmuRatioB,
                                   ipg_ecc_report *out);

/* ---- gauge fixing and gluon multiplicity ---------------------------------
 * GaugeFix::FFTChi (GaugeFix.cpp:17-165) and Evolution::multiplicity
 * (Evolution.cpp:2284-3188), which the reference runs at it = 1 and
 * it = itmax when computeGluonMultiplicity is set (Evolution.cpp:644-653).
 *
 * ipg_gauge_fix brings the fields to transverse Coulomb gauge by
 * Fourier-accelerated steepest descent, in place, as the reference does: per
 * iteration the residual <tr(g^dag g)> / Nc of g = sum_a Im tr(div A t^a) t^a,
 * the reference's two stopping rules (residual < 1e-9; residual above the one
 * recorded at the last multiple of 10 iterations and below 1e-6), then the
 * gauge transformation reu(expm(i chi)) with chi = IFFT(-1.5 / (k~^2 + 1e-9)
 * FFT(g)). The live fields are transformed and later steps continue from
 * them, as in the reference (on an FP32 context an FP64 copy of the fields
 * is transformed and rounded back). This matters: the reference's lattice
 * clamps neighbours at its edges (Lattice.cpp:19-27, Evolution.cpp:209-210)
 * while its gauge fixing is periodic (GaugeFix.cpp:54-66), so the evolution
 * is not covariant under that transformation at the edges, and a gauge
 * fixing part-way through changes what follows (by a few 1e-4 of the energy
 * at 64^2). */
typedef struct {
    int iterations;         /* gauge transformations applied */
    int residual_checks;    /* residuals computed (iterations + 1 when a rule
                               stopped it) */
    int nan_sites;          /* site transformations that were NaN and were
                               reset to 1 (GaugeFix.cpp:143-147) */
    double residual;        /* the last residual computed */
    double residual_every10[401]; /* at iterations 0, 10, 20, ... (the values
                               the reference prints); NaN past the last */
    double ms;              /* device time */
} ipg_gauge_report;

ipg_status ipg_gauge_fix(ipg_ctx *ctx, int max_iterations, ipg_gauge_report *report);

/* Parameters of Evolution::multiplicity read from the input file. */
typedef struct {
    int max_gauge_iterations; /* <= 0 -> 4000 (Evolution.cpp:2333) */
    int use_pseudorapidity;   /* usePseudoRapidity */
    double rapidity;          /* Rapidity */
    double jacobian_m;        /* Jacobianm, GeV */
    double roots;             /* roots, GeV (the mean p_T estimate of the
                                 pseudorapidity Jacobian) */
} ipg_multiplicity_params;

#define IPG_KT_BINS 100
/* The gluon spectrum of the current fields. dN/dy ("dN/dy 1") sums n(k) over
 * the lattice momenta; the binned values ("dN/dy 2") integrate the 100 k_T
 * bins of width 2.83/100 (lattice units); the cuts keep bins with
 * ik dkt / a hbarc above 3 and 6 GeV. With use_pseudorapidity the Jacobian
 * factors of Evolution.cpp:2896-2953 and 3098-3108 are applied. */
typedef struct {
    int it;                   /* the step of the fields */
    ipg_gauge_report gauge;
    double dNdy, dEdy;        /* GeV for E */
    double dNdy_binned, dEdy_binned;
    double dNdy_cut3, dEdy_cut3, dNdy_cut6, dEdy_cut6;
    double mean_pt;           /* dEdy / dNdy, GeV */
    double n_kt[IPG_KT_BINS]; /* bin averages (dN/d^2k_T in lattice units) */
    double E_kt[IPG_KT_BINS];
    int count_kt[IPG_KT_BINS];
    double ms_spectrum;       /* device time of the spectrum */
} ipg_multiplicity_result;

/* Gauge fixing followed by the spectrum of the context's current fields:
 * after ipg_evolve (it = completed steps, >= 1) or after ipg_run
 * (it = itmax, the fields after the final half step). dNdy == 0 is the
 * reference's "no collision happened" case (Evolution.cpp:3111-3122). */
ipg_status ipg_multiplicity(ipg_ctx *ctx, const ipg_multiplicity_params *params,
                            ipg_multiplicity_result *out);
/* ipg_run with the reference's computeGluonMultiplicity schedule: the
 * spectrum at it = 1 (at_first, after the first step; skipped when
 * itmax = 1) and at it = itmax (at_last, after the observables and the
 * final half step). The gauge fixing at it = 1 transforms the fields the
 * remaining steps start from. When dN/dy at it = 1 is zero the call returns
 * IPG_NO_COLLISION after filling at_first, with the context left at it = 1.
 * Any of the output pointers may be NULL. */
ipg_status ipg_run_multiplicity(ipg_ctx *ctx, const ipg_multiplicity_params *params,
                                ipg_result *result, ipg_multiplicity_result *at_first,
                                ipg_multiplicity_result *at_last);
/* The host part of Evolution::multiplicity, without a context: the k sums
 * dN, dE, the per-bin sums of n and E and the bin counts -> the fields of
 * out after `it` (it, dNdy .. count_kt; the gauge report and timings are
 * left alone). a is the lattice spacing in fm. */
ipg_status ipg_multiplicity_finish(double dN, double dE, const double *n_sum,
                                   const double *E_sum, const int *count, double a,
                                   const ipg_multiplicity_params *params,
                                   ipg_multiplicity_result *out);

/* ---- adjoint (no counterpart in the reference) ---------------------------
 * Reverse-mode derivatives of the evolution, with the autograd contract:
 * ipg_forward saves what ipg_backward consumes once. On an FP64 context the
 * plain form is differentiated in FP64. On an FP32 context (the FP32 adjoint)
 * the forward is the FP32 bulk form's own steps (deviation storage, per-step
 * reunitarisation), the reverse sweep runs in FP32 on those states (with
 * checkpoints, each segment is recomputed forward from its checkpoint instead
 * of reversed in time), and the adjoint of the tau = 0 state is widened to
 * FP64 for the initial conditions, whose adjoint stays FP64. The loss is
 *   L = w_ET * E_T + w_eps2 * eps2
 * at tau = itmax dtau a, from the state after the itmax leapfrog launches of
 * Evolution::run (where the reference evaluates T^{mu nu}):
 *   E_T  = tau a^2 hbarc sum_cells T^tautau (GeV), as ipg_result.E_T;
 *   eps2 = |sum w (x~ + i y~)^2| / sum w (x~^2 + y~^2) with the smooth weight
 *          w = T^tautau over cells [2, N-2)^2 and x~, y~ measured from the
 *          w-weighted centroid (the reference weights with e u^tau from the
 *          Landau matching, whose branch thresholds are not differentiable).
 * ipg_forward starts from the context's fresh tau = 0 state (after
 * ipg_init_fields, or ipg_set_field + ipg_mark_initialized) without changing
 * it; it stores the state before every checkpoint_every-th step. ipg_backward
 * walks back between checkpoints by exact time reversal of the step (FP64)
 * or by recomputing the segment from its checkpoint (FP32). With
 * checkpoint_every = 1 every state is kept (itmax + 1 states of 560 bytes a
 * site in FP64: 14.7 GB for 256^2 sites and 400 steps), each step writes its own
 * slot, the reverse sweep needs no time reversal, and ipg_backward may be
 * called again (other weights) without a new ipg_forward; checkpoint_every
 * = 0 takes 1 when those states fit in half of the free device memory, else
 * ~sqrt(itmax). ipg_backward returns dL/d(state at tau = 0) for U_x, U_y, E_1, E_2, phi, pi, each [N*N]
 * sites x 18 doubles (row-major 3x3, (re, im)), in that order (6*18*N*N
 * doubles; NULL skips the copy). For a complex entry z the pair is
 * (dL/dRe z, dL/dIm z); for the Hermitian fields it is the Hermitian part
 * (traceless for E).
 * When the tau = 0 state came from ipg_init_fields (not ipg_set_field), the
 * gradient continues through the initial conditions: grad_g2mu receives
 * dL/d(g2mu2A), dL/d(g2mu2B) ([2][N*N], lattice units) and grad_rho
 * dL/drho ([2][Ny][N*N][8], the layout of the noise of ipg_set_noise; rho =
 * g sqrt(g2mu2/Ny) xi); either may be NULL. This chain assumes the Newton
 * links are converged roots: set cfg.newton_tolerance to ~1e-12 for it (the
 * reference's 1e-6 leaves errors of that order in the links). Noise given
 * with ipg_set_noise_device must still be valid. */
ipg_status ipg_forward(ipg_ctx *ctx, int checkpoint_every, double *E_T, double *eps2);
ipg_status ipg_backward(ipg_ctx *ctx, double w_ET, double w_eps2, double *grad_state,
                        double *grad_g2mu, double *grad_rho);
/* Device time of the last ipg_forward (evolution, checkpoints, T^tautau) and
 * ipg_backward (reverse sweep and initial-condition adjoint, without the
 * copies of the gradients to the host). */
ipg_status ipg_adjoint_stats(const ipg_ctx *ctx, double *ms_forward, double *ms_backward);

/* ---- batches of events -------------------------------------------------
 * The reference runs one event per process (main.cpp:347-359, events handed
 * to MPI ranks). A batch advances many events -- contexts of possibly
 * different N (each >= 32) sharing one device, precision and time grid --
 * together: every leapfrog step is one persistent kernel launch over all
 * sites of all events, and the whole step sequence is a CUDA graph captured
 * on the first run and replayed afterwards. This is the multi-event form of
 * "ipg_evolve(ctx, ev_first, ev_count, nsteps)": each context is one event.
 * The batch does not own its contexts; destroy it before them. */
typedef struct ipg_batch ipg_batch;

/* Launch shape chosen by ipg_batch_tune. */
typedef struct {
    int variant;            /* tile-shape variant */
    int tile_rows;          /* a tile is 32 sites along y x tile_rows along x */
    int threads_per_block;  /* one thread per site */
    int blocks_per_sm;      /* resident blocks of the persistent grid */
    int grid;               /* blocks_per_sm x SM count */
    double ms_per_step;     /* measured time of one full step of the batch */
    int candidates;         /* shapes timed (0 when taken from the cache) */
    int from_cache;         /* 1 if the shape came from the tuning cache */
} ipg_tune_report;

const char *ipg_batch_last_error(const ipg_batch *batch);
ipg_status ipg_batch_create(ipg_ctx *const *events, int count, ipg_batch **out);
ipg_status ipg_batch_destroy(ipg_batch *batch);
/* ipg_init_fields for every event (g2mu and noise set on each), enqueued on
 * the events' own streams before any is waited for, so the initial
 * conditions of small lattices run side by side; reports[count] may be NULL.
 * Returns IPG_ERR_NEWTON_NONCONVERGED if any event has non-converged links. */
ipg_status ipg_batch_init(ipg_batch *batch, ipg_init_report *reports);
/* Time every tile shape and resident-block count on one full step of this
 * batch (events freshly initialised; their E and pi are restored) and keep
 * the fastest. Results are cached per (device, precision, lattice sizes) in
 * the process and, if the environment variable IPG_TUNE_CACHE names a file,
 * in that file. */
ipg_status ipg_batch_tune(ipg_batch *batch, ipg_tune_report *report);
/* Evolve every event (freshly initialised with ipg_init_fields) through the
 * schedule of Evolution::run and compute its observables; results[count].
 * ms_evolution of each result is the batch's shared leapfrog time. */
ipg_status ipg_batch_run(ipg_batch *batch, ipg_result *results);
/* Set the launch shape by hand: variants 0, 1, 2 (FP32) or 0, 1 (FP64) are
 * plain-load kernels on tiles of 2, 4 or 8 rows; variant 3 (FP32) or 2 (FP64)
 * is the TMA tile kernel of the single-event form run over every event's
 * tiles (1 block per SM); 1 <= blocks_per_sm <= what fits on an SM. */
ipg_status ipg_batch_set_shape(ipg_batch *batch, int variant, int blocks_per_sm);
ipg_status ipg_batch_stats(const ipg_batch *batch, double *ms_evolution,
                           double *ms_total, long long *launches);

/* Wilson lines of one nucleus without allocating anything: no counterpart in
 * the reference (it is an addition of this library). For callers that cannot
 * allocate device memory (code inside another framework's memory pool or
 * allocator hooks, hosts that forbid allocation after start-up, callers that
 * must avoid the synchronisation cudaMalloc/cudaFree can imply). Computes what
 * ipg_init_fields computes for V_A (or V_B): rho = g sqrt(g2mu2/Ny) xi, the
 * Poisson solve and the ordered product of the Ny sheet exponentials, on the
 * given stream (NULL = default stream). All pointers are device pointers the
 * caller owns: d_g2mu2[N*N], d_xi[Ny][N*N][8] (16-byte aligned), output
 * d_V[N*N*18] (3x3 per
 * site, row-major (re, im)). Scratch lives in one fixed device array sized for
 * N <= 256 (about 14 MB per GPU that loads the library, kept until exit);
 * larger N returns IPG_ERR_BAD_CONFIG. The first call on a device looks up
 * that array's address (make it before any stream capture). Calls share the
 * array: calls that overlap on the GPU race and must be serialised. */
ipg_status ipg_wilson_lines_noalloc(int N, int Ny, double L, double g, double m,
                                    double UVdamp, const double *d_g2mu2,
                                    const double *d_xi, double *d_V,
                                    void *stream);

#ifdef __cplusplus
}
#endif

#endif
