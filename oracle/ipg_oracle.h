/*
 * CPU restatement of IP-Glasma's per-event hot path (TEST INFRASTRUCTURE
 * ONLY): the checker the parity tests compare the CUDA library against, and
 * the "port" CPU baseline. Nothing shipped links or calls it.
 *
 * Parity pinned: tests/test_oracle_port.py checks every stage against the
 * reference itself (oracle/_ref/ipg_ref_harness, the reference sources
 * compiled unmodified) and against the committed fixtures in tests/golden/.
 *
 * Layout conventions follow the reference: site pos = ix * N + iy
 * (Lattice.cpp:15-28); a 3x3 complex matrix is 18 doubles, row-major
 * (re, im) pairs; all fields are full 3x3 matrices per site.
 */
#ifndef IPG_ORACLE_H
#define IPG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* MT19937-64 + polar Gaussian, Random.cpp:1-204: `count` normals of the
 * stream seeded with `seed` (the order Init::setV draws them). */
void ipgo_gauss_stream(uint64_t seed, long count, double *out);

/* exp(i in.t) (Matrix::expmCoeff + Init::getUfromExponent), 18 doubles */
void ipgo_expm(const double in[8], double out[18]);

/* Init::setV for one nucleus (Init.cpp:1678-1768): V[N*N*18] from the g2mu2
 * map [N*N] and unit normals xi[Ny][N*N][8]. */
void ipgo_wilson_lines(int N, int Ny, double L, double g, double m_GeV,
                       double uvdamp, const double *g2mu2, const double *xi,
                       double *V);

/* tau = 0 block of Init::init (Init.cpp:2437-2691): links Ux, Uy and pi;
 * newton_iters[2*N*N] (may be NULL) gets the iteration counts. Returns the
 * number of links that hit a restart (those use no random draws here and
 * are flagged, since the reference draws them from its serial stream). */
int ipgo_tau0(int N, double g, const double *VA, const double *VB,
              double *Ux, double *Uy, double *pi, int *newton_iters);

/* One call of the leapfrog pieces in the reference's order
 * (Evolution.cpp:35-293). Fields are full 3x3 per site. */
void ipgo_evolve_phi(int N, double dtau, double tau, double *phi,
                     const double *pi);
void ipgo_evolve_u(int N, double g, double dtau, double tau, double *Ux,
                   double *Uy, const double *E1, const double *E2);
void ipgo_evolve_pi(int N, double dtau, double tau, const double *Ux,
                    const double *Uy, const double *phi, double *pi);
void ipgo_evolve_e(int N, double g, double dtau, double tau, const double *Ux,
                   const double *Uy, const double *phi, double *E1,
                   double *E2);

/* Evolution::Tmunu (Evolution.cpp:659-1246): T10[10][N*N] in the order
 * tautau xx yy etaeta taux tauy taueta xy xeta yeta. */
void ipgo_tmunu(int N, double L, double g, double dtau, int it,
                const double *Ux, const double *Uy, const double *E1,
                const double *E2, const double *phi, const double *pi,
                double *T10);

/* MyEigen::flowVelocity4D (MyEigen.cpp:25-314): eps[N*N], u4[4][N*N],
 * pi10[10][N*N]; returns the number of cells without a time-like vector. */
int ipgo_landau(int N, double L, double dtau, int it, const double *T10,
                double *eps, double *u4, double *pi10);

/* Evolution::checkGaussLaw (Evolution.cpp:295-364) */
double ipgo_gauss_law(int N, const double *Ux, const double *Uy,
                      const double *E1, const double *E2, const double *phi,
                      const double *pi);

/* Evolution::eccentricity (Evolution.cpp:1280-1810), cutoff 0, constant
 * coupling: ecc[6] = epsilon_1..6, psi[6] = Psi_1..6 */
void ipgo_eccentricity(int N, double L, const double *eps, const double *utau,
                       double ecc[6], double psi[6]);

/* The whole event: setV for both nuclei, tau=0, Evolution::run schedule,
 * eccentricity. Outputs may be NULL. scalars[0] = Gauss violation,
 * scalars[1] = epsilon_2, scalars[2] = itmax, scalars[3] = dtau,
 * scalars[4] = Newton links with restarts. */
void ipgo_run_event(int N, int Ny, double L, double g, double m_GeV,
                    double uvdamp, double maxtime, double dtau_override,
                    const double *g2muA, const double *g2muB,
                    const double *xiA, const double *xiB, double *VA,
                    double *VB, double *tau0_Ux, double *tau0_Uy,
                    double *tau0_pi, double *eps, double *u4, double *pi10,
                    double *T10, double *scalars);

/* The output files of MyEigen::flowVelocity4D (MyEigen.cpp:380-797 hydro,
 * 801-1045 Tmunu), written serially with printf "%g" (what an ostream with
 * default flags prints). Return 0 on success; *Etot gets the hydro file's
 * total energy (MyEigen.cpp:755). */
int ipgo_write_hydro(const char *path, int N, double L, int sizeOutput,
                     double LOutput, int etaSizeOutput, double detaOutput,
                     int it, double dtau, const double *eps, const double *u4,
                     const double *pi10, double gfactor, double *Etot);
int ipgo_write_tmunu(const char *path, int N, double L, int sizeOutput,
                     double LOutput, int etaSizeOutput, double detaOutput,
                     int it, double dtau, const double *T10, double gfactor);

#ifdef __cplusplus
}
#endif

#endif
