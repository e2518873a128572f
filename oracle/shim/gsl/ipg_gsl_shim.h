/*
 * Minimal GSL API subset, written for this project so that the reference
 * IP-Glasma sources compile unmodified in a container without GSL.
 *
 * TEST INFRASTRUCTURE ONLY: part of the CPU oracle build (oracle/_ref).
 *
 * Implemented (on the IP-Glasma hot path):
 *   - real/complex LU decomposition with partial pivoting and the matching
 *     solve (Init.cpp:28-63), following the textbook Gaussian elimination of
 *     Golub & Van Loan, "Matrix Computations", Algorithm 3.4.1, which is the
 *     algorithm GSL 2.5 documents for gsl_linalg_LU_decomp;
 *   - the real nonsymmetric eigen-solver with eigenvectors
 *     (MyEigen.cpp:78-93) for 4x4 matrices: Householder reduction to
 *     Hessenberg form, Francis double-shift QR for the eigenvalues and a
 *     complete-pivoting null vector of (A - lambda I) for each eigenvector,
 *     scaled to unit Euclidean norm as the GSL manual specifies (ipg_eig4.h);
 *   - gsl_complex arithmetic helpers.
 * Declared but aborting when called (off the hot path): random-variate
 * generators, Gauss-Legendre tables and cubic splines.
 */
#ifndef IPG_GSL_SHIM_H
#define IPG_GSL_SHIM_H

#include <math.h> /* GSL headers pull in math.h through gsl_math.h */
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSL_SUCCESS 0

typedef struct {
    double dat[2];
} gsl_complex;

#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])
#define GSL_SET_COMPLEX(zp, x, y) \
    do {                          \
        (zp)->dat[0] = (x);       \
        (zp)->dat[1] = (y);       \
    } while (0)

typedef struct {
    size_t size;
    size_t stride;
    double *data;
    void *block;
    int owner;
} gsl_vector;

typedef struct {
    gsl_vector vector;
} gsl_vector_view;

typedef struct {
    size_t size;
    size_t stride;
    double *data; /* interleaved (re, im) */
    void *block;
    int owner;
} gsl_vector_complex;

typedef struct {
    gsl_vector_complex vector;
} gsl_vector_complex_view;

typedef struct {
    size_t size1;
    size_t size2;
    size_t tda;
    double *data;
    void *block;
    int owner;
} gsl_matrix;

typedef struct {
    gsl_matrix matrix;
} gsl_matrix_view;

typedef struct {
    size_t size1;
    size_t size2;
    size_t tda;
    double *data; /* interleaved (re, im), row-major with row stride tda */
    void *block;
    int owner;
} gsl_matrix_complex;

typedef struct {
    gsl_matrix_complex matrix;
} gsl_matrix_complex_view;

typedef struct {
    size_t size;
    size_t *data;
} gsl_permutation;

/* vectors and matrices */
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);

gsl_vector_complex *gsl_vector_complex_alloc(size_t n);
void gsl_vector_complex_free(gsl_vector_complex *v);
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i);
gsl_vector_complex_view gsl_vector_complex_view_array(double *base, size_t n);

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
gsl_matrix_complex_view gsl_matrix_complex_view_array(double *base, size_t n1,
                                                      size_t n2);
gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2);
void gsl_matrix_complex_free(gsl_matrix_complex *m);
gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m,
                                                  size_t j);

gsl_permutation *gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);

/* linear algebra */
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p,
                        const gsl_vector *b, gsl_vector *x);
int gsl_linalg_complex_LU_decomp(gsl_matrix_complex *A, gsl_permutation *p,
                                 int *signum);
int gsl_linalg_complex_LU_solve(const gsl_matrix_complex *LU,
                                const gsl_permutation *p,
                                const gsl_vector_complex *b,
                                gsl_vector_complex *x);

/* eigen-system of a general real matrix */
typedef struct {
    size_t size;
    double *work;
} gsl_eigen_nonsymmv_workspace;

gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n);
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w);
int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval,
                       gsl_matrix_complex *evec,
                       gsl_eigen_nonsymmv_workspace *w);

/* complex arithmetic */
gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b);
gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b);

/* random numbers (generator object only; variates abort) */
typedef struct {
    const char *name;
} gsl_rng_type;
typedef struct {
    const gsl_rng_type *type;
    unsigned long seed;
} gsl_rng;
extern const gsl_rng_type *gsl_rng_taus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long seed);
void gsl_rng_free(gsl_rng *r);
unsigned int gsl_ran_poisson(const gsl_rng *r, double mu);
unsigned int gsl_ran_negative_binomial(const gsl_rng *r, double p, double n);
double gsl_ran_tdist(const gsl_rng *r, double nu);

/* Gauss-Legendre tables (abort) */
typedef struct {
    size_t n;
} gsl_integration_glfixed_table;
gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n);
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi,
                                  double *wi,
                                  const gsl_integration_glfixed_table *t);

/* splines (abort) */
typedef struct {
    const char *name;
} gsl_interp_type;
typedef struct {
    size_t cache;
} gsl_interp_accel;
typedef struct {
    size_t size;
} gsl_spline;
extern const gsl_interp_type *gsl_interp_cspline;
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[],
                    size_t size);
double gsl_spline_eval_integ(const gsl_spline *spline, double a, double b,
                             gsl_interp_accel *acc);
void gsl_spline_free(gsl_spline *spline);

#ifdef __cplusplus
}
#endif

#endif
