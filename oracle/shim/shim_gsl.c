/*
 * GSL API subset for the CPU oracle build (TEST INFRASTRUCTURE ONLY).
 * See ipg_gsl_shim.h for the list of what is implemented and the published
 * algorithms each part restates.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/ipg_gsl_shim.h"

static void shim_abort(const char *what) {
    fprintf(stderr, "GSL shim: %s is not available in the oracle build\n",
            what);
    abort();
}

/* ------------------------------------------------------------------ */
/* vectors / matrices / permutations                                  */
/* ------------------------------------------------------------------ */

gsl_vector *gsl_vector_alloc(size_t n) {
    gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
    v->size = n;
    v->stride = 1;
    v->data = (double *)calloc(n ? n : 1, sizeof(double));
    v->owner = 1;
    return v;
}

void gsl_vector_free(gsl_vector *v) {
    if (!v) return;
    if (v->owner) free(v->data);
    free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i) {
    return v->data[i * v->stride];
}

gsl_vector_view gsl_vector_view_array(double *base, size_t n) {
    gsl_vector_view view;
    view.vector.size = n;
    view.vector.stride = 1;
    view.vector.data = base;
    view.vector.block = NULL;
    view.vector.owner = 0;
    return view;
}

gsl_vector_complex *gsl_vector_complex_alloc(size_t n) {
    gsl_vector_complex *v =
        (gsl_vector_complex *)calloc(1, sizeof(gsl_vector_complex));
    v->size = n;
    v->stride = 1;
    v->data = (double *)calloc(2 * (n ? n : 1), sizeof(double));
    v->owner = 1;
    return v;
}

void gsl_vector_complex_free(gsl_vector_complex *v) {
    if (!v) return;
    if (v->owner) free(v->data);
    free(v);
}

gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i) {
    gsl_complex z;
    z.dat[0] = v->data[2 * i * v->stride];
    z.dat[1] = v->data[2 * i * v->stride + 1];
    return z;
}

gsl_vector_complex_view gsl_vector_complex_view_array(double *base, size_t n) {
    gsl_vector_complex_view view;
    view.vector.size = n;
    view.vector.stride = 1;
    view.vector.data = base;
    view.vector.block = NULL;
    view.vector.owner = 0;
    return view;
}

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) {
    gsl_matrix_view view;
    view.matrix.size1 = n1;
    view.matrix.size2 = n2;
    view.matrix.tda = n2;
    view.matrix.data = base;
    view.matrix.block = NULL;
    view.matrix.owner = 0;
    return view;
}

gsl_matrix_complex_view gsl_matrix_complex_view_array(double *base, size_t n1,
                                                      size_t n2) {
    gsl_matrix_complex_view view;
    view.matrix.size1 = n1;
    view.matrix.size2 = n2;
    view.matrix.tda = n2;
    view.matrix.data = base;
    view.matrix.block = NULL;
    view.matrix.owner = 0;
    return view;
}

gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2) {
    gsl_matrix_complex *m =
        (gsl_matrix_complex *)calloc(1, sizeof(gsl_matrix_complex));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double *)calloc(2 * (n1 * n2 ? n1 * n2 : 1), sizeof(double));
    m->owner = 1;
    return m;
}

void gsl_matrix_complex_free(gsl_matrix_complex *m) {
    if (!m) return;
    if (m->owner) free(m->data);
    free(m);
}

gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m,
                                                  size_t j) {
    gsl_vector_complex_view view;
    view.vector.size = m->size1;
    view.vector.stride = m->tda;
    view.vector.data = m->data + 2 * j;
    view.vector.block = NULL;
    view.vector.owner = 0;
    return view;
}

gsl_permutation *gsl_permutation_alloc(size_t n) {
    gsl_permutation *p = (gsl_permutation *)calloc(1, sizeof(gsl_permutation));
    size_t i;
    p->size = n;
    p->data = (size_t *)calloc(n ? n : 1, sizeof(size_t));
    for (i = 0; i < n; i++) p->data[i] = i;
    return p;
}

void gsl_permutation_free(gsl_permutation *p) {
    if (!p) return;
    free(p->data);
    free(p);
}

/* ------------------------------------------------------------------ */
/* LU with partial pivoting (Golub & Van Loan, Alg. 3.4.1)            */
/* ------------------------------------------------------------------ */

#define RM(A, i, j) ((A)->data[(i) * (A)->tda + (j)])

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum) {
    size_t n = A->size1, col, row, k;
    *signum = 1;
    for (k = 0; k < n; k++) p->data[k] = k;
    for (col = 0; col + 1 < n; col++) {
        /* pivot: first row holding the largest |entry| in this column */
        size_t piv = col;
        double best = fabs(RM(A, col, col));
        for (row = col + 1; row < n; row++) {
            double c = fabs(RM(A, row, col));
            if (c > best) {
                best = c;
                piv = row;
            }
        }
        if (piv != col) {
            size_t t;
            for (k = 0; k < n; k++) {
                double tmp = RM(A, col, k);
                RM(A, col, k) = RM(A, piv, k);
                RM(A, piv, k) = tmp;
            }
            t = p->data[col];
            p->data[col] = p->data[piv];
            p->data[piv] = t;
            *signum = -(*signum);
        }
        {
            double d = RM(A, col, col);
            if (d != 0.0) {
                for (row = col + 1; row < n; row++) {
                    double l = RM(A, row, col) / d;
                    RM(A, row, col) = l;
                    for (k = col + 1; k < n; k++)
                        RM(A, row, k) = RM(A, row, k) - l * RM(A, col, k);
                }
            }
        }
    }
    return GSL_SUCCESS;
}

int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p,
                        const gsl_vector *b, gsl_vector *x) {
    size_t n = LU->size1, i, j;
    double *y = (double *)malloc(sizeof(double) * n);
    for (i = 0; i < n; i++)
        if (RM(LU, i, i) == 0.0) {
            fprintf(stderr, "GSL shim: LU_solve on a singular matrix\n");
            abort();
        }
    /* y = P b */
    for (i = 0; i < n; i++) y[i] = b->data[p->data[i] * b->stride];
    /* forward substitution, unit lower triangle */
    for (i = 1; i < n; i++) {
        double acc = y[i];
        for (j = 0; j < i; j++) acc -= RM(LU, i, j) * y[j];
        y[i] = acc;
    }
    /* back substitution, upper triangle */
    for (i = n; i-- > 0;) {
        double acc = y[i];
        for (j = i + 1; j < n; j++) acc -= RM(LU, i, j) * y[j];
        y[i] = acc / RM(LU, i, i);
    }
    for (i = 0; i < n; i++) x->data[i * x->stride] = y[i];
    free(y);
    return GSL_SUCCESS;
}

/* complex variant: same elimination order, modulus |z| for pivoting */
#define CR(A, i, j) ((A)->data[2 * ((i) * (A)->tda + (j))])
#define CI(A, i, j) ((A)->data[2 * ((i) * (A)->tda + (j)) + 1])

int gsl_linalg_complex_LU_decomp(gsl_matrix_complex *A, gsl_permutation *p,
                                 int *signum) {
    size_t n = A->size1, col, row, k;
    *signum = 1;
    for (k = 0; k < n; k++) p->data[k] = k;
    for (col = 0; col + 1 < n; col++) {
        size_t piv = col;
        double best = hypot(CR(A, col, col), CI(A, col, col));
        for (row = col + 1; row < n; row++) {
            double c = hypot(CR(A, row, col), CI(A, row, col));
            if (c > best) {
                best = c;
                piv = row;
            }
        }
        if (piv != col) {
            size_t t;
            for (k = 0; k < n; k++) {
                double tr = CR(A, col, k), ti = CI(A, col, k);
                CR(A, col, k) = CR(A, piv, k);
                CI(A, col, k) = CI(A, piv, k);
                CR(A, piv, k) = tr;
                CI(A, piv, k) = ti;
            }
            t = p->data[col];
            p->data[col] = p->data[piv];
            p->data[piv] = t;
            *signum = -(*signum);
        }
        {
            double dr = CR(A, col, col), di = CI(A, col, col);
            double den = dr * dr + di * di;
            if (den != 0.0) {
                for (row = col + 1; row < n; row++) {
                    double ar = CR(A, row, col), ai = CI(A, row, col);
                    double lr = (ar * dr + ai * di) / den;
                    double li = (ai * dr - ar * di) / den;
                    CR(A, row, col) = lr;
                    CI(A, row, col) = li;
                    for (k = col + 1; k < n; k++) {
                        double ur = CR(A, col, k), ui = CI(A, col, k);
                        CR(A, row, k) -= lr * ur - li * ui;
                        CI(A, row, k) -= lr * ui + li * ur;
                    }
                }
            }
        }
    }
    return GSL_SUCCESS;
}

int gsl_linalg_complex_LU_solve(const gsl_matrix_complex *LU,
                                const gsl_permutation *p,
                                const gsl_vector_complex *b,
                                gsl_vector_complex *x) {
    size_t n = LU->size1, i, j;
    double *y = (double *)malloc(sizeof(double) * 2 * n);
    for (i = 0; i < n; i++) {
        y[2 * i] = b->data[2 * p->data[i] * b->stride];
        y[2 * i + 1] = b->data[2 * p->data[i] * b->stride + 1];
    }
    for (i = 1; i < n; i++)
        for (j = 0; j < i; j++) {
            double lr = CR(LU, i, j), li = CI(LU, i, j);
            y[2 * i] -= lr * y[2 * j] - li * y[2 * j + 1];
            y[2 * i + 1] -= lr * y[2 * j + 1] + li * y[2 * j];
        }
    for (i = n; i-- > 0;) {
        double ar = y[2 * i], ai = y[2 * i + 1], dr, di, den;
        for (j = i + 1; j < n; j++) {
            double ur = CR(LU, i, j), ui = CI(LU, i, j);
            ar -= ur * y[2 * j] - ui * y[2 * j + 1];
            ai -= ur * y[2 * j + 1] + ui * y[2 * j];
        }
        dr = CR(LU, i, i);
        di = CI(LU, i, i);
        den = dr * dr + di * di;
        if (den == 0.0) {
            fprintf(stderr, "GSL shim: complex LU_solve on a singular matrix\n");
            abort();
        }
        y[2 * i] = (ar * dr + ai * di) / den;
        y[2 * i + 1] = (ai * dr - ar * di) / den;
    }
    for (i = 0; i < n; i++) {
        x->data[2 * i * x->stride] = y[2 * i];
        x->data[2 * i * x->stride + 1] = y[2 * i + 1];
    }
    free(y);
    return GSL_SUCCESS;
}

/* ------------------------------------------------------------------ */
/* complex helpers                                                    */
/* ------------------------------------------------------------------ */

gsl_complex gsl_complex_add(gsl_complex a, gsl_complex b) {
    gsl_complex z;
    z.dat[0] = a.dat[0] + b.dat[0];
    z.dat[1] = a.dat[1] + b.dat[1];
    return z;
}

gsl_complex gsl_complex_sub(gsl_complex a, gsl_complex b) {
    gsl_complex z;
    z.dat[0] = a.dat[0] - b.dat[0];
    z.dat[1] = a.dat[1] - b.dat[1];
    return z;
}

gsl_complex gsl_complex_mul(gsl_complex a, gsl_complex b) {
    gsl_complex z;
    z.dat[0] = a.dat[0] * b.dat[0] - a.dat[1] * b.dat[1];
    z.dat[1] = a.dat[0] * b.dat[1] + a.dat[1] * b.dat[0];
    return z;
}

/* ------------------------------------------------------------------ */
/* general real eigen-problem                                         */
/* ------------------------------------------------------------------ */

#include "gsl/ipg_eig4.h"

gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n) {
    gsl_eigen_nonsymmv_workspace *w = (gsl_eigen_nonsymmv_workspace *)calloc(
        1, sizeof(gsl_eigen_nonsymmv_workspace));
    w->size = n;
    w->work = NULL;
    return w;
}

void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w) { free(w); }

int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval,
                       gsl_matrix_complex *evec,
                       gsl_eigen_nonsymmv_workspace *w) {
    double a[16], er[4], ei[4], vr[16], vi[16];
    size_t i, j;
    (void)w;
    if (A->size1 != 4 || A->size2 != 4) shim_abort("nonsymmv for n != 4");
    for (i = 0; i < 4; i++)
        for (j = 0; j < 4; j++) a[4 * i + j] = RM(A, i, j);
    ipg_eig4(a, er, ei, vr, vi);
    for (i = 0; i < 4; i++) {
        eval->data[2 * i * eval->stride] = er[i];
        eval->data[2 * i * eval->stride + 1] = ei[i];
        for (j = 0; j < 4; j++) {
            /* column i holds eigenvector i */
            CR(evec, j, i) = vr[4 * i + j];
            CI(evec, j, i) = vi[4 * i + j];
        }
    }
    return GSL_SUCCESS;
}

/* ------------------------------------------------------------------ */
/* off-path pieces                                                    */
/* ------------------------------------------------------------------ */

static const gsl_rng_type taus_type = {"taus"};
const gsl_rng_type *gsl_rng_taus = &taus_type;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
    gsl_rng *r = (gsl_rng *)calloc(1, sizeof(gsl_rng));
    r->type = T;
    return r;
}

void gsl_rng_set(const gsl_rng *r, unsigned long seed) {
    ((gsl_rng *)r)->seed = seed;
}

void gsl_rng_free(gsl_rng *r) { free(r); }

unsigned int gsl_ran_poisson(const gsl_rng *r, double mu) {
    (void)r;
    (void)mu;
    shim_abort("gsl_ran_poisson");
    return 0;
}

unsigned int gsl_ran_negative_binomial(const gsl_rng *r, double p, double n) {
    (void)r;
    (void)p;
    (void)n;
    shim_abort("gsl_ran_negative_binomial");
    return 0;
}

double gsl_ran_tdist(const gsl_rng *r, double nu) {
    (void)r;
    (void)nu;
    shim_abort("gsl_ran_tdist");
    return 0.0;
}

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n) {
    (void)n;
    shim_abort("gsl_integration_glfixed_table_alloc");
    return NULL;
}

int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi,
                                  double *wi,
                                  const gsl_integration_glfixed_table *t) {
    (void)a;
    (void)b;
    (void)i;
    (void)xi;
    (void)wi;
    (void)t;
    shim_abort("gsl_integration_glfixed_point");
    return 0;
}

static const gsl_interp_type cspline_type = {"cspline"};
const gsl_interp_type *gsl_interp_cspline = &cspline_type;

gsl_interp_accel *gsl_interp_accel_alloc(void) {
    shim_abort("gsl_interp_accel_alloc");
    return NULL;
}

void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }

gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size) {
    (void)T;
    (void)size;
    shim_abort("gsl_spline_alloc");
    return NULL;
}

int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[],
                    size_t size) {
    (void)spline;
    (void)xa;
    (void)ya;
    (void)size;
    shim_abort("gsl_spline_init");
    return 0;
}

double gsl_spline_eval_integ(const gsl_spline *spline, double a, double b,
                             gsl_interp_accel *acc) {
    (void)spline;
    (void)a;
    (void)b;
    (void)acc;
    shim_abort("gsl_spline_eval_integ");
    return 0.0;
}

void gsl_spline_free(gsl_spline *spline) { free(spline); }
