/*
 * GSL stand-in implementations for compiling the reference CPU path
 * (src/utils.cpp:52-68, src/init.cpp:289-316) as a test oracle.
 * Backed by the project's table generator; see gsl/gsl_shim_types.h.
 */
#include "gsl/gsl_shim_types.h"
#include "../../c3d-2015_b200/host/tables.h"
#include <stdlib.h>
#include <string.h>

gsl_vector *gsl_vector_alloc(size_t n)
{
    gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
    v->size = n;
    v->stride = 1;
    v->data = (double *)calloc(n, sizeof(double));
    return v;
}
void gsl_vector_free(gsl_vector *v) { if (v) { free(v->data); free(v); } }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2)
{
    gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double *)calloc(n1 * n2, sizeof(double));
    return m;
}
void gsl_matrix_free(gsl_matrix *m) { if (m) { free(m->data); free(m); } }

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n)
{
    gsl_integration_glfixed_table *t = (gsl_integration_glfixed_table *)malloc(sizeof(*t));
    t->n = n;
    t->x = (double *)malloc(n * sizeof(double));
    t->w = (double *)malloc(n * sizeof(double));
    c3d_gauss_legendre((int)n, t->x, t->w);
    return t;
}
/* Points are returned in ascending order on [a,b]; for a=-1, b=1 they are the nodes themselves. */
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi,
                                  const gsl_integration_glfixed_table *t)
{
    double A = (b - a) / 2, B = (a + b) / 2;
    if (i >= t->n)
        return 1;
    *xi = B + A * t->x[i];
    *wi = A * t->w[i];
    return 0;
}
double gsl_sf_legendre_sphPlm(int l, int m, double x) { return c3d_sph_plm(l, m, x); }
int gsl_linalg_QR_decomp(gsl_matrix *A, gsl_vector *tau)
{
    c3d_qr_decomp((int)A->size1, (int)A->size2, A->data, tau->data);
    return 0;
}
int gsl_linalg_QR_lssolve(const gsl_matrix *QR, const gsl_vector *tau, const gsl_vector *b,
                          gsl_vector *x, gsl_vector *residual)
{
    c3d_qr_lssolve((int)QR->size1, (int)QR->size2, QR->data, tau->data, b->data, x->data,
                   residual ? residual->data : NULL);
    return 0;
}
