/*
 * Minimal stand-ins for the three GSL facilities the reference's setup code
 * calls (Gauss-Legendre table, normalised Legendre function, Householder QR
 * least squares). GSL is not installed in this image; the numerics come from
 * the project's own table generator (c3d-2015_b200/host/tables.c), so the
 * reference build and the B200 host consume identical M, M2, w and Omega.
 * Test infrastructure only: used to compile the reference CPU path as an oracle.
 */
#ifndef C3D_GSL_SHIM_TYPES_H
#define C3D_GSL_SHIM_TYPES_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct { size_t size; size_t stride; double *data; } gsl_vector;
typedef struct { size_t size1; size_t size2; size_t tda; double *data; } gsl_matrix;
typedef struct { size_t n; double *x; double *w; } gsl_integration_glfixed_table;

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
double gsl_vector_get(const gsl_vector *v, size_t i);
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n);
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi,
                                  const gsl_integration_glfixed_table *t);
double gsl_sf_legendre_sphPlm(int l, int m, double x);
int gsl_linalg_QR_decomp(gsl_matrix *A, gsl_vector *tau);
int gsl_linalg_QR_lssolve(const gsl_matrix *QR, const gsl_vector *tau, const gsl_vector *b,
                          gsl_vector *x, gsl_vector *residual);
#ifdef __cplusplus
}
#endif
#endif
