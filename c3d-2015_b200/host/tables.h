/*
 * Angular tables for the M_N / P_N moment closures: Gauss-Legendre nodes,
 * real orthonormal spherical harmonics, the tensor-product sphere quadrature
 * and the Gaunt least-squares coefficients.
 *
 * Plain C so that the C++ host and the C oracle consume bit-identical tables.
 *
 * Conventions follow ckrisgarrett/C3D-2015:
 *   nq  = 2 Q^2 points, q = 2*q1*Q + q2        (src/init.cpp:423,520)
 *   nm  = (N+1)^2 moments, ordered n=0..N, m=-n..n  (src/init.cpp:424,526-530)
 *   nm2 = (2N+1)^2 moments of degree <= 2N      (src/init.cpp:425,543-547)
 *   M[q*nm + k], M2[q*nm2 + k] row-major         (src/global.h:18-19)
 */
#ifndef C3D_TABLES_H
#define C3D_TABLES_H

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss-Legendre nodes mu[0..n-1] (ascending) and weights w[0..n-1] on [-1,1].
 * Replaces gsl_integration_glfixed_point(-1,1,i,...) as called at
 * src/utils.cpp:52-57. Newton iteration on P_n in long double, then rounded. */
void c3d_gauss_legendre(int n, double *mu, double *w);

/* Normalised associated Legendre function with the Condon-Shortley phase,
 * sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) P_l^m(x), 0 <= m <= l.
 * Same quantity as gsl_sf_legendre_sphPlm used at src/utils.cpp:60-68. */
double c3d_sph_plm(int l, int m, double x);

/* Real orthonormal spherical harmonic of degree n, order m (src/utils.cpp:60-68). */
double c3d_real_sh(int m, int n, double mu, double phi);

/* Tensor quadrature of src/init.cpp:509-548. Outputs (caller-allocated):
 *   w[nq], xi[nq], eta[nq], mu[nq], M[nq*nm] (degree <= N), M2[nq*nm2] (degree <= 2N; may be NULL). */
void c3d_build_quadrature(int momentOrder, int quadOrder, double *w, double *xi, double *eta,
                          double *mu, double *M, double *M2);

/* Householder QR least squares (replaces gsl_linalg_QR_decomp / QR_lssolve as
 * used at src/init.cpp:289-316). A is rows x cols row-major, rows >= cols.
 * c3d_qr_decomp overwrites A with R (upper) and the Householder vectors
 * (below the diagonal), tau[cols] receives the reflector scalars. */
void c3d_qr_decomp(int rows, int cols, double *A, double *tau);
/* Solves min ||A x - b|| given the factors. b[rows] is not modified. residual may be NULL. */
void c3d_qr_lssolve(int rows, int cols, const double *QR, const double *tau, const double *b,
                    double *x, double *residual);

/* Dense Gaunt coefficients beta[(i*nm+j)*nm2+k] so that m_i m_j = sum_k beta_ijk m2_k
 * at every quadrature point (least squares over the quadrature, src/init.cpp:288-316).
 * Returns the number of |beta| > 1e-13 entries (src/init.cpp:306-307). */
int c3d_gaunt_dense(int nm, int nm2, int nq, const double *M2, double *beta);

/* CSR form of the dense Gaunt table with |beta| > 1e-13 (src/init.cpp:318-336).
 * rowPtr[nm*nm+1]; val/colInd sized by c3d_gaunt_dense's return value. */
void c3d_gaunt_csr(int nm, int nm2, const double *beta, double *val, int *colInd, int *rowPtr);

/* CSR of the entries with |beta| > threshold (threshold 0: every nonzero, the dense
 * mode's terms). Returns nnz; val/colInd may be NULL to count only. */
int c3d_gaunt_csr_threshold(int nm, int nm2, const double *beta, double threshold, double *val,
                            int *colInd, int *rowPtr);

#ifdef __cplusplus
}
#endif
#endif
