/*
 * Angular tables for the moment closures (see tables.h).
 *
 * Gauss-Legendre: Newton's method on the three-term Legendre recurrence,
 * evaluated in long double (64-bit mantissa on x86-64) and rounded once to
 * double, so nodes and weights are accurate to the last double bit in almost
 * all cases. Nodes are mirrored exactly about 0, ascending order, as returned
 * by gsl_integration_glfixed_point(-1, 1, i, ...) (src/utils.cpp:52-57).
 *
 * Associated Legendre: the standard normalised recurrence (diagonal start
 * P~_m^m, one step to P~_{m+1}^m, then upward in l), also in long double.
 *
 * Least squares: Householder QR without pivoting (Golub & Van Loan,
 * Matrix Computations, Alg. 5.2.1), then R x = Q^T b.
 */
#include "tables.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_SQRT2
#define M_SQRT2 1.41421356237309504880
#endif

static const long double PI_L = 3.141592653589793238462643383279502884L;

/* Evaluates P_n(z) and P_{n-1}(z) by the three-term recurrence. */
static void legendre_pair(int n, long double z, long double *pn, long double *pnm1)
{
    long double p1 = 1.0L, p2 = 0.0L;
    for (int j = 1; j <= n; j++) {
        long double p3 = p2;
        p2 = p1;
        p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / (long double)j;
    }
    *pn = p1;
    *pnm1 = p2;
}

void c3d_gauss_legendre(int n, double *mu, double *w)
{
    int half = (n + 1) / 2;
    for (int i = 0; i < half; i++) {
        /* i-th largest root; classical asymptotic start value */
        long double z = cosl(PI_L * (i + 0.75L) / (n + 0.5L));
        long double pn, pnm1, dp;
        for (int it = 0; it < 100; it++) {
            legendre_pair(n, z, &pn, &pnm1);
            dp = n * (z * pn - pnm1) / (z * z - 1.0L);
            long double dz = pn / dp;
            z -= dz;
            if (fabsl(dz) <= 1e-19L * (1.0L + fabsl(z)))
                break;
        }
        /* one more polish step and the derivative at the final node */
        legendre_pair(n, z, &pn, &pnm1);
        dp = n * (z * pn - pnm1) / (z * z - 1.0L);
        z -= pn / dp;
        legendre_pair(n, z, &pn, &pnm1);
        dp = n * (z * pn - pnm1) / (z * z - 1.0L);
        long double wt = 2.0L / ((1.0L - z * z) * dp * dp);

        if ((n & 1) && i == half - 1) {
            /* middle node of an odd rule is exactly zero */
            mu[i] = 0.0;
            w[i] = (double)wt;
        } else {
            mu[n - 1 - i] = (double)z;
            mu[i] = -(double)z;
            w[i] = (double)wt;
            w[n - 1 - i] = (double)wt;
        }
    }
}

double c3d_sph_plm(int l, int m, double x)
{
    if (m < 0 || m > l)
        return 0.0;
    long double xx = x;
    long double s = sqrtl((1.0L - xx) * (1.0L + xx));
    /* P~_m^m = (-1)^m sqrt((2m+1)/(4 pi)) sqrt(prod_{k<=m} (2k-1)/(2k)) s^m */
    long double pmm = 1.0L / sqrtl(4.0L * PI_L);
    for (int k = 1; k <= m; k++)
        pmm *= -s * sqrtl((2.0L * k - 1.0L) / (2.0L * k));
    pmm *= sqrtl(2.0L * m + 1.0L);
    if (l == m)
        return (double)pmm;

    long double pm1 = xx * sqrtl(2.0L * m + 3.0L) * pmm; /* P~_{m+1}^m */
    if (l == m + 1)
        return (double)pm1;

    long double pm2 = pmm, cur = pm1;
    for (int ll = m + 2; ll <= l; ll++) {
        long double L = ll, M = m;
        long double a = sqrtl((4.0L * L * L - 1.0L) / (L * L - M * M));
        long double b = sqrtl(((L - 1.0L) * (L - 1.0L) - M * M) /
                              (4.0L * (L - 1.0L) * (L - 1.0L) - 1.0L));
        long double next = a * (xx * cur - b * pm2);
        pm2 = cur;
        cur = next;
    }
    return (double)cur;
}

double c3d_real_sh(int m, int n, double mu, double phi)
{
    /* double arithmetic in the order of src/utils.cpp:62-67 */
    if (m < 0)
        return M_SQRT2 * sin(m * phi) * c3d_sph_plm(n, -m, mu);
    else if (m > 0)
        return M_SQRT2 * cos(m * phi) * c3d_sph_plm(n, m, mu);
    return c3d_sph_plm(n, 0, mu);
}

void c3d_build_quadrature(int momentOrder, int quadOrder, double *w, double *xi, double *eta,
                          double *mu, double *M, double *M2)
{
    int Q = quadOrder;
    int nm = (momentOrder + 1) * (momentOrder + 1);
    int nm2 = (2 * momentOrder + 1) * (2 * momentOrder + 1);
    double *wgl = (double *)malloc(sizeof(double) * Q);
    double *mugl = (double *)malloc(sizeof(double) * Q);
    double *phi = (double *)malloc(sizeof(double) * 2 * Q);

    c3d_gauss_legendre(Q, mugl, wgl);
    for (int k = 0; k < 2 * Q; k++)
        phi[k] = (k + 0.5) * M_PI / Q; /* src/init.cpp:512-513 */

    for (int q1 = 0; q1 < Q; q1++) {
        for (int q2 = 0; q2 < 2 * Q; q2++) {
            int q = 2 * q1 * Q + q2;
            w[q] = M_PI / Q * wgl[q1];
            xi[q] = sqrt(1.0 - mugl[q1] * mugl[q1]) * cos(phi[q2]);
            eta[q] = sqrt(1.0 - mugl[q1] * mugl[q1]) * sin(phi[q2]);
            mu[q] = mugl[q1];
            int k = 0;
            for (int n = 0; n <= momentOrder; n++)
                for (int m = -n; m <= n; m++)
                    M[q * nm + k++] = c3d_real_sh(m, n, mugl[q1], phi[q2]);
            if (M2) {
                k = 0;
                for (int n = 0; n <= 2 * momentOrder; n++)
                    for (int m = -n; m <= n; m++)
                        M2[q * nm2 + k++] = c3d_real_sh(m, n, mugl[q1], phi[q2]);
            }
        }
    }
    free(wgl);
    free(mugl);
    free(phi);
}

/* Householder vector for x[0..n-1] with stride; returns tau, leaves beta in x[0]
 * and v[1..] (v[0] = 1 implicit) in x[1..]. */
static double householder(int n, double *x, int stride)
{
    if (n <= 1)
        return 0.0;
    double xnorm = 0.0;
    {
        /* scaled two-norm of x[1..] */
        double scale = 0.0, ssq = 1.0;
        for (int i = 1; i < n; i++) {
            double a = fabs(x[i * stride]);
            if (a != 0.0) {
                if (scale < a) {
                    ssq = 1.0 + ssq * (scale / a) * (scale / a);
                    scale = a;
                } else {
                    ssq += (a / scale) * (a / scale);
                }
            }
        }
        xnorm = scale * sqrt(ssq);
    }
    if (xnorm == 0.0)
        return 0.0;
    double alpha = x[0];
    double beta = -(alpha >= 0.0 ? 1.0 : -1.0) * hypot(alpha, xnorm);
    double tau = (beta - alpha) / beta;
    double s = alpha - beta;
    for (int i = 1; i < n; i++)
        x[i * stride] /= s;
    x[0] = beta;
    return tau;
}

void c3d_qr_decomp(int rows, int cols, double *A, double *tau)
{
    for (int j = 0; j < cols; j++) {
        double t = householder(rows - j, &A[j * cols + j], cols);
        tau[j] = t;
        if (t == 0.0)
            continue;
        /* apply (I - t v v^T) to columns j+1.. of rows j.. */
        for (int c = j + 1; c < cols; c++) {
            double dot = A[j * cols + c];
            for (int r = j + 1; r < rows; r++)
                dot += A[r * cols + j] * A[r * cols + c];
            dot *= t;
            A[j * cols + c] -= dot;
            for (int r = j + 1; r < rows; r++)
                A[r * cols + c] -= dot * A[r * cols + j];
        }
    }
}

void c3d_qr_lssolve(int rows, int cols, const double *QR, const double *tau, const double *b,
                    double *x, double *residual)
{
    double *y = (double *)malloc(sizeof(double) * rows);
    memcpy(y, b, sizeof(double) * rows);
    /* y = Q^T b */
    for (int j = 0; j < cols; j++) {
        if (tau[j] == 0.0)
            continue;
        double dot = y[j];
        for (int r = j + 1; r < rows; r++)
            dot += QR[r * cols + j] * y[r];
        dot *= tau[j];
        y[j] -= dot;
        for (int r = j + 1; r < rows; r++)
            y[r] -= dot * QR[r * cols + j];
    }
    /* R x = y[0..cols-1] */
    for (int i = cols - 1; i >= 0; i--) {
        double s = y[i];
        for (int k = i + 1; k < cols; k++)
            s -= QR[i * cols + k] * x[k];
        x[i] = s / QR[i * cols + i];
    }
    if (residual) {
        /* residual = Q [0; y(cols:)] */
        for (int i = 0; i < cols; i++)
            y[i] = 0.0;
        for (int j = cols - 1; j >= 0; j--) {
            if (tau[j] == 0.0)
                continue;
            double dot = y[j];
            for (int r = j + 1; r < rows; r++)
                dot += QR[r * cols + j] * y[r];
            dot *= tau[j];
            y[j] -= dot;
            for (int r = j + 1; r < rows; r++)
                y[r] -= dot * QR[r * cols + j];
        }
        memcpy(residual, y, sizeof(double) * rows);
    }
    free(y);
}

int c3d_gaunt_dense(int nm, int nm2, int nq, const double *M2, double *beta)
{
    double *A = (double *)malloc(sizeof(double) * nq * nm2);
    double *tau = (double *)malloc(sizeof(double) * nm2);
    double *b = (double *)malloc(sizeof(double) * nq);
    double *x = (double *)malloc(sizeof(double) * nm2);
    int nnz = 0;
    memcpy(A, M2, sizeof(double) * nq * nm2);
    c3d_qr_decomp(nq, nm2, A, tau);
    for (int i = 0; i < nm; i++) {
        for (int j = 0; j < nm; j++) {
            for (int q = 0; q < nq; q++)
                b[q] = M2[q * nm2 + i] * M2[q * nm2 + j];
            c3d_qr_lssolve(nq, nm2, A, tau, b, x, NULL);
            for (int k = 0; k < nm2; k++) {
                beta[(i * nm + j) * nm2 + k] = x[k];
                if (fabs(x[k]) > 1e-13)
                    nnz++;
            }
        }
    }
    free(A);
    free(tau);
    free(b);
    free(x);
    return nnz;
}

void c3d_gaunt_csr(int nm, int nm2, const double *beta, double *val, int *colInd, int *rowPtr)
{
    int ptr = 0;
    for (int idx = 0; idx < nm * nm; idx++) {
        rowPtr[idx] = ptr;
        for (int k = 0; k < nm2; k++) {
            double v = beta[idx * nm2 + k];
            if (fabs(v) > 1e-13) {
                val[ptr] = v;
                colInd[ptr] = k;
                ptr++;
            }
        }
    }
    rowPtr[nm * nm] = ptr;
}

int c3d_gaunt_csr_threshold(int nm, int nm2, const double *beta, double threshold, double *val,
                            int *colInd, int *rowPtr)
{
    int ptr = 0;
    for (int idx = 0; idx < nm * nm; idx++) {
        if (rowPtr)
            rowPtr[idx] = ptr;
        for (int k = 0; k < nm2; k++) {
            double v = beta[idx * nm2 + k];
            if (fabs(v) > threshold) {
                if (val)
                    val[ptr] = v;
                if (colInd)
                    colInd[ptr] = k;
                ptr++;
            }
        }
    }
    if (rowPtr)
        rowPtr[nm * nm] = ptr;
    return ptr;
}
