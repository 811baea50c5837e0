/*
 * Fortran LAPACK/BLAS names the reference calls (src/utils.h:26-58), forwarded
 * to the scipy_-prefixed exports of the OpenBLAS that ships inside scipy
 * (no system LAPACK in this image). Test infrastructure only.
 */
extern void scipy_dpotrf_(char *, int *, double *, int *, int *);
extern void scipy_dpocon_(char *, int *, double *, int *, double *, double *, double *, int *, int *);
extern void scipy_dpotrs_(char *, int *, int *, double *, int *, double *, int *, int *);
extern double scipy_dnrm2_(int *, double *, int *);

double dpotrf_(char *uplo, int *n, double *a, int *lda, int *info)
{
    scipy_dpotrf_(uplo, n, a, lda, info);
    return 0.0;
}
double dpocon_(char *uplo, int *n, double *a, int *lda, double *anorm, double *rcond, double *work,
               int *iwork, int *info)
{
    scipy_dpocon_(uplo, n, a, lda, anorm, rcond, work, iwork, info);
    return 0.0;
}
double dpotrs_(char *uplo, int *n, int *nrhs, double *a, int *lda, double *b, int *ldb, int *info)
{
    scipy_dpotrs_(uplo, n, nrhs, a, lda, b, ldb, info);
    return 0.0;
}
double dnrm2_(int *n, double *x, int *incx) { return scipy_dnrm2_(n, x, incx); }
