/*
 * TEST INFRASTRUCTURE ONLY (see c3d_oracle.h): CPU restatement of the
 * reference M_N / P_N time step. Each function cites the reference lines it
 * follows. Arithmetic is written in the reference's operation order
 * (q-sequential sums, products left to right); compiled without FMA
 * contraction (x86-64 baseline, -O2).
 */
#include "c3d_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define MINV(a, b) (((a) < (b)) ? (a) : (b))
#define MAXV(a, b) (((a) > (b)) ? (a) : (b))
#define SIGNV(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))

/* ---------------------------------------------------------------- LAPACK-like */

/* Unblocked lower Cholesky (LAPACK dpotf2 form): column j from the dot product
 * of the rows, scaled by 1/L_jj. Column-major, lda = n. Returns info (0 ok,
 * j+1 if the j-th leading minor is not positive definite). */
int orc_potrf_lower(int n, double *a)
{
    for (int j = 0; j < n; j++) {
        double ajj = a[j + n * j];
        for (int k = 0; k < j; k++)
            ajj -= a[j + n * k] * a[j + n * k];
        if (ajj <= 0.0 || isnan(ajj)) {
            a[j + n * j] = ajj;
            return j + 1;
        }
        ajj = sqrt(ajj);
        a[j + n * j] = ajj;
        double r = 1.0 / ajj;
        for (int i = j + 1; i < n; i++) {
            double s = a[i + n * j];
            for (int k = 0; k < j; k++)
                s -= a[i + n * k] * a[j + n * k];
            a[i + n * j] = s * r;
        }
    }
    return 0;
}

/* x <- A^{-1} x with A = L L^T (forward then backward substitution). */
static void apply_inverse(int n, const double *l, double *x)
{
    for (int i = 0; i < n; i++) {
        double s = x[i];
        for (int k = 0; k < i; k++)
            s -= l[i + n * k] * x[k];
        x[i] = s / l[i + n * i];
    }
    /* L^T x = y with the reference BLAS dtrsv('L','T') order (descending k) */
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = n - 1; k > i; k--)
            s -= l[k + n * i] * x[k];
        x[i] = s / l[i + n * i];
    }
}

static double asum(int n, const double *x)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += fabs(x[i]);
    return s;
}

static int iamax(int n, const double *x)
{
    int j = 0;
    double m = fabs(x[0]);
    for (int i = 1; i < n; i++)
        if (fabs(x[i]) > m) {
            m = fabs(x[i]);
            j = i;
        }
    return j;
}

/* Reciprocal condition estimate of A = L L^T in the 1-norm, as dpocon:
 * ||A^{-1}||_1 by Hager's method with Higham's refinements (N. J. Higham,
 * ACM TOMS 14 (1988) 381-396, Alg. 4.1, the algorithm of LAPACK's dlacn2),
 * rcond = (1/ainvnm)/anorm. A is symmetric, so A^{-T} = A^{-1}. */
double orc_pocon_lower(int n, const double *l, double anorm)
{
    if (n == 0)
        return 1.0;
    if (anorm == 0.0)
        return 0.0;
    double x[256], v[256];
    int isgn[256];
    double est, estold;
    for (int i = 0; i < n; i++)
        x[i] = 1.0 / (double)n;
    apply_inverse(n, l, x);
    if (n == 1) {
        est = fabs(x[0]);
        goto done;
    }
    est = asum(n, x);
    for (int i = 0; i < n; i++) {
        x[i] = x[i] >= 0.0 ? 1.0 : -1.0;
        isgn[i] = (int)x[i];
    }
    apply_inverse(n, l, x);
    int j = iamax(n, x);
    int iter = 2;
    for (;;) {
        for (int i = 0; i < n; i++)
            x[i] = 0.0;
        x[j] = 1.0;
        apply_inverse(n, l, x);
        memcpy(v, x, sizeof(double) * n);
        estold = est;
        est = asum(n, v);
        int same = 1;
        for (int i = 0; i < n; i++) {
            int s = x[i] >= 0.0 ? 1 : -1;
            if (s != isgn[i]) {
                same = 0;
                break;
            }
        }
        if (same || est <= estold)
            break;
        for (int i = 0; i < n; i++) {
            x[i] = x[i] >= 0.0 ? 1.0 : -1.0;
            isgn[i] = (int)x[i];
        }
        apply_inverse(n, l, x);
        int jlast = j;
        j = iamax(n, x);
        if (x[jlast] != fabs(x[j]) && iter < 5) {
            iter++;
            continue;
        }
        break;
    }
    {
        double altsgn = 1.0;
        for (int i = 0; i < n; i++) {
            x[i] = altsgn * (1.0 + (double)i / (double)(n - 1));
            altsgn = -altsgn;
        }
        apply_inverse(n, l, x);
        double temp = 2.0 * (asum(n, x) / (double)(3 * n));
        if (temp > est)
            est = temp;
    }
done:
    if (est == 0.0)
        return 0.0;
    return (1.0 / est) / anorm;
}

/* The reference's own triangular solves, src/utils.cpp:71-86. */
void orc_potrs_lower(int n, const double *L, double *d)
{
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < i; j++)
            d[i] -= L[i + n * j] * d[j];
        d[i] = d[i] / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        for (int j = n - 1; j > i; j--)
            d[i] -= L[j + n * i] * d[j];
        d[i] = d[i] / L[i * n + i];
    }
}

/* Classic scaled two-norm (reference BLAS dnrm2). */
double orc_nrm2(int n, const double *x)
{
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; i++) {
        if (x[i] != 0.0) {
            double a = fabs(x[i]);
            if (scale < a) {
                ssq = 1.0 + ssq * (scale / a) * (scale / a);
                scale = a;
            } else {
                ssq += (a / scale) * (a / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

/* Max row sum of |A|, src/utils.cpp:35-49. */
double orc_norm1(int n, const double *A)
{
    double oneNorm = 0.0;
    for (int i = 0; i < n; i++) {
        double t = 0;
        for (int j = 0; j < n; j++)
            t += fabs(A[i * n + j]);
        if (t > oneNorm)
            oneNorm = t;
    }
    return oneNorm;
}

/* ---------------------------------------------------------------- closure */

/* solveHMn, src/opt/fobj.cpp:34-102. gext: nm2 scratch. */
static void hessian(const orc_closure_opts *o, const orc_tables *t, const double *alpha, double *h,
                    double *gext)
{
    int nm = o->nm, nm2 = o->nm2, nq = o->nq;
    const double *p = t->M, *p2 = t->M2, *w = t->w;
    for (int k = 0; k < nm2 && o->hessMode; k++)
        gext[k] = 0.0;
    for (int i = 0; i < nm * nm; i++)
        h[i] = 0.0;
    for (int q = 0; q < nq; q++) {
        double temp = 0;
        for (int i = 0; i < nm; i++)
            temp = temp + alpha[i] * p[q * nm + i];
        temp = exp(temp);
        if (o->hessMode) {
            for (int k = 0; k < nm2; k++)
                gext[k] += w[q] * p2[q * nm2 + k] * temp;
        } else {
            for (int i = 0; i < nm; i++) {
                double pi = p[q * nm + i];
                for (int j = 0; j <= i; j++) {
                    double pj = p[q * nm + j];
                    h[i * nm + j] += w[q] * pi * pj * temp;
                }
            }
        }
    }
    if (o->hessMode == 1) {
        for (int i = 0; i < nm; i++)
            for (int j = i; j < nm; j++) {
                double hij = 0.0;
                for (int k = 0; k < nm2; k++)
                    hij += gext[k] * t->beta[(i * nm + j) * nm2 + k];
                h[i * nm + j] = h[j * nm + i] = hij;
            }
    } else if (o->hessMode == 2) {
        for (int i = 0; i < nm; i++)
            for (int j = i; j < nm; j++) {
                double hij = 0.0;
                int idx = i * nm + j;
                for (int k = t->betaRow[idx]; k < t->betaRow[idx + 1]; k++)
                    hij += gext[t->betaCol[k]] * t->betaVal[k];
                h[i * nm + j] = h[j * nm + i] = hij;
            }
    } else {
        for (int i = 0; i < nm; i++)
            for (int j = i + 1; j < nm; j++)
                h[i * nm + j] = h[j * nm + i];
    }
}

void orc_hessian(const orc_closure_opts *o, const orc_tables *t, const double *alpha, double *h)
{
    double *gext = (double *)malloc(sizeof(double) * (o->nm2 > 0 ? o->nm2 : 1));
    hessian(o, t, alpha, h, gext);
    free(gext);
}

/* fobjMn with g = h = NULL, src/opt/fobj.cpp:135-164. */
static double fobj_f(int nm, int nq, const double *alpha, const double *u, const double *w,
                     const double *p)
{
    double f = 0.0;
    for (int q = 0; q < nq; q++) {
        double temp = 0;
        for (int i = 0; i < nm; i++)
            temp = temp + alpha[i] * p[q * nm + i];
        temp = exp(temp);
        f = f + w[q] * temp;
    }
    for (int i = 0; i < nm; i++)
        f = f - alpha[i] * u[i];
    return f;
}

/* linesearch, src/opt/linesearch.cpp:29-79. */
static double linesearch(int nm, int nq, double *alpha, const double *d, double f, const double *g,
                         const double *u, const double *w, const double *p, double *alphaOld,
                         double *armijoUlps)
{
    double t = 1.0, fNew, delta = 1e-3, beta = .5, maxFactor = 0, temp;
    for (int i = 0; i < nm; i++)
        alphaOld[i] = alpha[i];
    for (int i = 0; i < nm; i++) {
        temp = fabs(d[i]) / (fabs(alphaOld[i]) + 1e-100);
        if (temp > maxFactor)
            maxFactor = temp;
    }
    while (t * maxFactor > DBL_EPSILON / 2) {
        for (int i = 0; i < nm; i++)
            alpha[i] = alphaOld[i] + t * d[i];
        fNew = fobj_f(nm, nq, alpha, u, w, p);
        temp = 0.0;
        for (int i = 0; i < nm; i++)
            temp += g[i] * d[i];
        double rhs = f + delta * t * temp;
        double margin = fabs(fNew - rhs) / (DBL_EPSILON * fabs(f) + DBL_MIN);
        if (margin < *armijoUlps)
            *armijoUlps = margin;
        if (fNew <= rhs)
            return t;
        t = beta * t;
    }
    for (int i = 0; i < nm; i++)
        alpha[i] = alphaOld[i];
    return 0.0;
}

/* isotropicAlpha, src/opt/opt.cpp:105-111. */
static void isotropic_alpha(int n, double *alpha)
{
    alpha[0] = 2.0 * sqrt(M_PI) * log(0.5 / sqrt(M_PI));
    for (int i = 1; i < n; i++)
        alpha[i] = 0.0;
}

/* modcfl, src/opt/opt.cpp:117-132. */
static double modcfl(int n, const double *da)
{
    double da_1 = 0.0;
    for (int i = 0; i < n; i++)
        da_1 = da_1 + fabs(da[i]);
    int pnOrder = (int)floor(sqrt((double)n)) + 1;
    double m_inf = sqrt((2 * pnOrder + 1) / (2 * M_PI));
    return exp(2.0 * da_1 * m_inf);
}

/* optScaled (src/opt/opt.cpp:139-324) and the batched per-iteration step
 * solveTheRest (src/opt/optBatch.cpp:143-283) as one loop; o->batched picks the
 * stop rule: absolute MN_TOL with MN_TOL_GAMMA (batched) or |u| * MN_TOL with
 * gamma <= 1.1 (unbatched). Both use the same factorisation and solves. */
static int newton_scaled(const orc_closure_opts *o, const orc_tables *t, double *u, double *alpha,
                         orc_cell_out *out, double *work)
{
    int nm = o->nm, nq = o->nq;
    const double *p = t->M, *w = t->w;
    double *g = work;
    double *h = g + nm;
    double *d = h + nm * nm;
    double *chol = d + nm;
    double *uOrig = chol + nm * nm;
    double *alpha0 = uOrig + nm;
    double *alphaOld = alpha0 + nm;
    double *gext = alphaOld + nm;

    int maxIter = o->maxIter;
    double rtol = o->batched ? o->tol : orc_nrm2(nm, u) * o->tol;
    int iter = 0, totalIter = 0, iterGamma = 0, regIndex = 0;
    double tstep = 1, r = 0.0, gamma = 0.0, err = 0.0;
    double armijoUlps = 1e300, tolRel = 1e300, condRel = 1e300, gammaRel = 1e300, capHits = 0;
    int status = 0;

    for (int i = 0; i < nm; i++)
        alpha0[i] = alpha[i];
    for (int i = 0; i < nm; i++)
        uOrig[i] = u[i];

    for (;;) {
        int maxIterEff = maxIter;
        if (o->batched && regIndex == o->nreg - 1)
            maxIterEff = 10 * maxIter; /* src/opt/optBatch.cpp:183-184 */
        iter = iter + 1;
        totalIter = totalIter + 1;

        /* f, g from H (src/opt/fobj.cpp:118-131, :171-185) */
        hessian(o, t, alpha, h, gext);
        for (int i = 0; i < nm; i++)
            g[i] = h[i] / p[0] - u[i];
        double f = h[0] / (p[0] * p[0]);
        for (int i = 0; i < nm; i++)
            f = f - alpha[i] * u[i];

        memcpy(chol, h, sizeof(double) * nm * nm);
        int cholErr = orc_potrf_lower(nm, chol);
        double norm1 = orc_norm1(nm, h);
        double condest = orc_pocon_lower(nm, chol, norm1);
        condest = 1.0 / condest;
        if (cholErr == 0 && fabs(condest - o->condHMax) / o->condHMax < condRel)
            condRel = fabs(condest - o->condHMax) / o->condHMax;

        if (totalIter == 1 && (cholErr != 0 || condest > o->condHMax)) {
            isotropic_alpha(nm, alpha0);
            if (!o->batched)
                rtol = orc_nrm2(nm, u) * o->tol;
            memcpy(alpha, alpha0, sizeof(double) * nm);
            iter = 0;
            iterGamma = 0;
            tstep = 1;
            continue;
        }

        if (iter >= maxIterEff || cholErr != 0 || tstep == 0 || condest > o->condHMax) {
            if (iter >= maxIterEff)
                capHits += 1;
            if (regIndex < o->nreg - 1) {
                regIndex++;
                r = o->reg[regIndex];
                u[0] = 1.0;
                for (int i = 1; i < nm; i++)
                    u[i] = uOrig[i] * (1.0 - r);
            } else {
                status = 2; /* the reference aborts here (src/opt/opt.cpp:261-266) */
                break;
            }
            if (!o->batched)
                rtol = orc_nrm2(nm, u) * o->tol;
            memcpy(alpha, alpha0, sizeof(double) * nm);
            iterGamma = 0;
            iter = 0;
            tstep = 1;
            if (!o->batched && regIndex == o->nreg - 1)
                maxIter = 10 * maxIter;
            continue;
        }

        for (int i = 0; i < nm; i++)
            d[i] = g[i];
        orc_potrs_lower(nm, chol, d);
        for (int i = 0; i < nm; i++)
            d[i] = -d[i];

        err = orc_nrm2(nm, g);
        gamma = modcfl(nm, d);
        if (fabs(err - rtol) / rtol < tolRel)
            tolRel = fabs(err - rtol) / rtol;
        if (err <= rtol && fabs(gamma - o->tolGamma) / o->tolGamma < gammaRel)
            gammaRel = fabs(gamma - o->tolGamma) / o->tolGamma;

        if (err <= rtol && gamma <= o->tolGamma)
            break;
        else if (err <= rtol && gamma > o->tolGamma)
            iterGamma++;

        tstep = linesearch(nm, nq, alpha, d, f, g, u, w, p, alphaOld, &armijoUlps);
    }
    if (out) {
        out->totalIter = totalIter;
        out->iterGamma = iterGamma < 0 ? 0 : iterGamma;
        out->regIndex = regIndex;
        out->status = status;
        out->r = r;
        out->gamma = gamma;
        out->err = err;
        out->armijoUlps = armijoUlps;
        out->tolRel = tolRel;
        out->condRel = condRel;
        out->gammaRel = gammaRel;
        out->capHits = capHits;
    }
    return status;
}

/* opt(), src/opt/opt.cpp:330-355 (and preProcess/postProcess,
 * src/opt/optBatch.cpp:312-344, which scale identically). */
static int closure_cell(const orc_closure_opts *o, const orc_tables *t, double *u, double *alpha,
                        orc_cell_out *out, double *work)
{
    int nm = o->nm;
    double u0 = u[0];
    double alphaScale = log(u0) * 2.0 * sqrt(M_PI);
    alpha[0] = alpha[0] - alphaScale;
    for (int i = 0; i < nm; i++)
        u[i] = u[i] / u0;
    if (u0 <= 0) {
        if (out) {
            memset(out, 0, sizeof(*out));
            out->status = 1;
        }
        return 1;
    }
    int st = newton_scaled(o, t, u, alpha, out, work);
    for (int i = 0; i < nm; i++)
        u[i] = u[i] * u0;
    alpha[0] = alpha[0] + alphaScale;
    return st;
}

static size_t work_doubles(const orc_closure_opts *o)
{
    return (size_t)(6 * o->nm + 2 * o->nm * o->nm + (o->nm2 > 0 ? o->nm2 : 1) + 8);
}

int orc_closure_cell(const orc_closure_opts *o, const orc_tables *t, double *u, double *alpha,
                     orc_cell_out *out)
{
    double *work = (double *)malloc(sizeof(double) * work_doubles(o));
    int st = closure_cell(o, t, u, alpha, out, work);
    free(work);
    return st;
}

long orc_closure_many(const orc_closure_opts *o, const orc_tables *t, long ncells, double *u,
                      double *alpha, orc_cell_out *out)
{
    long bad = 0;
    #pragma omp parallel reduction(+ : bad)
    {
        double *work = (double *)malloc(sizeof(double) * work_doubles(o));
        #pragma omp for schedule(dynamic, 16)
        for (long c = 0; c < ncells; c++) {
            orc_cell_out tmp;
            int st = closure_cell(o, t, u + c * o->nm, alpha + c * o->nm, out ? out + c : &tmp,
                                  work);
            if (st)
                bad++;
        }
        free(work);
    }
    return bad;
}

/* ---------------------------------------------------------------- P_N operators */

/* initPn, src/init.cpp:199-234. ops: xi+, xi-, eta+, eta-, mu+, mu- (nm*nm each). */
void orc_pn_operators(int nm, int nq, const orc_tables *t, double *ops)
{
    const double *m = t->M, *w = t->w;
    for (int i = 0; i < nm; i++) {
        for (int j = 0; j < nm; j++) {
            double v[6] = {0, 0, 0, 0, 0, 0};
            for (int q = 0; q < nq; q++) {
                if (t->xi[q] > 0)
                    v[0] += t->xi[q] * m[q * nm + i] * m[q * nm + j] * w[q];
                else
                    v[1] += t->xi[q] * m[q * nm + i] * m[q * nm + j] * w[q];
                if (t->eta[q] > 0)
                    v[2] += t->eta[q] * m[q * nm + i] * m[q * nm + j] * w[q];
                else
                    v[3] += t->eta[q] * m[q * nm + i] * m[q * nm + j] * w[q];
                if (t->mu[q] > 0)
                    v[4] += t->mu[q] * m[q * nm + i] * m[q * nm + j] * w[q];
                else
                    v[5] += t->mu[q] * m[q * nm + i] * m[q * nm + j] * w[q];
            }
            for (int k = 0; k < 6; k++)
                ops[k * nm * nm + i * nm + j] = v[k];
        }
    }
}

/* ---------------------------------------------------------------- grid kernels */

#define NXG(g) ((g)->nx + 4)
#define NYG(g) ((g)->ny + 4)
#define NZG(g) ((g)->nz + 4)
#define C3(g, i, j, k) ((long)(k) + (long)NZG(g) * ((long)(j) + (long)NYG(g) * (long)(i)))

/* Serial periodic communicateBoundaries, src/comm.cpp:281-323. */
void orc_ghost_fill(const orc_grid *g, double *u)
{
    int nm = g->nm;
    int x0 = 0, x1 = 2, x2 = g->nx + 1 + 1 - 2, x3 = g->nx + 3 + 1 - 2;
    int y0 = 0, y1 = 2, y2 = g->ny + 1 + 1 - 2, y3 = g->ny + 3 + 1 - 2;
    int z0 = 0, z1 = 2, z2 = g->nz + 1 + 1 - 2, z3 = g->nz + 3 + 1 - 2;
    for (int i = 0; i < 2; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 2; k <= g->nz + 1; k++)
                for (int m = 0; m < nm; m++) {
                    u[C3(g, x0 + i, j, k) * nm + m] = u[C3(g, x2 + i, j, k) * nm + m];
                    u[C3(g, x3 + i, j, k) * nm + m] = u[C3(g, x1 + i, j, k) * nm + m];
                }
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 2; k <= g->nz + 1; k++)
                for (int m = 0; m < nm; m++) {
                    u[C3(g, i, y0 + j, k) * nm + m] = u[C3(g, i, y2 + j, k) * nm + m];
                    u[C3(g, i, y3 + j, k) * nm + m] = u[C3(g, i, y1 + j, k) * nm + m];
                }
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 0; k < 2; k++)
                for (int m = 0; m < nm; m++) {
                    u[C3(g, i, j, z0 + k) * nm + m] = u[C3(g, i, j, z2 + k) * nm + m];
                    u[C3(g, i, j, z3 + k) * nm + m] = u[C3(g, i, j, z1 + k) * nm + m];
                }
}

/* minmod / slopefit, src/flux_kinetic.cpp:45-60. */
static inline double minmod(double x, double y)
{
    return SIGNV(1.0, x) * MAXV(0.0, MINV(fabs(x), y * SIGNV(1.0, x)));
}
static inline double slopefit(double theta, double left, double center, double right)
{
    return minmod(theta * (right - center), minmod(0.5 * (right - left), theta * (center - left)));
}

/* solveFluxKinetic CPU path, src/flux_kinetic.cpp:66-198. ansatz: ncellsAll scratch. */
void orc_flux_kinetic(const orc_grid *g, const orc_tables *t, const double *alpha, int isPn,
                      double *flux, double *ansatz)
{
    int nm = g->nm, nq = g->nq;
    const double *M = t->M;
    double th = g->theta;
    #pragma omp parallel for
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 2; k <= g->nz + 1; k++)
                for (int m = 0; m < nm; m++)
                    flux[C3(g, i, j, k) * nm + m] = 0.0;

    for (int q = 0; q < nq; q++) {
        #pragma omp parallel for
        for (int i = 0; i < NXG(g); i++)
            for (int j = 0; j < NYG(g); j++)
                for (int k = 0; k < NZG(g); k++) {
                    long c = C3(g, i, j, k);
                    double kin = 0.0;
                    for (int m = 0; m < nm; m++)
                        kin += alpha[c * nm + m] * M[q * nm + m];
                    ansatz[c] = isPn ? kin : exp(kin);
                }
        double xq = t->xi[q], eq = t->eta[q], mq = t->mu[q], wq = t->w[q];
        #pragma omp parallel for
        for (int i = 2; i <= g->nx + 1; i++)
            for (int j = 2; j <= g->ny + 1; j++)
                for (int k = 2; k <= g->nz + 1; k++) {
                    double k1, k2, k3, k4, fx, fy, fz;
                    if (xq > 0) {
                        k1 = ansatz[C3(g, i - 2, j, k)]; k2 = ansatz[C3(g, i - 1, j, k)];
                        k3 = ansatz[C3(g, i, j, k)];     k4 = ansatz[C3(g, i + 1, j, k)];
                        fx = k3 + 0.5 * slopefit(th, k2, k3, k4) - k2 - 0.5 * slopefit(th, k1, k2, k3);
                    } else {
                        k1 = ansatz[C3(g, i - 1, j, k)]; k2 = ansatz[C3(g, i, j, k)];
                        k3 = ansatz[C3(g, i + 1, j, k)]; k4 = ansatz[C3(g, i + 2, j, k)];
                        fx = k3 - 0.5 * slopefit(th, k2, k3, k4) - k2 + 0.5 * slopefit(th, k1, k2, k3);
                    }
                    fx = fx * xq * wq;
                    if (eq > 0) {
                        k1 = ansatz[C3(g, i, j - 2, k)]; k2 = ansatz[C3(g, i, j - 1, k)];
                        k3 = ansatz[C3(g, i, j, k)];     k4 = ansatz[C3(g, i, j + 1, k)];
                        fy = k3 + 0.5 * slopefit(th, k2, k3, k4) - k2 - 0.5 * slopefit(th, k1, k2, k3);
                    } else {
                        k1 = ansatz[C3(g, i, j - 1, k)]; k2 = ansatz[C3(g, i, j, k)];
                        k3 = ansatz[C3(g, i, j + 1, k)]; k4 = ansatz[C3(g, i, j + 2, k)];
                        fy = k3 - 0.5 * slopefit(th, k2, k3, k4) - k2 + 0.5 * slopefit(th, k1, k2, k3);
                    }
                    fy = fy * eq * wq;
                    if (mq > 0) {
                        k1 = ansatz[C3(g, i, j, k - 2)]; k2 = ansatz[C3(g, i, j, k - 1)];
                        k3 = ansatz[C3(g, i, j, k)];     k4 = ansatz[C3(g, i, j, k + 1)];
                        fz = k3 + 0.5 * slopefit(th, k2, k3, k4) - k2 - 0.5 * slopefit(th, k1, k2, k3);
                    } else {
                        k1 = ansatz[C3(g, i, j, k - 1)]; k2 = ansatz[C3(g, i, j, k)];
                        k3 = ansatz[C3(g, i, j, k + 1)]; k4 = ansatz[C3(g, i, j, k + 2)];
                        fz = k3 - 0.5 * slopefit(th, k2, k3, k4) - k2 + 0.5 * slopefit(th, k1, k2, k3);
                    }
                    fz = fz * mq * wq;
                    long c = C3(g, i, j, k);
                    for (int m = 0; m < nm; m++)
                        flux[c * nm + m] += M[q * nm + m] * (fx / g->dx + fy / g->dy + fz / g->dz);
                }
    }
}

/* mvProduct, src/flux_moment.cpp:15-24. */
static void mv_product(int n, double beta, const double *A, const double *x, double *b)
{
    for (int i = 0; i < n; i++)
        b[i] = beta * b[i];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            b[i] += A[i * n + j] * x[j];
}

/* solveFluxMoment, src/flux_moment.cpp:30-104. */
void orc_flux_moment(const orc_grid *g, const orc_tables *t, const double *u, double *flux)
{
    int nm = g->nm;
    const double *ops = t->pnops;
    #pragma omp parallel
    {
        /* zeroed: mvProduct scales b by beta = 0 before accumulating (src/flux_moment.cpp:17) */
        double *tmp = (double *)calloc((size_t)nm * 4, sizeof(double));
        double *xf = tmp + nm, *yf = xf + nm, *zf = yf + nm;
        #pragma omp for
        for (int i = 2; i <= g->nx + 1; i++)
            for (int j = 2; j <= g->ny + 1; j++)
                for (int k = 2; k <= g->nz + 1; k++) {
#define U(a, b, c, m) u[C3(g, a, b, c) * nm + (m)]
                    for (int m = 0; m < nm; m++)
                        tmp[m] = 0.25 * U(i + 1, j, k, m) + 0.75 * U(i, j, k, m) -
                                 1.25 * U(i - 1, j, k, m) + 0.25 * U(i - 2, j, k, m);
                    mv_product(nm, 0.0, ops + 0 * nm * nm, tmp, xf);
                    for (int m = 0; m < nm; m++)
                        tmp[m] = -0.25 * U(i + 2, j, k, m) + 1.25 * U(i + 1, j, k, m) -
                                 0.75 * U(i, j, k, m) - 0.25 * U(i - 1, j, k, m);
                    mv_product(nm, 1.0, ops + 1 * nm * nm, tmp, xf);
                    for (int m = 0; m < nm; m++)
                        tmp[m] = 0.25 * U(i, j + 1, k, m) + 0.75 * U(i, j, k, m) -
                                 1.25 * U(i, j - 1, k, m) + 0.25 * U(i, j - 2, k, m);
                    mv_product(nm, 0.0, ops + 2 * nm * nm, tmp, yf);
                    for (int m = 0; m < nm; m++)
                        tmp[m] = -0.25 * U(i, j + 2, k, m) + 1.25 * U(i, j + 1, k, m) -
                                 0.75 * U(i, j, k, m) - 0.25 * U(i, j - 1, k, m);
                    mv_product(nm, 1.0, ops + 3 * nm * nm, tmp, yf);
                    for (int m = 0; m < nm; m++)
                        tmp[m] = 0.25 * U(i, j, k + 1, m) + 0.75 * U(i, j, k, m) -
                                 1.25 * U(i, j, k - 1, m) + 0.25 * U(i, j, k - 2, m);
                    mv_product(nm, 0.0, ops + 4 * nm * nm, tmp, zf);
                    for (int m = 0; m < nm; m++)
                        tmp[m] = -0.25 * U(i, j, k + 2, m) + 1.25 * U(i, j, k + 1, m) -
                                 0.75 * U(i, j, k, m) - 0.25 * U(i, j, k - 1, m);
                    mv_product(nm, 1.0, ops + 5 * nm * nm, tmp, zf);
#undef U
                    long c = C3(g, i, j, k);
                    for (int m = 0; m < nm; m++)
                        flux[c * nm + m] = xf[m] / g->dx + yf[m] / g->dy + zf[m] / g->dz;
                }
        free(tmp);
    }
}

/* eulerStep, src/update.cpp:21-37. */
void orc_euler(const orc_grid *g, double *u, const double *flux, const double *sigT,
               const double *sigS, double dt)
{
    int nm = g->nm;
    #pragma omp parallel for
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 2; k <= g->nz + 1; k++) {
                long c = C3(g, i, j, k);
                u[c * nm] = u[c * nm] * (1.0 + dt * sigS[c] - dt * sigT[c]) - dt * flux[c * nm];
                for (int m = 1; m < nm; m++)
                    u[c * nm + m] = u[c * nm + m] * (1.0 - dt * sigT[c]) - dt * flux[c * nm + m];
            }
}

/* update(), src/update.cpp:185-275. */
long orc_step(const orc_grid *g, const orc_closure_opts *o, const orc_tables *t, int solver,
              int pnKinetic, double *u, double *alpha, const double *sigT, const double *sigS,
              double dt, orc_cell_out *records, double *scratch)
{
    int nm = g->nm;
    long nall = (long)NXG(g) * NYG(g) * NZG(g);
    double *uOld = scratch;
    double *flux = uOld + nall * nm;
    double *ansatz = flux + nall * nm;
    long bad = 0;
    #pragma omp parallel for
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 2; k <= g->nz + 1; k++)
                for (int m = 0; m < nm; m++)
                    uOld[C3(g, i, j, k) * nm + m] = u[C3(g, i, j, k) * nm + m];
    for (int s = 0; s < 2; s++) {
        orc_ghost_fill(g, u);
        if (solver == 1) {
            bad += orc_closure_many(o, t, nall, u, alpha, records ? records + s * nall : NULL);
            orc_flux_kinetic(g, t, alpha, 0, flux, ansatz);
        } else if (!pnKinetic) {
            orc_flux_moment(g, t, u, flux);
        } else {
            orc_flux_kinetic(g, t, u, 1, flux, ansatz);
        }
        orc_euler(g, u, flux, sigT, sigS, dt);
    }
    #pragma omp parallel for
    for (int i = 2; i <= g->nx + 1; i++)
        for (int j = 2; j <= g->ny + 1; j++)
            for (int k = 2; k <= g->nz + 1; k++)
                for (int m = 0; m < nm; m++) {
                    long c = C3(g, i, j, k) * nm + m;
                    u[c] = 0.5 * (u[c] + uOld[c]);
                }
    return bad;
}
