/*
 * TEST INFRASTRUCTURE ONLY: a CPU restatement of the M_N / P_N time step of
 * ckrisgarrett/C3D-2015, used by tests/ and by bench.py's CPU-baseline leg to
 * check the B200 kernels. Nothing in the product links or calls this code.
 *
 * Layouts match the reference: cell-major arrays over the grid with two
 * ghost layers per face, moment index fastest (IU, src/global.h:16), cells
 * ordered with k fastest (I3D, src/global.h:15); tables row-major M[q*nm+m].
 *
 * LAPACK calls of the reference (dpotrf_, dpocon_, dpotrs_, dnrm2_) are
 * restated from the published algorithms (unblocked Cholesky; Hager's 1-norm
 * estimator with Higham's refinements as in LAPACK's dlacn2; classic scaled
 * two-norm), so results agree with the reference to rounding, not bit for bit.
 */
#ifndef C3D_ORACLE_H
#define C3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nm, nm2, nq;
    int batched;        /* 1: src/opt/optBatch.cpp rules, 0: src/opt/opt.cpp rules */
    int maxIter;        /* MN_MAX_ITER */
    double tol;         /* MN_TOL: absolute (batched) or relative to |u| (unbatched) */
    double tolGamma;    /* MN_TOL_GAMMA (batched); 1.1 for unbatched (src/update.cpp:57) */
    double condHMax;    /* MN_COND_H_MAX */
    int hessMode;       /* 0 direct, 1 Gaunt dense, 2 Gaunt sparse (src/opt/fobj.cpp:58-101) */
    int nreg;           /* regularisation ladder (src/opt/opt.h:37-38) */
    double reg[16];
} orc_closure_opts;

typedef struct {
    int totalIter;      /* OUTS.iter / c_totalIter */
    int iterGamma;
    int regIndex;
    int status;         /* 0 ok, 1 u0 <= 0, 2 ladder exhausted */
    double r, gamma, err;
    /* Smallest decision margins met during the solve, used to classify
     * rounding ties: |fNew - (f + delta t g.d)| in units of eps*|f| over all
     * Armijo tests, |err - tol| / tol over all stop tests, and
     * |condest - condHMax| / condHMax over all condition tests of a successful
     * factorisation, |gamma - tolGamma| / tolGamma over the stop tests whose
     * gradient passed; capHits counts regularisations forced by the iteration cap. */
    double armijoUlps, tolRel, condRel, gammaRel, capHits;
} orc_cell_out;

typedef struct {
    const double *M, *M2, *w, *xi, *eta, *mu;
    const double *beta;                         /* dense Gaunt, may be NULL */
    const double *betaVal; const int *betaCol, *betaRow; /* CSR Gaunt, may be NULL */
    const double *pnops;                        /* 6*nm*nm: xi+, xi-, eta+, eta-, mu+, mu- */
} orc_tables;

typedef struct {
    int nx, ny, nz;     /* interior cells per axis; arrays hold (n+4) per axis */
    int nm, nq;
    double dx, dy, dz;
    double theta;       /* THETA of slopefit (src/flux_kinetic.cpp:55-60) */
} orc_grid;

/* One dual solve, in place on u[nm] and alpha[nm] (src/opt/opt.cpp:330-355 and
 * src/opt/optBatch.cpp:143-344 with preProcess/postProcess). Returns status. */
int orc_closure_cell(const orc_closure_opts *o, const orc_tables *t, double *u, double *alpha,
                     orc_cell_out *out);
/* All ncells cells (OpenMP); out may be NULL. Returns the number of cells with status != 0. */
long orc_closure_many(const orc_closure_opts *o, const orc_tables *t, long ncells, double *u,
                      double *alpha, orc_cell_out *out);

/* H (row-major, full symmetric), from solveHMn (src/opt/fobj.cpp:34-102). */
void orc_hessian(const orc_closure_opts *o, const orc_tables *t, const double *alpha, double *h);

void orc_pn_operators(int nm, int nq, const orc_tables *t, double *ops);
void orc_ghost_fill(const orc_grid *g, double *u);
void orc_flux_kinetic(const orc_grid *g, const orc_tables *t, const double *alpha, int isPn,
                      double *flux, double *ansatzScratch);
void orc_flux_moment(const orc_grid *g, const orc_tables *t, const double *u, double *flux);
void orc_euler(const orc_grid *g, double *u, const double *flux, const double *sigT,
               const double *sigS, double dt);

/* One SSP-RK2 step in the order of update() (src/update.cpp:185-275).
 * solver: 1 M_N, 0 P_N. records: 2*ncellsAll entries (stage-major) or NULL.
 * scratch: 2*ncellsAll*nm + ncellsAll doubles. Returns cells with status != 0. */
long orc_step(const orc_grid *g, const orc_closure_opts *o, const orc_tables *t, int solver,
              int pnKinetic, double *u, double *alpha, const double *sigT, const double *sigS,
              double dt, orc_cell_out *records, double *scratch);

/* LAPACK-equivalents, exposed for unit tests (column-major lower L, lda = n). */
int orc_potrf_lower(int n, double *a);
double orc_pocon_lower(int n, const double *l, double anorm);   /* returns rcond */
void orc_potrs_lower(int n, const double *l, double *d);         /* src/utils.cpp:71-86 */
double orc_nrm2(int n, const double *x);
double orc_norm1(int n, const double *a);                       /* src/utils.cpp:35-49 */

#ifdef __cplusplus
}
#endif
#endif
