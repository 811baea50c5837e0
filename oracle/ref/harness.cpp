/*
 * ctypes-facing harness around the reference CPU path (ckrisgarrett/C3D-2015),
 * compiled together with the reference's unmodified sources into
 * oracle/_ref/libc3dref.so. Test infrastructure only: used by tests/ and by
 * bench.py's CPU-baseline leg, never by the product.
 *
 * The reference keeps all state in process globals (src/global.h:64-129) and
 * reads "input.deck" from the working directory (src/init.cpp:362), so one
 * process holds one problem.
 *
 * c3dref_step_traced() re-composes update() (src/update.cpp:185-275) from the
 * reference's own public pieces (communicateBoundaries, Optimization::opt /
 * opt, solveFluxKinetic / solveFluxMoment) so that per-cell iteration counts
 * can be recorded. The Euler stage (a file-static function in update.cpp) is
 * restated below with the same expression. A test checks that it reproduces
 * update() bit for bit.
 */
#include "global.h"
#include "opt/opt.h"
#include "utils.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

extern "C" {
int c3dref_num_regularizations = 5;
double c3dref_regularizations[16] = {0.0, 1e-3, 1e-2, 1e-1, 5e-1};
}

static double *s_uOld = NULL;
static double *s_flux = NULL;

static long ncells_all()
{
    return (long)(g_gX[3] - g_gX[0] + 1) * (g_gY[3] - g_gY[0] + 1) * (g_gZ[3] - g_gZ[0] + 1);
}

extern "C" {

void c3dref_set_ladder(int n, const double *r)
{
    if (n < 1 || n > 16)
        return;
    c3dref_num_regularizations = n;
    for (int i = 0; i < n; i++)
        c3dref_regularizations[i] = r[i];
}

/* Runs the reference init() with input.deck taken from directory dir. */
int c3dref_init(const char *dir)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)))
        return -1;
    if (chdir(dir) != 0)
        return -2;
    init();
    if (chdir(cwd) != 0)
        return -3;
    long n = ncells_all() * g_numMoments;
    s_uOld = (double *)calloc(n, sizeof(double));
    s_flux = (double *)calloc(n, sizeof(double));
    return 0;
}

/* iv: nx ny nz (interior), nm, nm2, nq, solver(0 pn,1 mn), batched, useGaunt, useGauntSparse,
 *     pnUseKinetic, maxIter, cudaBatchSize
 * dv: dx dy dz maxDt theta tol tolGamma condHMax tFinal */
void c3dref_info(int *iv, double *dv)
{
    iv[0] = g_nx; iv[1] = g_ny; iv[2] = g_nz;
    iv[3] = g_numMoments; iv[4] = g_numMoments2; iv[5] = g_numQuadPoints;
    iv[6] = g_solver == SOLVER_MN ? 1 : 0;
    iv[7] = g_mnBatched; iv[8] = g_mnUseGaunt; iv[9] = g_mnUseGauntSparse;
    iv[10] = g_pnUseKineticFlux; iv[11] = g_mnMaxIter; iv[12] = g_cudaBatchSize;
    dv[0] = g_dx; dv[1] = g_dy; dv[2] = g_dz; dv[3] = g_maxDt; dv[4] = g_theta;
    dv[5] = g_mnTol; dv[6] = g_mnTolGamma; dv[7] = g_mnCondHMax; dv[8] = g_tFinal;
}

double *c3dref_ptr(int which)
{
    switch (which) {
    case 0: return g_u;
    case 1: return g_mnAlpha;
    case 2: return g_sigmaT;
    case 3: return g_sigmaS;
    case 4: return g_m;
    case 5: return g_m2;
    case 6: return g_w;
    case 7: return g_xi;
    case 8: return g_eta;
    case 9: return g_mu;
    case 10: return g_pnFluxOperatorXiPlus;
    case 11: return g_pnFluxOperatorXiMinus;
    case 12: return g_pnFluxOperatorEtaPlus;
    case 13: return g_pnFluxOperatorEtaMinus;
    case 14: return g_pnFluxOperatorMuPlus;
    case 15: return g_pnFluxOperatorMuMinus;
    case 16: return s_flux;
    case 17: return g_beta;
    }
    return NULL;
}

/* The reference's own time step. */
void c3dref_update(double dt) { update(dt); }

/* The reference's outputOptStats() and outputTimings() (src/output.cpp:116-222) run in
 * directory dir (with an output/ subdirectory); returns 0 on success. */
int c3dref_output_stats(const char *dir)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0)
        return -1;
    outputOptStats();
    outputTimings();
    return chdir(cwd) == 0 ? 0 : -2;
}

/* The reference's outputData(time) (src/output.cpp:19-110) run in directory dir, which must
 * hold an output/ subdirectory; returns 0 on success. */
int c3dref_output_data(double time, const char *dir)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0)
        return -1;
    bool saved = g_outputData;
    g_outputData = true;
    outputData(time);
    g_outputData = saved;
    return chdir(cwd) == 0 ? 0 : -2;
}

void c3dref_comm() { communicateBoundaries(); }
void c3dref_flux_kinetic(const double *alpha)
{
    solveFluxKinetic(g_u, s_flux, (double *)alpha, g_dx, g_dy, g_dz);
}
void c3dref_flux_moment() { solveFluxMoment(g_u, s_flux, g_dx, g_dy, g_dz); }

/* out: maxIterHist, maxGammaIter, iterMean, iterGammaMean, numDualSolves, hist[0..nreg-1] */
void c3dref_stats(double *out)
{
    out[0] = g_mnMaxIterHist;
    out[1] = g_mnMaxGammaIter;
    out[2] = g_mnIterMean;
    out[3] = g_mnIterGammaMean;
    out[4] = g_mnNumDualSolves;
    for (int i = 0; i < NUM_REGULARIZATIONS; i++)
        out[5 + i] = g_mnHistReg[i];
}

static void account(int iter, int iterGamma, double r)
{
    if (iter > g_mnMaxIterHist)
        g_mnMaxIterHist = iter;
    if (iterGamma > g_mnMaxGammaIter)
        g_mnMaxGammaIter = iterGamma;
    for (int k = 0; k < NUM_REGULARIZATIONS; k++)
        if (fabs(r - REGULARIZATIONS[k]) < 1e-10)
            g_mnHistReg[k]++;
    g_mnIterMean = (g_mnNumDualSolves * g_mnIterMean + iter) / (g_mnNumDualSolves + 1.0);
    g_mnIterGammaMean =
        (g_mnNumDualSolves * g_mnIterGammaMean + iterGamma) / (g_mnNumDualSolves + 1.0);
    g_mnNumDualSolves++;
}

static int reg_index_of(double r)
{
    for (int k = 0; k < NUM_REGULARIZATIONS; k++)
        if (fabs(r - REGULARIZATIONS[k]) < 1e-10)
            return k;
    return -1;
}

/* Closure over every cell (ghosts included) with per-cell records.
 * iters/iterGamma/regIdx are indexed by the cell's I3D index (may be NULL). */
static void closure_traced(int *iters, int *iterGamma, int *regIdx)
{
    if (g_mnBatched) {
        /* as solveBatchOptimization, src/update.cpp:105-178 */
        if (Optimization::c_stack1 == NULL) {
            Optimization::c_stack1 = new std::stack<Optimization *>;
            Optimization::c_stack2 = new std::stack<Optimization *>;
            Optimization::c_stack3 = new std::stack<Optimization *>;
        }
        for (int i = g_gX[0]; i <= g_gX[3]; i++)
            for (int j = g_gY[0]; j <= g_gY[3]; j++)
                for (int k = g_gZ[0]; k <= g_gZ[3]; k++)
                    Optimization::c_stack1->push(new Optimization(
                        i, j, k, g_numMoments, &g_u[IU(i, j, k, 0)], &g_mnAlpha[IU(i, j, k, 0)]));
        Optimization::opt(g_numMoments, g_numMoments2, g_numQuadPoints);
        while (!Optimization::c_stack3->empty()) {
            Optimization *o = Optimization::c_stack3->top();
            Optimization::c_stack3->pop();
            int i = o->c_i, j = o->c_j, k = o->c_k;
            memcpy(&g_mnAlpha[IU(i, j, k, 0)], o->c_alpha, g_numMoments * sizeof(double));
            memcpy(&g_u[IU(i, j, k, 0)], o->c_u, g_numMoments * sizeof(double));
            free(o->c_alpha);
            free(o->c_u);
            long c = I3D(i, j, k);
            if (iters) iters[c] = o->c_totalIter;
            if (iterGamma) iterGamma[c] = o->c_iterGamma;
            if (regIdx) regIdx[c] = o->c_regIndex;
            account(o->c_totalIter, o->c_iterGamma, o->c_r);
            delete o;
        }
    } else {
        /* as solveOptimization, src/update.cpp:43-99 */
        int nx = g_gX[3] - g_gX[0] + 1, ny = g_gY[3] - g_gY[0] + 1, nz = g_gZ[3] - g_gZ[0] + 1;
        long n = (long)nx * ny * nz;
        #pragma omp parallel for schedule(dynamic, 16)
        for (long c = 0; c < n; c++) {
            int i = (int)(c / ((long)ny * nz)), j = (int)((c / nz) % ny), k = (int)(c % nz);
            OPTIONS options;
            OUTS outs;
            options.maxIter = g_mnMaxIter;
            options.tolAbs = g_mnTol * g_mnTol;
            options.tolRel = g_mnTol;
            options.tolGamma = 1.1;
            options.condHMax = g_mnCondHMax;
            options.useGaunt = g_mnUseGaunt;
            options.useGauntSparse = g_mnUseGauntSparse;
            opt(g_numMoments, g_numMoments2, g_numQuadPoints, &g_u[IU(i, j, k, 0)],
                &g_mnAlpha[IU(i, j, k, 0)], options, g_w, g_m, g_m2, &outs);
            if (iters) iters[c] = outs.iter;
            if (iterGamma) iterGamma[c] = outs.iterGamma;
            if (regIdx) regIdx[c] = reg_index_of(outs.r);
            #pragma omp critical
            account(outs.iter, outs.iterGamma, outs.r);
        }
    }
}

/* Same expression as the file-static eulerStep, src/update.cpp:21-37. */
static void euler_step(double *u, double *flux, double dt)
{
    #pragma omp parallel for
    for (int i = g_gX[1]; i <= g_gX[2]; i++) {
        for (int j = g_gY[1]; j <= g_gY[2]; j++) {
            for (int k = g_gZ[1]; k <= g_gZ[2]; k++) {
                u[IU(i, j, k, 0)] =
                    u[IU(i, j, k, 0)] *
                        (1.0 + dt * g_sigmaS[I3D(i, j, k)] - dt * g_sigmaT[I3D(i, j, k)]) -
                    dt * flux[IU(i, j, k, 0)];
                for (int m = 1; m < g_numMoments; m++)
                    u[IU(i, j, k, m)] =
                        u[IU(i, j, k, m)] * (1.0 - dt * g_sigmaT[I3D(i, j, k)]) -
                        dt * flux[IU(i, j, k, m)];
            }
        }
    }
}

/* One SSP-RK2 step with the order of update(); records[stage*ncells + cell] per stage.
 * Returns the elapsed seconds of the closure (opt) part summed over both stages in
 * times[0], flux in times[1], euler+comm+copies in times[2] (times may be NULL). */
void c3dref_step_traced(double dt, int *iters, int *iterGamma, int *regIdx, double *times)
{
    long n = ncells_all();
    struct timespec t0, t1;
    double topt = 0, tflux = 0, trest = 0;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    #pragma omp parallel for
    for (int i = g_gX[1]; i <= g_gX[2]; i++)
        for (int j = g_gY[1]; j <= g_gY[2]; j++)
            for (int k = g_gZ[1]; k <= g_gZ[2]; k++)
                for (int m = 0; m < g_numMoments; m++)
                    s_uOld[IU(i, j, k, m)] = g_u[IU(i, j, k, m)];
    clock_gettime(CLOCK_MONOTONIC, &t1);
    trest += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);

    for (int s = 0; s < 2; s++) {
        clock_gettime(CLOCK_MONOTONIC, &t0);
        communicateBoundaries();
        clock_gettime(CLOCK_MONOTONIC, &t1);
        trest += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
        if (g_solver == SOLVER_MN) {
            clock_gettime(CLOCK_MONOTONIC, &t0);
            closure_traced(iters ? iters + s * n : NULL, iterGamma ? iterGamma + s * n : NULL,
                           regIdx ? regIdx + s * n : NULL);
            clock_gettime(CLOCK_MONOTONIC, &t1);
            topt += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
            clock_gettime(CLOCK_MONOTONIC, &t0);
            solveFluxKinetic(g_u, s_flux, g_mnAlpha, g_dx, g_dy, g_dz);
        } else {
            clock_gettime(CLOCK_MONOTONIC, &t0);
            if (g_pnUseKineticFlux == 0)
                solveFluxMoment(g_u, s_flux, g_dx, g_dy, g_dz);
            else
                solveFluxKinetic(g_u, s_flux, g_u, g_dx, g_dy, g_dz);
        }
        clock_gettime(CLOCK_MONOTONIC, &t1);
        tflux += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
        clock_gettime(CLOCK_MONOTONIC, &t0);
        euler_step(g_u, s_flux, dt);
        clock_gettime(CLOCK_MONOTONIC, &t1);
        trest += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    }
    g_numUpdates++;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    #pragma omp parallel for
    for (int i = g_gX[1]; i <= g_gX[2]; i++)
        for (int j = g_gY[1]; j <= g_gY[2]; j++)
            for (int k = g_gZ[1]; k <= g_gZ[2]; k++)
                for (int m = 0; m < g_numMoments; m++)
                    g_u[IU(i, j, k, m)] = 0.5 * (g_u[IU(i, j, k, m)] + s_uOld[IU(i, j, k, m)]);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    trest += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    if (times) {
        times[0] = topt;
        times[1] = tflux;
        times[2] = trest;
    }
}

/* Closure of the current grid only (one stage's opt part), with records. */
void c3dref_closure(int *iters, int *iterGamma, int *regIdx) { closure_traced(iters, iterGamma, regIdx); }

/* Standalone unbatched closures of ncells independent moment vectors with the
 * reference's opt() (src/opt/opt.cpp:330-355), in parallel. Needs a prior
 * c3dref_opt_init(nm, nm2). One moment count per process (opt() sizes its
 * thread-private scratch on first use, src/opt/opt.cpp:176-191). */
void c3dref_opt_init(int nm, int nm2)
{
    linesearch_init(nm);
    fobj_init(nm2);
}
void c3dref_opt_many(int nm, int nm2, int nq, long ncells, double *u, double *alpha, int maxIter,
                     double tol, double tolGamma, double condHMax, double *w, double *p, double *p2,
                     int *iters, int *iterGamma, double *r)
{
    #pragma omp parallel for schedule(dynamic, 8)
    for (long c = 0; c < ncells; c++) {
        OPTIONS options;
        OUTS outs;
        options.maxIter = maxIter;
        options.tolAbs = tol * tol;
        options.tolRel = tol;
        options.tolGamma = tolGamma;
        options.condHMax = condHMax;
        options.useGaunt = false;
        options.useGauntSparse = false;
        opt(nm, nm2, nq, u + c * nm, alpha + c * nm, options, w, p, p2, &outs);
        if (iters) iters[c] = outs.iter;
        if (iterGamma) iterGamma[c] = outs.iterGamma;
        if (r) r[c] = outs.r;
    }
}

/* The reference's batched closure (Optimization::opt, src/opt/optBatch.cpp:350-472)
 * applied to n given moment vectors, with the tables and MN options of the current
 * problem (c3dref_init first). Solved in place; iters may be NULL. */
void c3dref_opt_batched_vectors(long n, double *u, double *alpha, int *iters)
{
    if (Optimization::c_stack1 == NULL) {
        Optimization::c_stack1 = new std::stack<Optimization *>;
        Optimization::c_stack2 = new std::stack<Optimization *>;
        Optimization::c_stack3 = new std::stack<Optimization *>;
    }
    const int nm = g_numMoments;
    for (long c = 0; c < n; c++)
        Optimization::c_stack1->push(new Optimization((int)c, 0, 0, nm, u + c * nm, alpha + c * nm));
    Optimization::opt(g_numMoments, g_numMoments2, g_numQuadPoints);
    while (!Optimization::c_stack3->empty()) {
        Optimization *o = Optimization::c_stack3->top();
        Optimization::c_stack3->pop();
        long c = o->c_i;
        memcpy(alpha + c * nm, o->c_alpha, nm * sizeof(double));
        memcpy(u + c * nm, o->c_u, nm * sizeof(double));
        if (iters)
            iters[c] = o->c_totalIter;
        free(o->c_alpha);
        free(o->c_u);
        delete o;
    }
}

int c3dref_num_threads()
{
    int n = 1;
    #pragma omp parallel
    {
        #pragma omp single
        n = omp_get_num_threads();
    }
    return n;
}

} /* extern "C" */
