/*
 * Forced-include header for compiling the reference CPU path as a test
 * oracle. It declares the same interface as the reference's src/opt/opt.h
 * (OPTIONS / OUTS structs, the opt/fobj/linesearch prototypes, the Gaunt
 * globals and class Optimization, src/opt/opt.h:14-91) under the same include
 * guard, so the reference's own header is skipped. The one difference: the
 * regularisation ladder (src/opt/opt.h:37-38, a compile-time table of 5
 * values) becomes a runtime table, so decks may use other ladders, such as the
 * 6-level {0, 1e-8, 1e-6, 1e-4, 1e-2, 1e-1}. Default values are the reference's.
 * No reference source file is modified.
 */
#ifndef __OPT_H
#define __OPT_H

#include <stack>

struct OPTIONS
{
    int maxIter;
    double tolAbs;
    double tolRel;
    double tolGamma;
    double condHMax;
    bool useGaunt;
    bool useGauntSparse;
};

struct OUTS
{
    double r;
    int iter;
    int iterGamma;
    double gamma;
    double normG;
};

extern "C" int c3dref_num_regularizations;
extern "C" double c3dref_regularizations[16];
#define NUM_REGULARIZATIONS c3dref_num_regularizations
#define REGULARIZATIONS c3dref_regularizations

void opt(int nm, int nm2, int nq, double *u, double *alpha, OPTIONS options, double *w, double *p,
         double *p2, OUTS *outs);
void fobj_init(int nm2);
double fobjMn(int nm, int nm2, int nq, double *alpha, double *u, double *w, double *p, double *p2,
              double *g, double *h, bool useGaunt, bool useGauntSparse);
double fobjMnUseH(int nm, double *alpha, double *u, double *p, double *g, double *h);
void solveHMn(int nm, int nm2, int nq, double *alpha, double *w, double *p, double *p2, double *h,
              bool useGaunt, bool useGauntSparse);
void linesearch_init(int nm);
double linesearch(int n1, int n2, int nq, double *alpha, double *d, double f, double *g, double *u,
                  double *w, double *p);

extern double *g_beta;
extern double *g_betaVal;
extern int *g_betaColInd;
extern int *g_betaRowPtr;

class Optimization
{
public:
    Optimization(int i, int j, int k, int n, double *u, double *alpha);
    void preProcess(int n);
    void postProcess(int n);

    static void opt(int nm, int nm2, int nq);

    static std::stack<Optimization *> *c_stack1;
    static std::stack<Optimization *> *c_stack2;
    static std::stack<Optimization *> *c_stack3;

    double *c_u;
    double *c_alpha;
    double *c_h;
    double *c_alpha0;
    double *c_uOriginal;
    double c_t;
    double c_r;
    double c_err;
    int c_iter;
    int c_iterGamma;
    int c_totalIter;
    int c_i, c_j, c_k;
    int c_regIndex;
    double c_u0;
    bool c_preProcessed;
};

#endif
