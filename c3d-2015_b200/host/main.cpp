// c3d_solver: the input.deck driver (the reference's main(), src/main.cpp:30-113)
// with every stage of the time step on the GPU.
//   usage: c3d_solver [deck path, default ./input.deck]
#include "../../include/c3d_b200.h"

#include <chrono>
#include <cstdio>

extern "C" {
typedef struct c3d_solver c3d_solver;
c3d_status c3d_solver_create(const char *deckPath, void *stream, c3d_solver **out);
void c3d_solver_destroy(c3d_solver *s);
c3d_status c3d_solver_run(c3d_solver *s, int *steps);
c3d_ctx *c3d_solver_context(c3d_solver *s);
}

int main(int argc, char **argv)
{
    const char *deck = argc > 1 ? argv[1] : "input.deck";
    c3d_solver *s = nullptr;
    c3d_status st = c3d_solver_create(deck, nullptr, &s);
    if (st != C3D_OK) {
        fprintf(stderr, "init failed (%d): %s\n", (int)st, c3d_last_error());
        return 1;
    }
    printf("Init done.\n");
    auto t0 = std::chrono::steady_clock::now();
    int steps = 0;
    st = c3d_solver_run(s, &steps);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st != C3D_OK) {
        fprintf(stderr, "run failed (%d): %s\n", (int)st, c3d_last_error());
        c3d_solver_destroy(s);
        return 2;
    }
    printf("Time taken: %.3lfs (%d steps)\n", secs, steps);
    c3d_closure_stats cs;
    if (c3d_closure_stats_get(c3d_solver_context(s), &cs) == C3D_OK && cs.cells > 0) {
        printf("g_mnMaxIterHist = %d\n", cs.maxIter);
        printf("g_mnMaxGammaIter = %d\n", cs.maxIterGamma);
        printf("g_mnIterMean = %f\n", (double)cs.totalIters / (double)cs.cells);
        printf("g_mnIterGammaMean = %f\n", (double)cs.totalIterGamma / (double)cs.cells);
        printf("g_mnNumDualSolves = %lld\n", cs.cells);
        for (int i = 0; i < 16 && (cs.regHist[i] || i < 5); ++i)
            printf("  g_mnHistReg[%d] = %lld\n", i, cs.regHist[i]);
    }
    c3d_solver_destroy(s);
    return 0;
}
