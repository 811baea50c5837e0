/*
 * C ABI of the host solver of libc3d_b200.so: the reference's init() / update() / time loop
 * / output (src/init.cpp:344-576, src/update.cpp:185-275, src/main.cpp:57-97,
 * src/output.cpp:19-110) driven from an input.deck, with every stage on the GPU through the
 * device API of c3d_b200.h. All functions return C3D_OK or an error code; none aborts.
 */
#ifndef C3D_SOLVER_H
#define C3D_SOLVER_H

#include "c3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct c3d_solver c3d_solver;

/* Reads a deck and runs init() (tables, IC, multipliers, dt) on the current device;
 * stream: a cudaStream_t or NULL. Replaces init() of src/init.cpp:344-576. */
c3d_status c3d_solver_create(const char *deckPath, void *stream, c3d_solver **out);

/* Host half of init() only (no GPU): tables, initial state, cross sections, multipliers,
 * dt_max. errbuf receives the first missing or invalid key. */
c3d_status c3d_solver_prepare(const char *deckPath, c3d_solver **out, char *errbuf, int errlen);

void c3d_solver_destroy(c3d_solver *s);

/* update(dt) of src/update.cpp:185-275 (no host synchronisation). */
c3d_status c3d_solver_update(c3d_solver *s, double dt);

/* The time loop of src/main.cpp:57-76 (or NSTEPS steps), with outputData at t = 0 and at
 * every output time when the deck says OUTPUT_DATA true. */
c3d_status c3d_solver_run(c3d_solver *s, int *steps);

/* Device state -> host mirrors (u, alpha), and back (u, alpha, sigma_t, sigma_s). */
c3d_status c3d_solver_pull(c3d_solver *s);
c3d_status c3d_solver_push(c3d_solver *s);

/* The solver's device context (NULL for c3d_solver_prepare). */
c3d_ctx *c3d_solver_context(c3d_solver *s);

/* iv: nx ny nz nm nq solver(0 P_N / 1 M_N) nsteps nreg; dv: dx dy dz maxDt theta tFinal. */
void c3d_solver_info(c3d_solver *s, int *iv, double *dv);

/* Host mirrors (valid after c3d_solver_pull): 0 u, 1 alpha, 2 sigT, 3 sigS, 4 M, 5 w, 6 xi,
 * 7 eta, 8 mu, 9 P_N operators. */
double *c3d_solver_host_array(c3d_solver *s, int which);

/* outputData(time) of src/output.cpp:19-110 into directory dir: out_<time>.master (text)
 * and out_<time>_0.pn (int64 nx ny nz, the interior moments, the closure statistics), in
 * the reference's formats. */
c3d_status c3d_solver_output_data(c3d_solver *s, double time, const char *dir);

/* outputTimings / outputOptStats of src/output.cpp:116-222 into directory dir:
 * times.master + times_0.dat (8 seconds per update: per RK stage ghost fill, closure, flux,
 * Euler) and stats_0.dat (per closure the x-line records {r, iter, iterGamma, gamma, normG});
 * recorded during the run when the deck sets OUTPUT_TIMINGS / OUTPUT_OPT_STATS true. */
c3d_status c3d_solver_output_timings(c3d_solver *s, const char *dir);
c3d_status c3d_solver_output_opt_stats(c3d_solver *s, const char *dir);

/* Checkpoint of (u, alpha) of all cells and the time ("C3DCKPT1", int64 nx ny nz nm,
 * double time, u, alpha); restore loads one written for the same grid and moment count.
 * No counterpart in the reference. */
c3d_status c3d_solver_checkpoint(c3d_solver *s, double time, const char *path);
c3d_status c3d_solver_restore(c3d_solver *s, const char *path, double *time);

#ifdef __cplusplus
}
#endif
#endif
