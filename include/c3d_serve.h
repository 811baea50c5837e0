/*
 * Serving loop of libc3d_b200.so (no counterpart in the reference, which runs one problem per
 * process): independent transport problems, each given as input.deck text, are admitted
 * against a device-memory budget and keep their state on the device from submission to
 * completion. One scheduling thread advances every admitted problem by one time step per pass,
 * the M_N problems together in ONE launch: a CUDA graph whose parallel branches are their RK
 * steps (c3d_group_step), rebuilt when the set of problems changes. While the GPU runs a pass
 * the thread admits the requests that arrived (in arrival order, while the active problems'
 * estimated footprints leave room), which join the next pass; problems that took their last
 * step leave after it. Each problem's result is what c3d_solver_run gives for it alone, bit for
 * bit: problems share launches but no data. Output keys of the decks are ignored (results come
 * back through c3d_server_wait).
 */
#ifndef C3D_SERVE_H
#define C3D_SERVE_H

#include "c3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct c3d_server c3d_server;

/* workers: problems active at once at most (slots of the shared pass); hbmBudgetBytes: device
 * memory the admitted problems' estimated footprints may add up to (0: no limit). Uses the
 * current CUDA device. */
c3d_status c3d_server_create(int workers, size_t hbmBudgetBytes, c3d_server **out);

/* Queues a problem (input.deck text, the reference's keys; NSTEPS or TFINAL bound its run);
 * returns at once with its id. A deck that does not parse is rejected here. */
c3d_status c3d_server_submit(c3d_server *s, const char *deckText, long long *id);

/* Waits for request id. dims (may be NULL) receives nx, ny, nz, nm; u (may be NULL) the final
 * interior moments (nx*ny*nz*nm doubles, (i, j, k, m) with m fastest) if capacity allows;
 * latency the seconds from submission to completion; steps the steps taken. Returns the
 * problem's own status (e.g. C3D_ERR_CLOSURE when a cell's regularisation ladder ran out). */
c3d_status c3d_server_wait(c3d_server *s, long long id, int *dims, double *u, long long capacity,
                           double *latency, int *steps);

/* Peak estimated device bytes and peak number of problems active at once so far. */
c3d_status c3d_server_stats(c3d_server *s, long long *peakBytes, int *peakActive);

/* Where the scheduling thread's time went so far: seconds[0] admitting problems (host set-up
 * of tables, initial state and device context), [1] creating groups and launching passes
 * (graph captures included), [2] waiting for passes to finish on the GPU, [3] finishing problems
 * (results to the host, contexts freed); counts[0] passes, [1] group builds. Either pointer may
 * be NULL. */
c3d_status c3d_server_timing(c3d_server *s, double *seconds, long long *counts);

/* Estimated device footprint of a deck's problem in bytes (the admission test's figure). */
c3d_status c3d_server_estimate(const char *deckText, long long *bytes);

/* Waits for every queued problem, then frees the server. */
void c3d_server_destroy(c3d_server *s);

#ifdef __cplusplus
}
#endif
#endif
