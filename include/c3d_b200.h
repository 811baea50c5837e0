/*
 * C ABI of the B200 M_N / P_N time step (libc3d_b200.so).
 *
 * Two groups of entry points:
 *
 * 1. Drop-in replacements for the reference's GPU offload layer,
 *    src/cuda/cuda_headers.h:10-21 of ckrisgarrett/C3D-2015. Same names,
 *    arguments and meaning (host pointers in and out, synchronous), so a build
 *    of the reference links against this library instead of its own
 *    src/cuda/*.cu files without source changes.
 *
 * 2. The device-resident step API that the C++ host (c3d-2015_b200/host) uses
 *    to run update() (src/update.cpp:185-275) on one GPU: state stays in HBM
 *    across stages and steps, the MPI halo exchange (src/comm.cpp) is an
 *    on-device periodic ghost fill, and the closure runs as work-list rounds in a
 *    device-side graph loop (or as persistent work-queue kernels). Every function
 *    returns a c3d_status; none aborts.
 *
 * Arrays use the reference's layouts: per-cell moment vectors with the moment
 * index fastest (IU, src/global.h:16), cells over the grid including two ghost
 * layers per face with k fastest (I3D, src/global.h:15); tables row-major
 * M[q*nm + m] (IM, src/global.h:18).
 */
#ifndef C3D_B200_H
#define C3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    C3D_OK = 0,
    C3D_ERR_INVALID = 1,     /* bad argument or unsupported size */
    C3D_ERR_CUDA = 2,        /* CUDA runtime error (see c3d_last_error) */
    C3D_ERR_NO_DEVICE = 3,   /* no CUDA device / extension unusable */
    C3D_ERR_CLOSURE = 4,     /* one or more cells failed (u0 <= 0 or ladder exhausted) */
    C3D_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    C3D_ERR_OOM = 6          /* device allocation failed */
} c3d_status;

/* Text of the last error on this thread. */
const char *c3d_last_error(void);

/* ------------------------------------------------------------------ 1. reference GPU entry points */

/* Kinetic flux on the whole grid; replaces src/cuda/cuda_headers.h:10-13.
 * nx,ny,nz include the ghost layers; alpha and flux are host arrays of
 * nx*ny*nz*nm doubles; flux is zero on ghost cells; theta = 2 as in the
 * reference's GPU path (src/cuda/cuda_flux_kinetic.cu:82). isPn selects the
 * linear P_N ansatz. */
void solveFluxKinetic_cuda(int nx, int ny, int nz, int nm, int nq, double dx, double dy, double dz,
                           double *alpha, double *flux, double *xi, double *eta, double *mu,
                           double *w, double *p, int isPn);

/* Batched Hessians H_b = sum_q w_q exp(alpha_b . m_q) m_q m_q^T for batchSize
 * multiplier vectors (host, batchSize*nm), written to hs (host, batchSize*nm*nm,
 * row-major, symmetric). Replaces src/cuda/cuda_headers.h:15-17. useGaunt = 1 forms
 * H from the extended moments over p2 and beta (src/cuda/cuda_solveH.cu:224-241):
 * dense beta with useGauntSparse = 0, the CSR table with 1. If the sizes or tables
 * were not set up by solveHInit_cuda, or the device fails, a message goes to stderr
 * and hs is filled with NaN (never left unwritten). */
void solveH_cuda(int nm, int nm2, int nq, int batchSize, double *alphas, double *hs, int useGaunt,
                 int useGauntSparse);

/* One-time set-up for solveH_cuda (tables to the device); replaces
 * src/cuda/cuda_headers.h:19-21. p2/beta/betaVal/betaColInd/betaRowPtr may be
 * NULL when useGaunt is 0; with useGaunt = 1, beta (dense, [nm*nm][nm2]) serves
 * useGauntSparse = 0 and the CSR arrays serve useGauntSparse = 1 (either may be NULL
 * if that mode is not used). nm <= 64, nm2 <= 232. */
void solveHInit_cuda(int nm, int nm2, int nq, int batchSize, double *w, double *p, double *p2,
                     double *beta, double *betaVal, int *betaColInd, int *betaRowPtr, int useGaunt);

/* ------------------------------------------------------------------ 2. device-resident step API */

typedef struct c3d_ctx c3d_ctx;

/* Problem parameters: the input.deck keys the time step reads
 * (src/init.cpp:364-381, :195, :252-258). */
typedef struct {
    int nx, ny, nz;            /* interior cells per axis (NX, NY, NZ) */
    int nm;                    /* moments (MOMENT_ORDER+1)^2 */
    int nq;                    /* quadrature points 2*QUAD_ORDER^2 */
    double dx, dy, dz;
    double theta;              /* THETA (slope limiter of the kinetic flux) */
    int solver;                /* 0: P_N, 1: M_N (SOLVER) */
    int pnUseKineticFlux;      /* PN_USE_KINETIC_FLUX */
    int mnBatched;             /* MN_BATCHED: 1 batched stop rules, 0 unbatched rules */
    int mnMaxIter;             /* MN_MAX_ITER */
    double mnTol;              /* MN_TOL */
    double mnTolGamma;         /* MN_TOL_GAMMA (batched rules; unbatched use 1.1) */
    double mnCondHMax;         /* MN_COND_H_MAX */
    int nreg;                  /* regularisation ladder (reference: 5 values) */
    double reg[16];
    size_t psiBytes;           /* budget for the materialised ansatz (0 = default, 32 GiB);
                                  the closure's ansatz hand-off needs nq * nall * 8 bytes */
    int mnReproject;           /* 1: after each grid closure set u = <m e^{alpha.m}> with u_0
                                  kept (the robustness note of the reference's readme.txt);
                                  deck key MN_REPROJECT; no counterpart in the reference code */
} c3d_params;

/* Closure counters accumulated on the device since the last reset (the
 * reference's g_mn* statistics, src/update.cpp:79-97). */
typedef struct {
    long long cells;           /* dual solves (all cells, ghosts included) */
    long long interiorCells;   /* unused (0) */
    long long totalIters;      /* sum of Newton iterations */
    int maxIter;               /* g_mnMaxIterHist */
    int maxIterGamma;          /* g_mnMaxGammaIter */
    long long totalIterGamma;
    long long failed;          /* cells with a non-zero status */
    long long trials;          /* line-search objective evaluations */
    long long clkRefill;       /* SM clocks summed over warps: work-queue refill and set-up */
    long long clkPass;         /* ... in passes over the staged basis (moments/Hessian/trials) */
    long long clkSerial;       /* ... in the per-cell Newton logic between passes */
    long long passes;          /* passes, summed over CTAs */
    long long regHist[16];     /* g_mnHistReg */
    long long iterHist[64];    /* cells per iteration count (last bin: >= 63) */
    long long clkNewton[8];    /* SM clocks of the work-list Newton kernel, builds with
                                  C3D_NEWTON_CLOCKS only: state load + H assembly, g/f/norms,
                                  Cholesky, condition estimate, direction solve, after_hessian in
                                  total, state store, line-search trial updates */
    long long hessBf16;        /* mixed precision (c3d_set_precision): Hessian visits with BF16 */
    long long hessTf32x3;      /*   ... with 3xTF32 split products */
    long long hessFp64;        /*   ... with FP64 moments */
    long long escalated;       /*   reduced-precision visits redone in FP64 */
    long long certified;       /* first visits ended by the convergence certificate */
    long long hostSyncs;       /* host waits inside the stages since creation (the face-ghost
                                  mirror check and host-driven rounds; 0 with graphs) */
} c3d_closure_stats;

/* Creates a context on the current CUDA device with the tables M[nq*nm],
 * w, xi, eta, mu [nq] (host arrays, copied). pnOps (6*nm*nm host array:
 * xi+, xi-, eta+, eta-, mu+, mu-, src/init.cpp:193-238) is needed for the P_N
 * moment flux and may be NULL otherwise. stream: a cudaStream_t or NULL for a
 * new non-blocking stream owned by the context. */
c3d_status c3d_create(const c3d_params *p, const double *M, const double *w, const double *xi,
                      const double *eta, const double *mu, const double *pnOps, void *stream,
                      c3d_ctx **out);
void c3d_destroy(c3d_ctx *ctx);

/* State transfer. where: 0 host arrays (synchronous copies), 1 device
 * pointers (stream-ordered). Any pointer may be NULL to skip it. u/alpha
 * hold nall*nm doubles, sigT/sigS nall doubles, nall = (nx+4)(ny+4)(nz+4). */
c3d_status c3d_set_state(c3d_ctx *ctx, const double *u, const double *alpha, const double *sigT,
                         const double *sigS, int where);
c3d_status c3d_get_state(c3d_ctx *ctx, double *u, double *alpha, int where);
c3d_status c3d_get_flux(c3d_ctx *ctx, double *flux, int where);

/* Device pointers of the resident state (valid for the context's lifetime). */
c3d_status c3d_device_state(c3d_ctx *ctx, double **u, double **alpha, double **flux);

/* Stages of update(); stream-ordered, no host synchronisation. */
c3d_status c3d_ghost_fill(c3d_ctx *ctx);                   /* communicateBoundaries */
c3d_status c3d_closure(c3d_ctx *ctx);                      /* Optimization::opt / opt on all cells */
c3d_status c3d_flux_kinetic(c3d_ctx *ctx, int alphaIsU);   /* solveFluxKinetic */
c3d_status c3d_flux_moment(c3d_ctx *ctx);                  /* solveFluxMoment */
c3d_status c3d_euler(c3d_ctx *ctx, double dt);             /* eulerStep */
/* One SSP-RK2 step, update(dt). */
c3d_status c3d_step(c3d_ctx *ctx, double dt);

/* One RK stage of update(dt) (src/update.cpp:204-274): stage 0 saves u, then ghost fill,
 * closure, flux and Euler stage; stage 1 does the same and ends with the RK average.
 * c3d_step is stage 0 then stage 1. The x-slab decomposition exchanges halos between them. */
c3d_status c3d_stage(c3d_ctx *ctx, int stage, double dt);

/* x-slab decomposition (replacing the MPI halo exchange, src/comm.cpp:170-276, with slabs
 * as in src/init.cpp:125-186): with on = 1 the ghost fill leaves the two x ghost planes on
 * each side to the caller, who fills them from the neighbouring slabs before each stage;
 * face-ghost mirroring is off for such a context. */
c3d_status c3d_set_x_halo_external(c3d_ctx *ctx, int on);

/* One RK stage of a slab context (c3d_set_x_halo_external on; M_N, work-list engine) in two
 * parts, so that the halo exchange overlaps the closure: part 0 = [stage 0: save u,] the y and
 * z ghost fill and the closure of the cells of the x-planes 2 .. nx+1, which need no halo;
 * part 1 = the closure of the four x-ghost planes, then the flux and Euler stage [stage 1: RK
 * average]. The caller copies u's first and last two interior x-planes out before part 0 (they
 * hold the stage's pre-closure moments, as the reference's exchange before the closure,
 * src/update.cpp:216-221), exchanges them while part 0 runs, and fills the x ghost planes
 * before part 1. Part 0 then part 1 equals c3d_stage bit for bit (cells are solved
 * independently). Launch by launch (no stage graph). */
c3d_status c3d_stage_part(c3d_ctx *ctx, int stage, double dt, int part);

/* Copies the x-planes i0 .. i0+count-1 (ghost indices 0 .. nx+3; each plane (ny+4)(nz+4) nm
 * doubles, contiguous) of u (field 0) or alpha (field 1) to (toBuf = 1) or from (toBuf = 0)
 * buf: a device buffer (where = 1, ordered on the context's stream) or a host buffer
 * (where = 0, synchronous). */
c3d_status c3d_copy_x_planes(c3d_ctx *ctx, int field, int i0, int count, void *buf, int toBuf,
                             int where);
/* Waits for the context's stream; reports device-side failures. */
c3d_status c3d_sync(c3d_ctx *ctx);

/* Per-cell records of the last closure (host arrays of nall ints; any may be
 * NULL): Newton iterations, gamma-only iterations, ladder index, status. */
c3d_status c3d_closure_records(c3d_ctx *ctx, int *iters, int *iterGamma, int *regIndex,
                               int *status);
/* Counters accumulated since creation or the last reset (synchronises). */
c3d_status c3d_closure_stats_get(c3d_ctx *ctx, c3d_closure_stats *st);
c3d_status c3d_closure_stats_reset(c3d_ctx *ctx);

/* Switches the closure to the Gaunt form of the Hessian (MN_USE_GAUNT_COEF true,
 * src/opt/fobj.cpp:58-95): extended moments over the harmonics of degree <= 2N, then
 * H_ij = sum_k beta_ijk mom_k in CSR order. M2[nq*nm2] and the CSR table
 * rowPtr[nm*nm+1], colInd[nnz], val[nnz] indexed by i*nm+j are host arrays (copied);
 * keep |beta| > 1e-13 for MN_USE_GAUNT_SPARSE true (src/init.cpp:318-336), all nonzeros
 * for the dense mode. NULL tables switch back to the direct form. N <= 7 (the persistent
 * engine forms H by direct quadrature for N = 7). */
c3d_status c3d_set_gaunt(c3d_ctx *ctx, int nm2, const double *M2, const int *rowPtr,
                         const int *colInd, const double *val);

/* The Gaunt tables built on the device (replaces the host loop of src/init.cpp:288-336).
 * beta_ij is the least-squares solution of M2 beta_ij = m_i .* m_j over the nq quadrature
 * points (one Householder QR of M2, then one solve per pair, pair = i*nm + j); the sparse
 * table keeps |beta| > threshold (1e-13 for MN_USE_GAUNT_SPARSE) in (pair, k) order, as
 * c3d_set_gaunt takes it. M2[nq*nm2] (q-major, the host layout of src/global.h IM2) and all
 * outputs are host arrays: beta[nm*nm*nm2] (dense, may be NULL), rowPtr[nm*nm+1] with
 * colInd/val of room for capacity entries (all three NULL: count only); *nnz receives the
 * entry count (C3D_ERR_INVALID when it exceeds capacity). Needs nm <= nm2 <= nq and
 * (nq + nm2) * 8 <= 200 KiB. Allocates device memory for the call and synchronises. The
 * sums run in another order than the host build's, so the values agree to rounding. */
c3d_status c3d_gaunt_build(int nm, int nm2, int nq, const double *M2, double threshold,
                           double *beta, int *rowPtr, long long capacity, int *colInd,
                           double *val, long long *nnz);

/* Closure engine: 0 (default) runs rounds over a device work list -- a pass kernel for
 * the quadrature sums of every listed cell, then a Newton kernel with one warp per cell,
 * re-listing cells that need another pass (the reference's Optimization::opt stacks,
 * src/opt/optBatch.cpp:350-472); 1 runs one persistent kernel whose warps pull cells
 * from a device counter. Both run the reference's per-cell algorithm; they differ in the
 * blocking of the Cholesky factorisation and of the triangular solves (engine 0: 8x8 tiles
 * with tensor-core trailing updates), so results agree to rounding. */
c3d_status c3d_set_engine(c3d_ctx *ctx, int engine);

/* Precision of the closure (work-list engine, Gaunt form; no counterpart in the reference).
 * mode 0 (default): FP64 throughout, the drop-in. mode 1: mixed -- an inexact Newton whose
 * Hessian's extended moments run on the tensor cores in BF16 (cell's last condition
 * estimate <= condBf16, default 1e4) or as 3xTF32 split products (<= condMixedMax, default
 * 1e7, and for a cell's first Hessian without a record), with FP32 accumulation and a
 * per-cell exponent shift of e^{alpha.m}; beyond, after mixedIterMax (default 8) iterations at
 * one regularisation level, and for the rest of the closure once a reduced-precision
 * factorisation fails or its moments are not finite, the cell's Hessian is FP64. The
 * gradient of the stopping test, the objective of the line search and the factorisation stay
 * FP64, so converged cells satisfy the same residual test as in mode 0; iteration counts
 * and multipliers differ within the tolerance. The steps that end a cell's iteration are
 * FP64 Newton steps: a reduced-precision visit whose gradient norm |g| lies in
 * (tol, polish * tol] (default polish 1e3; polish = 1 turns this off) is redone with FP64
 * moments, and the cell keeps them for the rest of the closure, so that the last steps
 * converge quadratically as in mode 0 and the moments track mode 0's closely. Values <= 0
 * select the defaults. For N <= 2 the Hessian moments stay FP64 (the tensor-core tile would
 * be mostly padding). */
c3d_status c3d_set_precision(c3d_ctx *ctx, int mode, double condBf16, double condMixedMax,
                             int mixedIterMax, double polish);

/* Convergence certificate of a cell's first Newton iteration (work-list engine, Gaunt form;
 * on by default; no counterpart in the reference). The first visit runs a probe pass --
 * exponents, e^{alpha.m}, the first-order moments and the extreme values e_min, e_max of
 * e^{alpha.m} over the quadrature -- instead of the Hessian pass. Since H >= e_min G with G the
 * quadrature's Gram matrix, |H^-1 g| and the condition estimate are bounded without H; a cell
 * whose gradient passes the stopping test with these bounds inside the test's thresholds (by
 * factors of 2 and 4) ends exactly as the full iteration would end it -- same multipliers,
 * moments, counts and status -- and is finalized without forming or factoring H; its gamma
 * record is then the bound. Other cells continue with the Hessian pass of the same
 * iteration. Off while the x-line statistics log (which records gamma) is enabled. */
c3d_status c3d_set_certificate(c3d_ctx *ctx, int on);

/* Flux autotuner (no counterpart in the reference): times the kinetic flux of the context's
 * current multipliers for each candidate direction chunk (the largest the psi budget allows
 * and the balanced splits into up to 3 more chunks) and z run length per CTA of the staged
 * kernel (64, and 32 where nz is a multiple of 32), then keeps the fastest for later calls.
 * The flux buffer is overwritten; u and alpha are not touched. Outputs may be NULL
 * (runLen 0: min(64, nz)). */
c3d_status c3d_autotune(c3d_ctx *ctx, int *qChunk, int *runLen, double *msPerCall);

/* The work-list closure as one CUDA graph (engine 0; on by default; no counterpart in the
 * reference, whose host loop hands the GPU one Hessian batch at a time,
 * src/opt/optBatch.cpp:350-472). Round 0, then a conditional WHILE node whose body runs two
 * rounds and sets its own condition on the device; each list's kernels sit in a SWITCH node
 * whose branch (launch size, or none for an empty list) a control kernel picks from the
 * list's device counter. A closure then needs no host round trip: c3d_closure enqueues one
 * graph launch on the context's stream (built on the first call and again whenever the
 * closure's parameters or buffers change). The round limit of c3d_set_limits is checked on
 * the device and reported by c3d_sync as C3D_ERR_TIMEOUT ("closure: round limit exceeded").
 * off: the host reads the list counts after every round (c3d_closure itself returns
 * C3D_ERR_TIMEOUT at the limit). Results are identical either way. */
c3d_status c3d_set_graphs(c3d_ctx *ctx, int on);

/* Ansatz hand-off from the closure to the kinetic flux (on by default; no counterpart in the
 * reference). A grid closure with the convergence certificate evaluates e^{alpha.m_q} of
 * every cell and direction in its probe pass; with this on, that pass also stores them as the
 * flux's ansatz psi (one buffer of nq * nall doubles, within the params' psiBytes budget),
 * face ghosts copy their images' values and the few cells whose multipliers change after the
 * probe are recomputed at the end of the closure, and the next c3d_flux_kinetic runs the
 * limited stencil and projection alone instead of forming psi again. The flux equals the
 * one formed from the closure's multipliers up to rounding (the probe forms
 * u_0 e^{alpha_scaled . m_q}). Any change of the multipliers in between (c3d_set_state,
 * c3d_copy_x_planes) drops the hand-off. */
c3d_status c3d_set_ansatz_handoff(c3d_ctx *ctx, int on);

/* Safety bounds of the closure (no counterpart in the reference, which loops until each cell
 * converges or aborts): at most maxRounds work-list rounds per closure (engine 0; default
 * 2^24), after which the closure returns C3D_ERR_TIMEOUT with the unfinished cells' state
 * left as it was, and at most passBudget Hessian and line-search passes per cell (default
 * 2^40), after which the cell ends with status 3 and c3d_sync reports C3D_ERR_CLOSURE, and at
 * most batch list entries per pass and Newton launch (default 2^20; the pass output buffer
 * holds that many; longer lists run in several launches, or carry over between the graph's
 * rounds). Values <= 0 restore the defaults. */
c3d_status c3d_set_limits(c3d_ctx *ctx, long long maxRounds, long long passBudget,
                          long long batch);

/* Face-ghost mirroring of the grid closure (engine 0; on by default). The reference solves
 * every cell, ghosts included (src/update.cpp:51-53, 119-123). A face ghost holds a copy of
 * its periodic image's moments, so when its multipliers (the warm start) also equal the
 * image's bit for bit -- checked on the device before each closure -- its solve would
 * reproduce the image's; the closure then solves the other cells and copies multipliers,
 * regularised moments and records to the face ghosts, whose records also enter the closure
 * statistics. Results and statistics are identical either way. No counterpart in the
 * reference. */
c3d_status c3d_set_ghost_mirroring(c3d_ctx *ctx, int on);

/* Standalone batched closure of n independent moment vectors (device
 * pointers u[n*nm], alpha[n*nm], solved in place; records may be NULL).
 * Uses the context's tables and MN options; grid state is untouched. */
c3d_status c3d_closure_vectors(c3d_ctx *ctx, long long n, double *u, double *alpha, int *iters,
                               int *iterGamma, int *regIndex, int *status);

/* Closure group: the standalone closures of several contexts (e.g. one per moment order, each
 * with its own tables and options) as ONE launch -- a CUDA graph whose parallel branches are
 * the contexts' closures, each with its work-list rounds in a device-side loop, so that the
 * orders' rounds share the GPU and no closure waits for the host. The contexts must be M_N
 * contexts on one stream (the one they were created with; the group launches there), with the
 * work-list engine and graphs on (the defaults) and timing off; a context appears once. The
 * graph is rebuilt when a context's options, a size or a buffer changes. Per context k:
 * n[k] vectors at u[k], alpha[k] (device, solved in place), records iters/iterGamma/regIndex/
 * status[k] as in c3d_closure_vectors (each array of pointers, or an entry of one, may be
 * NULL). Results are those of calling c3d_closure_vectors per context, bit for bit. Errors
 * (failed cells, round limit) are reported per context by c3d_sync. The group refers to its
 * contexts: destroy it before any of them. No counterpart in the reference, whose closure
 * works one batch of one order at a time. */
typedef struct c3d_group c3d_group;
c3d_status c3d_group_create(int count, c3d_ctx *const *ctx, c3d_group **out);
c3d_status c3d_group_closure_vectors(c3d_group *group, const long long *n, double *const *u,
                                     double *const *alpha, int *const *iters,
                                     int *const *iterGamma, int *const *regIndex,
                                     int *const *status);
/* One SSP-RK2 step of every context of the group (dt[k] for context k; each as c3d_step) as
 * ONE CUDA graph launch that runs the contexts' steps one after another (each step's kernels
 * fill the GPU; as parallel branches the same steps ran slower). Results are those of c3d_step
 * per context, bit for bit. Each context needs the work-list engine and graphs on, and timing, the x-line log
 * and re-projection off. The graph is rebuilt when a dt, an option or a buffer changes. */
c3d_status c3d_group_step(c3d_group *group, const double *dt);
void c3d_group_destroy(c3d_group *group);

/* Tables of src/init.cpp:509-548 (host arrays), so callers without GSL can
 * build M, w, xi, eta, mu identical to the host's. M2 may be NULL. */
void c3d_build_quadrature(int momentOrder, int quadOrder, double *w, double *xi, double *eta,
                          double *mu, double *M, double *M2);

/* Number of kernel launches issued by this context so far (synchronises the context's stream
 * to add those of device-side round loops). */
long long c3d_launch_count(c3d_ctx *ctx);

/* ------------------------------------------------------------------ allocation-free closure */

/* Closure options for the allocation-free entry point (the MN_* deck keys). */
typedef struct {
    int batched;        /* 1: batched stop rules (absolute tol, tolGamma); 0: unbatched */
    int maxIter;
    double tol;
    double tolGamma;
    double condHMax;
    int nreg;
    double reg[16];
} c3d_closure_opts;

/* Bytes of the per-GPU static scratch array used by c3d_closure_vectors_noalloc. */
#define C3D_NOALLOC_SCRATCH_BYTES 1202176

/* Standalone closure of n moment vectors that allocates no device memory. It has no
 * counterpart in the reference: it exists for callers that may not call cudaMalloc,
 * such as an application that serves this library device memory from its own
 * pre-reserved pool (where an extra cudaMalloc fails or breaks its accounting) or
 * a latency-critical caller that must avoid the implicit device synchronisation of
 * cudaMalloc/cudaFree. All arguments are the caller's device pointers (M[nq*nm],
 * w[nq], u and alpha [n*nm] solved in place; iters and status [n] may be NULL;
 * unsolved cells report status -1) except opts (host). The kernel's scratch (work
 * counter, failure and statistics counters, the chunked basis) lives in one static
 * __device__ array of C3D_NOALLOC_SCRATCH_BYTES held by every GPU that loads the
 * library until exit; sizes above nm = 64 or nq = 2048 are rejected with
 * C3D_ERR_INVALID. The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture. All
 * calls share the array: calls that overlap on the GPU race, so order them (one
 * stream). Stream-ordered; returns without synchronising. opts must hold maxIter >= 1
 * and positive finite tol, condHMax (and tolGamma under the batched rules). Status per
 * cell: 0 converged, 1 u0 <= 0, 2 ladder exhausted, -1 not reached because a bounded
 * device wait gave up; c3d_closure_vectors_noalloc_check reports the call's outcome. */
c3d_status c3d_closure_vectors_noalloc(int nm, int nq, const double *M, const double *w,
                                       long long n, double *u, double *alpha, int *iters,
                                       int *status, const c3d_closure_opts *opts, void *stream);

/* Outcome of the last c3d_closure_vectors_noalloc call on the current device, read out of
 * the same static array (allocates nothing): waits for stream, then returns
 * C3D_ERR_TIMEOUT if a bounded device wait gave up (the kernel stopped early; unsolved
 * cells keep their inputs), C3D_ERR_CLOSURE if cells failed (their number in *failed, which
 * may be NULL), else C3D_OK, and clears both records. Call it after each call whose
 * outcome matters, before the next call. */
c3d_status c3d_closure_vectors_noalloc_check(void *stream, long long *failed);

/* Event timing on the context's stream around every grid closure (kind 0), kinetic flux
 * (1), ghost fill (2) and Euler stage (3) (off by default). c3d_timing_get returns the
 * summed milliseconds ms[0] closure, ms[1] kinetic flux and their counts since enabling;
 * c3d_timing_events copies up to maxEvents (kind, ms) pairs in launch order and returns
 * their number (-1 on error). They feed the reference's per-update timers
 * (src/update.cpp:217-262). */
c3d_status c3d_timing_enable(c3d_ctx *ctx, int on);
c3d_status c3d_timing_get(c3d_ctx *ctx, double *ms, long long *count);
int c3d_timing_events(c3d_ctx *ctx, int *kinds, double *ms, int maxEvents);

/* Per-cell final gamma and |g| of the last closure (host arrays of nall doubles; either may
 * be NULL). */
c3d_status c3d_closure_records_fp(c3d_ctx *ctx, double *gamma, double *normG);

/* x-line statistics of the reference (g_optStats, src/update.cpp:66-75,147-155): after
 * each grid closure, for the interior cells (i, (ny+3)/2, (nz+3)/2) the records
 * {r, iter, iterGamma, gamma, normG} (5 doubles per cell; gamma holds iterGamma under the
 * batched rules, as the reference's batched path stores it) are appended to a device log of
 * up to maxClosures closures (0 disables). c3d_line_stats_get copies count*nx*5 doubles. */
c3d_status c3d_line_stats_enable(c3d_ctx *ctx, int maxClosures);
c3d_status c3d_line_stats_get(c3d_ctx *ctx, double *out, int *count);

#ifdef __cplusplus
}
#endif
#endif
