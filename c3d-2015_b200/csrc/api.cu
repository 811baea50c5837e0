// C ABI of libc3d_b200.so (declarations and contracts in include/c3d_b200.h).
#include "../../include/c3d_b200.h"
#include "c3d_common.cuh"
#include "rounds_launch.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace c3d {
struct ClosureLaunch {
    const ClosureParams *P;
    const double *chunks;
    long long ncells;
    unsigned long long *counter;
    double *u, *alpha;
    int *iters, *iterGamma, *regIdx, *status;
    unsigned long long *failCount;
    unsigned long long *stats;
    double *gamma, *normG; // per-cell final gamma and |g| (may be null)
    int *errorFlag;
    int numSMs;
    cudaStream_t stream;
};
cudaError_t launch_closure_fp64(const ClosureLaunch &L);
int closure_fp64_nmp(int nm);
struct GauntTables {
    const double *chunks;
    const int *row, *col;
    const double *val;
};
cudaError_t launch_closure_gaunt(const ClosureLaunch &L, const GauntTables &G);
bool closure_gaunt_supported(int nm);
int closure_gaunt_nm2p(int nm2);
cudaError_t launch_hessian_batch(int nm, int nchunks, const double *chunks, const double *alphas,
                                 long long n, double *hs, int *errorFlag, cudaStream_t st);
size_t gaunt_batch_smem(int nm, int nm2p);
cudaError_t launch_gaunt_batch(int nm, int nm2, int nm2p, int nchunks, const double *chunks,
                               const double *alphas, long long n, const double *betaT,
                               const int *rowPtr, const int *colInd, const double *val,
                               int sparse, double *hs, int *errorFlag, cudaStream_t st);
cudaError_t launch_ghost_fill(const GridDims &g, double *u, int numSMs, cudaStream_t st,
                              bool skipX = false);
cudaError_t launch_euler(const GridDims &g, double *u, const double *flux, const double *sigT,
                         const double *sigS, double dt, int numSMs, cudaStream_t st);
cudaError_t launch_rk(const GridDims &g, double *u, double *uOld, int mode, int numSMs,
                      cudaStream_t st);
cudaError_t launch_kinetic_flux(const GridDims &g, const double *alpha, const double *mfA,
                                const double *mfP, const double *xi, const double *eta, int nq,
                                int qChunk, int runLen, double theta, int isPn, double *psi,
                                bool psiReady, double *flux, int *errorFlag,
                                const int *wrapFlag, cudaStream_t st);
bool kinetic_staged_used(const GridDims &g, int runLen);
cudaError_t launch_psi_handoff(const GridDims &g, int nq, const double *M, const double *alpha,
                               bool faceCopy, const int *refresh, const unsigned int *refreshCount,
                               double *psi, int *psiValid, int numSMs, cudaStream_t st);
size_t flux_frag_doubles(int nm, int nq, int which);
cudaError_t launch_reproject(const GridDims &g, double *u, double *alpha, const double *mfA,
                             const double *mfP, int nq, int *errorFlag, cudaStream_t st);
cudaError_t launch_ghost_fill_int(const GridDims &g, int *a, int numSMs, cudaStream_t st);
cudaError_t launch_ghost_fill_1(const GridDims &g, double *a, int numSMs, cudaStream_t st);
cudaError_t launch_line_log(const GridDims &g, const ClosureParams &P, const int *iters,
                            const int *iterGamma, const int *regIdx, const double *gamma,
                            const double *normG, double *out, cudaStream_t st);
cudaError_t launch_ghost_stats(const GridDims &g, const int *iters, const int *iterGamma,
                               const int *regIdx, const int *status, unsigned long long *stats,
                               int numSMs, cudaStream_t st);
cudaError_t launch_ghost_mirror_check(const GridDims &g, const double *a, int *flag, int numSMs,
                                      cudaStream_t st);
void flux_frags(int nm, int nq, const double *M, const double *w, const double *xi,
                const double *eta, const double *mu, double rdx, double rdy, double rdz,
                double *mfA, double *mfP);
cudaError_t launch_moment_flux(const GridDims &g, const double *u, const double *ops, double dx,
                               double dy, double dz, double *flux, cudaStream_t st);
} // namespace c3d


using namespace c3d;

static thread_local std::string g_lastError;

namespace c3d {
void set_last_error(const std::string &msg) { g_lastError = msg; }
} // namespace c3d

static c3d_status fail(c3d_status s, const std::string &msg)
{
    g_lastError = msg;
    return s;
}

#define C3D_CUDA(call)                                                                             \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? C3D_ERR_OOM : C3D_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

// Chunk-blocked, transposed basis for the closure's bulk copies:
// chunk k holds rows i < NMP of M^T restricted to directions [k*QC, k*QC+QC)
// with row stride QCP, then one row of weights; zero padding elsewhere.
static std::vector<double> build_chunks(int nm, int nq, const double *M, const double *w)
{
    int nmp = closure_fp64_nmp(nm);
    int nch = ceil_div(nq, QC);
    size_t chunk = (size_t)(nmp + 1) * QCP;
    std::vector<double> out((size_t)nch * chunk, 0.0);
    for (int k = 0; k < nch; ++k) {
        double *c = out.data() + k * chunk;
        for (int qq = 0; qq < QC; ++qq) {
            int q = k * QC + qq;
            if (q >= nq)
                break;
            for (int i = 0; i < nm; ++i)
                c[i * QCP + qq] = M[(size_t)q * nm + i];
            c[nmp * QCP + qq] = w[q];
        }
    }
    return out;
}

struct c3d_ctx {
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    GridDims g{};
    int nq = 0;
    double dx = 0, dy = 0, dz = 0, theta = 2.0;
    int solver = 1, pnKinetic = 0;
    ClosureParams cp{};
    size_t psiBytes = 0;
    int qChunk = 0;
    int runLen = 0;     // z run per CTA of the staged kinetic kernel (0: min(64, nz))
    size_t psiAlloc = 0; // bytes of the psi buffer
    // ansatz hand-off: the last grid closure left psi of every direction for its multipliers
    // (the probe pass wrote it; face ghosts and cells changed after the probe were refreshed),
    // so the next kinetic flux runs the stencil alone. Cleared by the flux and by any change
    // of the multipliers.
    bool psiReady = false;
    bool psiHandoffPending = false;     // the closure's probe wrote psi; completed in closure_grid
    bool handoff = true;                // c3d_set_ansatz_handoff
    int *psiRefresh = nullptr;          // cells whose psi is rewritten after the closure
    unsigned int *psiRefreshCount = nullptr;
    // device flag: psi holds the ansatz of every cell but the face ghosts for the current
    // multipliers (set by a closure's hand-off, cleared by whatever may break that)
    int *psiValid = nullptr;
    long long launches = 0;
    long long hostSyncs = 0; // host waits inside the stages (c3d_closure_stats.hostSyncs)
    // device buffers
    double *u = nullptr, *alpha = nullptr, *uOld = nullptr, *flux = nullptr;
    double *sigT = nullptr, *sigS = nullptr;
    double *M = nullptr, *w = nullptr, *xi = nullptr, *eta = nullptr, *mu = nullptr;
    double *mfA = nullptr, *mfP = nullptr; // basis in the flux kernels' fragment order
    bool reproject = false;                // MN_REPROJECT
    bool xHaloExternal = false;            // x ghosts filled by the caller (x-slab decomposition)
    double *cellGamma = nullptr, *cellErr = nullptr; // per-cell final gamma and |g|
    // x-line statistics log (the reference's g_optStats, src/update.cpp:66-75,147-155)
    double *lineLog = nullptr;
    int lineCap = 0, lineCount = 0;
    double *chunks = nullptr, *pnops = nullptr, *psi = nullptr;
    int *iters = nullptr, *iterGamma = nullptr, *regIdx = nullptr, *status = nullptr;
    unsigned long long *counter = nullptr, *failCount = nullptr, *stats = nullptr;
    int *errorFlag = nullptr;
    double m0 = 0.0; // M[0][0]
    int engine = 0;  // 0: work-list rounds, 1: persistent kernels
    long long maxRounds = 1LL << 24; // work-list rounds per closure before C3D_ERR_TIMEOUT
    long long maxBatch = 1LL << 20;  // list entries per pass/Newton launch
    void *roundsGraph = nullptr;     // the closure as one CUDA graph (c3d_set_graphs)
    bool graphs = true;
    // each RK stage as one CUDA graph (c3d_set_graphs): instantiated per stage and rebuilt
    // when its key (dt, options, buffers) changes; sc: the streams its capture uses
    struct StageGraph {
        std::vector<unsigned char> key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
        unsigned long long used = 0;
    } sg[8]; // the last few stage configurations (both stages, e.g. of two precisions)
    unsigned long long sgTick = 0;
    cudaStream_t sc[4] = {nullptr, nullptr, nullptr, nullptr};
    unsigned long long *launchDev = nullptr; // kernels launched by device-side round loops
    // work-list buffers (sized on first use)
    void *rState = nullptr;
    int *rListA = nullptr, *rListB = nullptr;
    unsigned int *rCounts = nullptr, *rHostCount = nullptr;
    double *rBuf = nullptr;
    long long rCells = 0, rBatch = 0, rBatchUse = 0; // rBatch: buffer capacity, rBatchUse: in use
    size_t rBufPer = 0;
    int nm2 = 0;
    // Gaunt form of the Hessian (c3d_set_gaunt)
    bool gaunt = false;
    double *gChunks = nullptr, *gVal = nullptr;
    int *gRow = nullptr, *gCol = nullptr;
    // face-ghost mirroring: when every face ghost's multipliers equal its periodic image's
    // (bitwise), the closure solves only the other cells (cellMap) and copies the face ghosts
    int *cellMap = nullptr;
    // x-slab split of the closure (c3d_stage_part): cells of the x-planes 2 .. nx+1, and of the
    // four x-ghost planes
    int *xSplit[2] = {nullptr, nullptr};
    long long xSplitCount[2] = {0, 0};
    long long cellMapCount = 0;
    int *mirrorFlag = nullptr;     // device
    int *mirrorHost = nullptr;     // pinned
    bool mirror = true;
    long long mirroredClosures = 0;
    double *gChunksC = nullptr;    // work-list engine: chunks of nm2 M2 rows + the weight row
    GauntTerm *gStream = nullptr;  // tiled assembly streams of the work-list engine
    int gStreamLen = 0;
    // mixed-precision closure (c3d_set_precision): staged chunks of the mixed pass -- FP64
    // rows (the nm rows of M2 of degree <= N, then the weights) and the A operand in BF16 and
    // in TF32 hi + lo -- and the per-cell condition records that seed each cell's precision
    double *mixF64 = nullptr;
    unsigned char *mixA[2] = {nullptr, nullptr};
    float *cellCond = nullptr;
    // convergence certificate of first visits (c3d_set_certificate): the Gaunt terms of H's
    // column 0 (g0n per row) for the FP64 gradient, and whether they lie in the probe's rows
    GauntTerm *g0 = nullptr;
    int g0n = 0;
    bool g0Valid = false;
    bool certificate = true;
    // optional event timing of the closure and flux launches (kind 0 closure, 1 flux)
    bool timing = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> events;
};

static void timing_begin(c3d_ctx *c, cudaEvent_t *a)
{
    if (!c->timing)
        return;
    cudaEventCreate(a);
    cudaEventRecord(*a, c->stream);
}
static void timing_end(c3d_ctx *c, int kind, cudaEvent_t a)
{
    if (!c->timing)
        return;
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, c->stream);
    c->events.push_back({kind, {a, b}});
}
static void timing_clear(c3d_ctx *c)
{
    for (auto &e : c->events) {
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    c->events.clear();
}

static void free_ctx(c3d_ctx *c)
{
    if (c->stream)
        cudaStreamSynchronize(c->stream); // graphs and buffers may still be in use
    void *ptrs[] = {c->u,     c->alpha,  c->uOld,     c->flux,    c->sigT,   c->sigS,
                    c->M,     c->w,      c->xi,       c->eta,     c->mu,     c->chunks,
                    c->pnops, c->psi,    c->iters,    c->iterGamma, c->regIdx, c->status,
                    c->counter, c->failCount, c->stats, c->errorFlag, c->gChunks, c->gVal,
                    c->gRow, c->gCol, c->gStream, c->rState, c->rListA, c->rListB,
                    c->rCounts, c->rBuf, c->mfA, c->mfP, c->cellMap, c->mirrorFlag,
                    c->gChunksC, c->cellGamma, c->cellErr, c->lineLog, c->mixF64,
                    c->mixA[0], c->mixA[1], c->cellCond, c->g0, c->psiRefresh,
                    c->psiRefreshCount, c->xSplit[0], c->xSplit[1], c->psiValid};
    for (void *p : ptrs)
        if (p)
            cudaFree(p);
    if (c->launchDev)
        cudaFree(c->launchDev);
    if (c->roundsGraph)
        rounds_graph_free(c->roundsGraph);
    for (auto &g : c->sg)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    for (cudaStream_t s : c->sc)
        if (s)
            cudaStreamDestroy(s);
    timing_clear(c);
    if (c->rHostCount)
        cudaFreeHost(c->rHostCount);
    if (c->mirrorHost)
        cudaFreeHost(c->mirrorHost);
    if (c->ownStream && c->stream)
        cudaStreamDestroy(c->stream);
    delete c;
}

// psi no longer matches the multipliers (or may not): the next hand-off closure writes all of it.
static void psi_invalidate(c3d_ctx *c)
{
    if (c->psiValid)
        cudaMemsetAsync(c->psiValid, 0, sizeof(int), c->stream);
}

extern "C" {

const char *c3d_last_error(void) { return g_lastError.c_str(); }

c3d_status c3d_create(const c3d_params *p, const double *M, const double *w, const double *xi,
                      const double *eta, const double *mu, const double *pnOps, void *stream,
                      c3d_ctx **out)
{
    if (!p || !M || !w || !xi || !eta || !mu || !out)
        return fail(C3D_ERR_INVALID, "c3d_create: null argument");
    if (p->nx < 1 || p->ny < 1 || p->nz < 1)
        return fail(C3D_ERR_INVALID, "c3d_create: grid sizes must be positive");
    if (p->nm < 1 || p->nm > 64)
        return fail(C3D_ERR_INVALID, "c3d_create: nm must be in [1, 64] (moment order <= 7)");
    int sq = (int)std::lround(std::sqrt((double)p->nm));
    if (sq * sq != p->nm)
        return fail(C3D_ERR_INVALID, "c3d_create: nm must be (N+1)^2");
    if (p->nq < 1)
        return fail(C3D_ERR_INVALID, "c3d_create: nq must be positive");
    if (p->nreg < 1 || p->nreg > MAX_REG)
        return fail(C3D_ERR_INVALID, "c3d_create: ladder length must be in [1, 16]");
    if (p->solver == 0 && !p->pnUseKineticFlux && !pnOps)
        return fail(C3D_ERR_INVALID, "c3d_create: P_N moment flux needs the six operators");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(C3D_ERR_NO_DEVICE, "c3d_create: no CUDA device");

    c3d_ctx *c = new c3d_ctx();
    cudaGetDevice(&c->device);
    cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, c->device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return fail(C3D_ERR_CUDA, "c3d_create: stream creation failed");
        }
        c->ownStream = true;
    }
    c->g = GridDims{p->nx, p->ny, p->nz, p->nm};
    c->nq = p->nq;
    c->dx = p->dx;
    c->dy = p->dy;
    c->dz = p->dz;
    c->theta = p->theta;
    c->solver = p->solver;
    c->pnKinetic = p->pnUseKineticFlux;
    ClosureParams &cp = c->cp;
    cp.nm = p->nm;
    cp.nq = p->nq;
    cp.nchunks = ceil_div(p->nq, QC);
    cp.batched = p->mnBatched ? 1 : 0;
    cp.maxIter = p->mnMaxIter;
    cp.nreg = p->nreg;
    cp.tol = p->mnTol;
    cp.tolGamma = p->mnBatched ? p->mnTolGamma : 1.1;
    cp.condHMax = p->mnCondHMax;
    c->m0 = M[0];
    for (int i = 0; i < p->nreg; ++i)
        cp.reg[i] = p->reg[i];
    cp.passBudget = 1LL << 40;
    c->psiBytes = p->psiBytes ? p->psiBytes : (size_t)32 << 30;
    c->reproject = p->mnReproject != 0;

    const long long nall = c->g.nall();
    const int nm = p->nm, nq = p->nq;
    auto alloc = [&](void **ptr, size_t bytes) -> bool {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    bool ok = alloc((void **)&c->u, nall * nm * 8) && alloc((void **)&c->alpha, nall * nm * 8) &&
              alloc((void **)&c->uOld, nall * nm * 8) && alloc((void **)&c->flux, nall * nm * 8) &&
              alloc((void **)&c->sigT, nall * 8) && alloc((void **)&c->sigS, nall * 8) &&
              alloc((void **)&c->M, (size_t)nq * nm * 8) && alloc((void **)&c->w, nq * 8) &&
              alloc((void **)&c->xi, nq * 8) && alloc((void **)&c->eta, nq * 8) &&
              alloc((void **)&c->mu, nq * 8) && alloc((void **)&c->iters, nall * 4) &&
              alloc((void **)&c->iterGamma, nall * 4) && alloc((void **)&c->regIdx, nall * 4) &&
              alloc((void **)&c->status, nall * 4) && alloc((void **)&c->counter, 8) &&
              alloc((void **)&c->failCount, 8) && alloc((void **)&c->errorFlag, 4) &&
              alloc((void **)&c->stats, STAT_COUNT * 8) && alloc((void **)&c->cellGamma, nall * 8) &&
              alloc((void **)&c->cellErr, nall * 8) && alloc((void **)&c->cellCond, nall * 4);
    std::vector<double> ch = build_chunks(nm, nq, M, w);
    ok = ok && alloc((void **)&c->chunks, ch.size() * 8);
    std::vector<double> mfA(flux_frag_doubles(nm, nq, 0)), mfP(flux_frag_doubles(nm, nq, 1));
    flux_frags(nm, nq, M, w, xi, eta, mu, 1.0 / p->dx, 1.0 / p->dy, 1.0 / p->dz, mfA.data(),
               mfP.data());
    ok = ok && alloc((void **)&c->mfA, mfA.size() * 8) && alloc((void **)&c->mfP, mfP.size() * 8);
    if (ok && pnOps)
        ok = alloc((void **)&c->pnops, (size_t)6 * nm * nm * 8);
    if (!ok) {
        free_ctx(c);
        return fail(C3D_ERR_OOM, "c3d_create: device allocation failed");
    }
    cudaMemcpy(c->M, M, (size_t)nq * nm * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->w, w, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->xi, xi, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->eta, eta, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->mu, mu, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->chunks, ch.data(), ch.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->mfA, mfA.data(), mfA.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(c->mfP, mfP.data(), mfP.size() * 8, cudaMemcpyHostToDevice);
    if (pnOps)
        cudaMemcpy(c->pnops, pnOps, (size_t)6 * nm * nm * 8, cudaMemcpyHostToDevice);
    cudaMemset(c->u, 0, nall * nm * 8);
    cudaMemset(c->alpha, 0, nall * nm * 8);
    cudaMemset(c->uOld, 0, nall * nm * 8);
    cudaMemset(c->flux, 0, nall * nm * 8);
    cudaMemset(c->iters, 0, nall * 4);
    cudaMemset(c->iterGamma, 0, nall * 4);
    cudaMemset(c->regIdx, 0, nall * 4);
    cudaMemset(c->status, 0, nall * 4);
    cudaMemset(c->failCount, 0, 8);
    cudaMemset(c->errorFlag, 0, 4);
    cudaMemset(c->stats, 0, STAT_COUNT * 8);
    {
        std::vector<float> none((size_t)nall, -1.0f); // no condition record yet
        cudaMemcpy(c->cellCond, none.data(), (size_t)nall * 4, cudaMemcpyHostToDevice);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        free_ctx(c);
        return fail(C3D_ERR_CUDA, std::string("c3d_create: ") + cudaGetErrorString(e));
    }
    // direction chunk of the materialised ansatz: shared-memory and HBM budgets
    // (whole tiles of 32 unless one chunk covers every direction)
    long long byBudget = (long long)(c->psiBytes / ((size_t)nall * 8));
    int qc = byBudget >= nq ? nq : (int)(byBudget / 32) * 32;
    if (qc < 32)
        qc = nq < 32 ? nq : 32;
    c->qChunk = qc;
    *out = c;
    return C3D_OK;
}

void c3d_destroy(c3d_ctx *ctx)
{
    if (!ctx)
        return;
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
}

c3d_status c3d_set_state(c3d_ctx *c, const double *u, const double *alpha, const double *sigT,
                         const double *sigS, int where)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_state: null context");
    if (alpha) {
        c->psiReady = false;
        psi_invalidate(c);
    }
    const long long nall = c->g.nall();
    const size_t vb = nall * c->g.nm * 8, sb = nall * 8;
    cudaMemcpyKind k = where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (u)
        C3D_CUDA(cudaMemcpyAsync(c->u, u, vb, k, c->stream));
    if (alpha)
        C3D_CUDA(cudaMemcpyAsync(c->alpha, alpha, vb, k, c->stream));
    if (sigT)
        C3D_CUDA(cudaMemcpyAsync(c->sigT, sigT, sb, k, c->stream));
    if (sigS)
        C3D_CUDA(cudaMemcpyAsync(c->sigS, sigS, sb, k, c->stream));
    if (!where)
        C3D_CUDA(cudaStreamSynchronize(c->stream));
    return C3D_OK;
}

c3d_status c3d_get_state(c3d_ctx *c, double *u, double *alpha, int where)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_get_state: null context");
    const size_t vb = c->g.nall() * c->g.nm * 8;
    cudaMemcpyKind k = where ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (u)
        C3D_CUDA(cudaMemcpyAsync(u, c->u, vb, k, c->stream));
    if (alpha)
        C3D_CUDA(cudaMemcpyAsync(alpha, c->alpha, vb, k, c->stream));
    if (!where)
        C3D_CUDA(cudaStreamSynchronize(c->stream));
    return C3D_OK;
}

c3d_status c3d_get_flux(c3d_ctx *c, double *flux, int where)
{
    if (!c || !flux)
        return fail(C3D_ERR_INVALID, "c3d_get_flux: null argument");
    const size_t vb = c->g.nall() * c->g.nm * 8;
    C3D_CUDA(cudaMemcpyAsync(flux, c->flux, vb, where ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                             c->stream));
    if (!where)
        C3D_CUDA(cudaStreamSynchronize(c->stream));
    return C3D_OK;
}

c3d_status c3d_device_state(c3d_ctx *c, double **u, double **alpha, double **flux)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_device_state: null context");
    if (u)
        *u = c->u;
    if (alpha)
        *alpha = c->alpha;
    if (flux)
        *flux = c->flux;
    return C3D_OK;
}

c3d_status c3d_ghost_fill(c3d_ctx *c)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_ghost_fill: null context");
    cudaEvent_t t0 = nullptr;
    timing_begin(c, &t0);
    C3D_CUDA(launch_ghost_fill(c->g, c->u, c->numSMs, c->stream, c->xHaloExternal));
    timing_end(c, 2, t0);
    c->launches += 1;
    return C3D_OK;
}

// Work-list buffers for n cells (grown on demand).
static c3d_status ensure_rounds(c3d_ctx *c, long long n)
{
    size_t per = rounds_buf_doubles(c->g.nm, c->nm2, c->gaunt, c->gaunt && c->cp.mixed);
    long long batch = n < c->maxBatch ? n : c->maxBatch;
    if (n <= c->rCells && per <= c->rBufPer && batch <= c->rBatch) {
        c->rBatchUse = batch;
        return C3D_OK;
    }
    void *ptrs[] = {c->rState, c->rListA, c->rListB, c->rCounts, c->rBuf};
    for (void *p : ptrs)
        if (p)
            cudaFree(p);
    c->rState = nullptr;
    c->rListA = c->rListB = nullptr;
    c->rCounts = nullptr;
    c->rBuf = nullptr;
    c->rCells = c->rBatch = 0;
    C3D_CUDA(cudaMalloc(&c->rState, (size_t)n * rounds_state_bytes(c->g.nm)));
    // one list per precision level (the FP64 closure uses the first)
    C3D_CUDA(cudaMalloc(&c->rListA, 4 * (size_t)n * sizeof(int)));
    C3D_CUDA(cudaMalloc(&c->rListB, 4 * (size_t)n * sizeof(int)));
    C3D_CUDA(cudaMalloc(&c->rCounts, 16 * sizeof(unsigned int)));
    C3D_CUDA(cudaMalloc(&c->rBuf, (size_t)batch * per * sizeof(double)));
    if (!c->rHostCount)
        C3D_CUDA(cudaMallocHost(&c->rHostCount, 4 * sizeof(unsigned int)));
    c->rCells = n;
    c->rBatch = batch;
    c->rBatchUse = batch;
    c->rBufPer = per;
    return C3D_OK;
}

// gridRecords: the closure covers the context's grid (directly or through cellMap), so the
// per-cell gamma and |g| records of the context (nall entries) receive its results.
// The work-list closure of n cells (engine 0): buffers sized, the launch description filled;
// the hand-off's refresh count is cleared on st (the stream the closure will run on, or the
// stream capturing it).
static c3d_status rounds_setup(c3d_ctx *c, long long n, double *u, double *alpha, int *iters,
                               int *iterGamma, int *regIdx, int *status, const int *cellMap,
                               bool gridRecords, cudaStream_t st, RoundsLaunch &R)
{
    double *recGamma = gridRecords ? c->cellGamma : nullptr;
    double *recErr = gridRecords ? c->cellErr : nullptr;
    {
        c3d_status s = ensure_rounds(c, n);
        if (s != C3D_OK)
            return s;
        R = RoundsLaunch{};
        R.P = &c->cp;
        R.chunks = c->gaunt ? c->gChunksC : c->chunks;
        R.nm2 = c->nm2;
        R.gstream = c->gStream;
        R.streamLen = c->gStreamLen;
        R.m0 = c->m0;
        R.ncells = n;
        R.cellMap = cellMap;
        R.u = u;
        R.alpha = alpha;
        R.iters = iters;
        R.iterGamma = iterGamma;
        R.regIdx = regIdx;
        R.status = status;
        R.failCount = c->failCount;
        R.stats = c->stats;
        R.gamma = recGamma;
        R.normG = recErr;
        R.cond = gridRecords ? c->cellCond : nullptr;
        R.mixF64 = c->mixF64;
        R.mixA[0] = c->mixA[0];
        R.mixA[1] = c->mixA[1];
        R.g0 = c->g0;
        R.g0n = c->g0n;
        // the certificate's gamma record is a bound: off while the x-line log records gammas
        c->cp.probe = c->gaunt && c->certificate && c->lineCap == 0 &&
                      (c->cp.mixed || c->g0Valid) && c->cp.gramLo > 0.0;
        R.state = c->rState;
        R.listA = c->rListA;
        R.listB = c->rListB;
        R.counts = c->rCounts;
        R.hostCount = c->rHostCount;
        R.buf = c->rBuf;
        R.batch = c->rBatchUse;
        R.errorFlag = c->errorFlag;
        R.stream = c->stream;
        R.launches = &c->launches;
        R.hostSyncs = &c->hostSyncs;
        R.maxRounds = c->maxRounds;
        R.graphs = nullptr;
        R.launchDev = nullptr;
        if (c->graphs) {
            if (!c->roundsGraph)
                c->roundsGraph = rounds_graph_new();
            if (!c->launchDev) {
                C3D_CUDA(cudaMalloc(&c->launchDev, sizeof(unsigned long long)));
                C3D_CUDA(cudaMemset(c->launchDev, 0, sizeof(unsigned long long)));
            }
            R.graphs = c->roundsGraph;
            R.launchDev = c->launchDev;
        }
        R.psi = nullptr;
        if (gridRecords && c->cp.probe && c->handoff && c->solver == 1) {
            // hand the probe's ansatz to the kinetic flux when psi of every direction fits the
            // budget
            const size_t need = (size_t)c->nq * c->g.nall() * 8;
            if (need <= c->psiBytes) {
                if (!c->psiRefresh) {
                    C3D_CUDA(cudaMalloc(&c->psiRefresh, (size_t)c->g.nall() * sizeof(int)));
                    C3D_CUDA(cudaMalloc(&c->psiRefreshCount, sizeof(unsigned int)));
                    C3D_CUDA(cudaMalloc(&c->psiValid, sizeof(int)));
                    C3D_CUDA(cudaMemset(c->psiValid, 0, sizeof(int)));
                }
                if (!c->psi || c->psiAlloc < need) {
                    if (c->psi)
                        cudaFree(c->psi);
                    c->psi = nullptr;
                    c->psiAlloc = 0;
                    C3D_CUDA(cudaMalloc(&c->psi, need));
                    c->psiAlloc = need;
                    C3D_CUDA(cudaMemset(c->psiValid, 0, sizeof(int)));
                }
                C3D_CUDA(cudaMemsetAsync(c->psiRefreshCount, 0, sizeof(unsigned int), st));
                R.psi = c->psi;
                R.psiNall = c->g.nall();
                R.refresh = c->psiRefresh;
                R.refreshCount = c->psiRefreshCount;
                R.psiValid = c->psiValid;
                R.gnx = c->g.nx;
                R.gny = c->g.ny;
                R.gnz = c->g.nz;
            }
        }
        R.stream = st;
    }
    return C3D_OK;
}

static c3d_status run_closure(c3d_ctx *c, long long n, double *u, double *alpha, int *iters,
                              int *iterGamma, int *regIdx, int *status, const int *cellMap = nullptr,
                              bool gridRecords = false)
{
    double *recGamma = gridRecords ? c->cellGamma : nullptr;
    double *recErr = gridRecords ? c->cellErr : nullptr;
    if (c->engine == 0) {
        RoundsLaunch R;
        c3d_status s = rounds_setup(c, n, u, alpha, iters, iterGamma, regIdx, status, cellMap,
                                    gridRecords, c->stream, R);
        if (s != C3D_OK)
            return s;
        c->psiReady = false;
        if (gridRecords && !R.psi)
            psi_invalidate(c);
        cudaError_t e = launch_closure_rounds(R, c->gaunt);
        if (e == cudaErrorLaunchTimeout)
            return fail(C3D_ERR_TIMEOUT, "closure: round limit exceeded");
        C3D_CUDA(e);
        if (R.psi)
            c->psiHandoffPending = true;
        return C3D_OK;
    }
    c->cp.probe = 0; // the persistent kernels always form H
    if (gridRecords)
        psi_invalidate(c);
    ClosureLaunch L{};
    L.P = &c->cp;
    L.chunks = c->chunks;
    L.ncells = n;
    L.counter = c->counter;
    L.u = u;
    L.alpha = alpha;
    L.iters = iters;
    L.iterGamma = iterGamma;
    L.regIdx = regIdx;
    L.status = status;
    L.failCount = c->failCount;
    L.stats = c->stats;
    L.gamma = recGamma;
    L.normG = recErr;
    L.errorFlag = c->errorFlag;
    L.numSMs = c->numSMs;
    L.stream = c->stream;
    if (c->gaunt && closure_gaunt_supported(c->g.nm)) {
        // (the persistent Gaunt kernels cover N <= 6; N = 7 forms H by direct quadrature,
        // the same H up to rounding)
        GauntTables G{c->gChunks, c->gRow, c->gCol, c->gVal};
        C3D_CUDA(launch_closure_gaunt(L, G));
    } else {
        C3D_CUDA(launch_closure_fp64(L));
    }
    c->launches += 2; // counter reset + closure kernel
    return C3D_OK;
}

static c3d_status closure_grid(c3d_ctx *c);

c3d_status c3d_closure(c3d_ctx *c)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_closure: null context");
    if (c->solver != 1)
        return fail(C3D_ERR_INVALID, "c3d_closure: the closure belongs to the M_N solver");
    cudaEvent_t t0 = nullptr;
    timing_begin(c, &t0);
    c3d_status s = closure_grid(c);
    if (s != C3D_OK)
        return s;
    if (c->lineLog && c->lineCount < c->lineCap) {
        C3D_CUDA(launch_line_log(c->g, c->cp, c->iters, c->iterGamma, c->regIdx, c->cellGamma,
                                 c->cellErr, c->lineLog + (size_t)c->lineCount * c->g.nx * 5,
                                 c->stream));
        c->lineCount++;
        c->launches += 1;
    }
    if (c->reproject) {
        C3D_CUDA(launch_reproject(c->g, c->u, c->alpha, c->mfA, c->mfP, c->nq, c->errorFlag,
                                  c->stream));
        c->launches += 1;
        psi_invalidate(c); // alpha_0 moved
    }
    timing_end(c, 0, t0);
    return C3D_OK;
}

// Completes the ansatz hand-off of a grid closure whose probe pass wrote psi: face ghosts
// copied from their images (mirrored closures), the listed cells recomputed from their final
// multipliers; the next kinetic flux then runs the stencil alone.
static c3d_status finish_handoff(c3d_ctx *c, bool faceCopy)
{
    if (!c->psiHandoffPending)
        return C3D_OK;
    c->psiHandoffPending = false;
    C3D_CUDA(launch_psi_handoff(c->g, c->nq, c->M, c->alpha, faceCopy, c->psiRefresh,
                                c->psiRefreshCount, c->psi, c->psiValid, c->numSMs, c->stream));
    c->launches += faceCopy ? 2 : 1;
    c->psiReady = true;
    return C3D_OK;
}

// The closure cells of a mirrored closure: every cell but the face ghosts.
static c3d_status ensure_cellmap(c3d_ctx *c)
{
    {
        if (!c->cellMap) {
            std::vector<int> map;
            const GridDims &g = c->g;
            map.reserve((size_t)g.nall());
            for (int i = 0; i < g.nxg(); ++i)
                for (int j = 0; j < g.nyg(); ++j)
                    for (int k = 0; k < g.nzg(); ++k) {
                        int gi = (i >= 2 && i < g.nx + 2), gj = (j >= 2 && j < g.ny + 2),
                            gk = (k >= 2 && k < g.nz + 2);
                        if (gi + gj + gk != 2) // not a face ghost
                            map.push_back((int)g.cell(i, j, k));
                    }
            if (cudaMalloc(&c->cellMap, map.size() * sizeof(int)) != cudaSuccess ||
                cudaMalloc(&c->mirrorFlag, sizeof(int)) != cudaSuccess ||
                cudaMallocHost(&c->mirrorHost, sizeof(int)) != cudaSuccess) {
                cudaGetLastError();
                return fail(C3D_ERR_OOM, "c3d_closure: device allocation failed");
            }
            C3D_CUDA(cudaMemcpy(c->cellMap, map.data(), map.size() * sizeof(int),
                                cudaMemcpyHostToDevice));
            c->cellMapCount = (long long)map.size();
        }
    }
    return C3D_OK;
}

static c3d_status closure_grid(c3d_ctx *c)
{
    if (c->engine == 0 && c->mirror && !c->xHaloExternal) {
        // Face ghosts hold copies of their periodic images (src/comm.cpp:281-323); when their
        // multipliers (the warm starts) are bitwise those of the images too, the per-cell
        // solve of the reference gives them the images' results, so they are copied after
        // solving the other cells instead. Edge and corner ghosts are solved as before.
        c3d_status sm = ensure_cellmap(c);
        if (sm != C3D_OK)
            return sm;
        C3D_CUDA(cudaMemsetAsync(c->mirrorFlag, 0, sizeof(int), c->stream));
        C3D_CUDA(launch_ghost_mirror_check(c->g, c->alpha, c->mirrorFlag, c->numSMs, c->stream));
        C3D_CUDA(cudaMemcpyAsync(c->mirrorHost, c->mirrorFlag, sizeof(int), cudaMemcpyDeviceToHost,
                                 c->stream));
        C3D_CUDA(cudaStreamSynchronize(c->stream));
        c->hostSyncs++;
        c->launches += 1;
        if (*c->mirrorHost == 0) {
            c3d_status s = run_closure(c, c->cellMapCount, c->u, c->alpha, c->iters, c->iterGamma,
                                       c->regIdx, c->status, c->cellMap, true);
            if (s != C3D_OK)
                return s;
            C3D_CUDA(launch_ghost_fill(c->g, c->alpha, c->numSMs, c->stream));
            C3D_CUDA(launch_ghost_fill(c->g, c->u, c->numSMs, c->stream));
            for (int *a : {c->iters, c->iterGamma, c->regIdx, c->status})
                C3D_CUDA(launch_ghost_fill_int(c->g, a, c->numSMs, c->stream));
            for (double *a : {c->cellGamma, c->cellErr})
                C3D_CUDA(launch_ghost_fill_1(c->g, a, c->numSMs, c->stream));
            C3D_CUDA(launch_ghost_stats(c->g, c->iters, c->iterGamma, c->regIdx, c->status,
                                        c->stats, c->numSMs, c->stream));
            c->launches += 9;
            c->mirroredClosures++;
            return finish_handoff(c, true);
        }
    }
    c3d_status s = run_closure(c, c->g.nall(), c->u, c->alpha, c->iters, c->iterGamma, c->regIdx,
                               c->status, nullptr, true);
    if (s != C3D_OK)
        return s;
    return finish_handoff(c, false);
}

// Round to nearest even (BF16) and to nearest with ties away (TF32, as cvt.rna), on the
// FP32 bit pattern; finite inputs.
static uint16_t host_bf16(float x)
{
    uint32_t b;
    std::memcpy(&b, &x, 4);
    b += 0x7FFFu + ((b >> 16) & 1u);
    return (uint16_t)(b >> 16);
}
static uint32_t host_tf32(float x)
{
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return (b + 0x1000u) & 0xFFFFE000u;
}

// Staged chunks of the mixed-precision pass (closure_rounds.cu): per 32-direction chunk the
// nm rows of M2 of degree <= N and the weight row in FP64 (row stride QCP), and the A
// operand -- M2's rows padded to max(nm2p, 128) -- in the tensor cores' K-major core-matrix
// layout: element (r, q) at (r / 8) SBO + (q es / 16) 128 + (r % 8) 16 + (q es) % 16 with
// SBO = 128 (QC es / 16); BF16 (es 2), and TF32 (es 4) hi then lo = tf32(M2 - hi).
static c3d_status build_mixed_chunks(c3d_ctx *c, int nm2, const double *M2,
                                     const std::vector<double> &wh)
{
    const int nm = c->g.nm, nq = c->nq, nch = ceil_div(nq, QC);
    const size_t perF = (size_t)(nm + 1) * QCP;
    std::vector<double> f((size_t)nch * perF, 0.0);
    const size_t ab[2] = {mixed_a_chunk_bytes(nm2, 0), mixed_a_chunk_bytes(nm2, 1)};
    const int nm2p = 8 * ((nm2 + 7) / 8), na = nm2p < 128 ? 128 : nm2p;
    std::vector<unsigned char> a0((size_t)nch * ab[0], 0), a1((size_t)nch * ab[1], 0);
    const size_t tfPiece = (size_t)na * QC * 4;
    for (int k = 0; k < nch; ++k)
        for (int qq = 0; qq < QC; ++qq) {
            const int q = k * QC + qq;
            if (q >= nq)
                break;
            for (int r = 0; r < nm; ++r)
                f[k * perF + (size_t)r * QCP + qq] = M2[(size_t)q * nm2 + r];
            f[k * perF + (size_t)nm * QCP + qq] = wh[q];
            for (int r = 0; r < nm2; ++r) {
                const double v = M2[(size_t)q * nm2 + r];
                const size_t o16 = (size_t)(r / 8) * (QC * 2 / 16) * 128 + (qq * 2 / 16) * 128 +
                                   (r % 8) * 16 + (qq * 2) % 16;
                const uint16_t h = host_bf16((float)v);
                std::memcpy(&a0[k * ab[0] + o16], &h, 2);
                const size_t o32 = (size_t)(r / 8) * (QC * 4 / 16) * 128 + (qq * 4 / 16) * 128 +
                                   (r % 8) * 16 + (qq * 4) % 16;
                const uint32_t hi = host_tf32((float)v);
                float hf;
                std::memcpy(&hf, &hi, 4);
                const uint32_t lo = host_tf32((float)(v - (double)hf));
                std::memcpy(&a1[k * ab[1] + o32], &hi, 4);
                std::memcpy(&a1[k * ab[1] + tfPiece + o32], &lo, 4);
            }
        }
    double *df = nullptr;
    unsigned char *da0 = nullptr, *da1 = nullptr;
    if (cudaMalloc(&df, f.size() * 8) != cudaSuccess || cudaMalloc(&da0, a0.size()) != cudaSuccess ||
        cudaMalloc(&da1, a1.size()) != cudaSuccess) {
        cudaGetLastError();
        if (df) cudaFree(df);
        if (da0) cudaFree(da0);
        return fail(C3D_ERR_OOM, "c3d_set_gaunt: device allocation failed");
    }
    C3D_CUDA(cudaMemcpy(df, f.data(), f.size() * 8, cudaMemcpyHostToDevice));
    C3D_CUDA(cudaMemcpy(da0, a0.data(), a0.size(), cudaMemcpyHostToDevice));
    C3D_CUDA(cudaMemcpy(da1, a1.data(), a1.size(), cudaMemcpyHostToDevice));
    if (c->mixF64) cudaFree(c->mixF64);
    if (c->mixA[0]) cudaFree(c->mixA[0]);
    if (c->mixA[1]) cudaFree(c->mixA[1]);
    c->mixF64 = df;
    c->mixA[0] = da0;
    c->mixA[1] = da1;
    return C3D_OK;
}

// Tables of the first-visit convergence certificate: the Gaunt terms of H's column 0 (CSR
// row i of element (i, 0), in order; rows padded to the longest with col -2) -- valid when
// they reference only moments of the probe's rows (< nm) -- and the Gershgorin bounds of the
// quadrature's Gram matrix G = sum_q w_q m_q m_q^T (the first nm rows of M2 are the basis).
static c3d_status build_certificate(c3d_ctx *c, int nm2, const double *M2,
                                    const std::vector<double> &wh, const int *rowPtr,
                                    const int *colInd, const double *val)
{
    const int nm = c->g.nm, nq = c->nq;
    int g0n = 1;
    bool valid = true;
    for (int i = 0; i < nm; ++i) {
        g0n = std::max(g0n, rowPtr[i + 1] - rowPtr[i]);
        for (int k = rowPtr[i]; k < rowPtr[i + 1]; ++k)
            valid = valid && colInd[k] >= 0 && colInd[k] < nm;
    }
    std::vector<GauntTerm> t((size_t)nm * g0n, GauntTerm{0.0, -2, -1});
    for (int i = 0; i < nm; ++i)
        for (int k = rowPtr[i]; k < rowPtr[i + 1]; ++k)
            t[(size_t)i * g0n + (k - rowPtr[i])] = GauntTerm{val[k], colInd[k], -1};
    std::vector<double> G((size_t)nm * nm, 0.0);
    for (int q = 0; q < nq; ++q)
        for (int i = 0; i < nm; ++i)
            for (int j = 0; j < nm; ++j)
                G[(size_t)i * nm + j] += wh[q] * M2[(size_t)q * nm2 + i] * M2[(size_t)q * nm2 + j];
    double lo = 1.0 / 0.0, hi = 0.0;
    for (int i = 0; i < nm; ++i) {
        double off = 0.0;
        for (int j = 0; j < nm; ++j)
            if (j != i)
                off += std::fabs(G[(size_t)i * nm + j]);
        lo = std::min(lo, G[(size_t)i * nm + i] - off);
        hi = std::max(hi, G[(size_t)i * nm + i] + off);
    }
    // rounding of the host sums: a relative margin far above nq eps
    lo *= 1.0 - 1e-9;
    hi *= 1.0 + 1e-9;
    GauntTerm *d = nullptr;
    if (cudaMalloc(&d, t.size() * sizeof(GauntTerm)) != cudaSuccess) {
        cudaGetLastError();
        return fail(C3D_ERR_OOM, "c3d_set_gaunt: device allocation failed");
    }
    C3D_CUDA(cudaMemcpy(d, t.data(), t.size() * sizeof(GauntTerm), cudaMemcpyHostToDevice));
    if (c->g0) cudaFree(c->g0);
    c->g0 = d;
    c->g0n = g0n;
    c->g0Valid = valid;
    c->cp.gramLo = lo;
    c->cp.gramHi = hi;
    return C3D_OK;
}

c3d_status c3d_set_gaunt(c3d_ctx *c, int nm2, const double *M2, const int *rowPtr,
                         const int *colInd, const double *val)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_gaunt: null context");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    if (!M2 || !rowPtr || !colInd || !val) {
        // back to the direct form (FP64: the mixed closure needs the Gaunt form)
        c->gaunt = false;
        c->cp.mixed = 0;
        return C3D_OK;
    }
    const int nm = c->g.nm, nq = c->nq;
    int n2 = (int)std::lround(std::sqrt((double)nm));
    if (nm2 != (2 * n2 - 1) * (2 * n2 - 1))
        return fail(C3D_ERR_INVALID, "c3d_set_gaunt: nm2 must be (2N+1)^2");
    if (!rounds_gaunt_supported(nm))
        return fail(C3D_ERR_INVALID, "c3d_set_gaunt: the Gaunt form is provided for N <= 7");
    const int nm2p = closure_gaunt_nm2p(nm2);
    const int nch = ceil_div(nq, QC);
    const size_t per = (size_t)(nm2p + 1) * QCP;
    std::vector<double> ch((size_t)nch * per, 0.0), wh(nq);
    C3D_CUDA(cudaMemcpy(wh.data(), c->w, nq * 8, cudaMemcpyDeviceToHost));
    for (int k = 0; k < nch; ++k)
        for (int qq = 0; qq < QC; ++qq) {
            int q = k * QC + qq;
            if (q >= nq)
                break;
            for (int r = 0; r < nm2; ++r)
                ch[k * per + (size_t)r * QCP + qq] = M2[(size_t)q * nm2 + r];
            ch[k * per + (size_t)nm2p * QCP + qq] = wh[q];
        }
    const int nnz = rowPtr[nm * nm];
    double *dch = nullptr, *dval = nullptr;
    int *drow = nullptr, *dcol = nullptr;
    if (cudaMalloc(&dch, ch.size() * 8) != cudaSuccess ||
        cudaMalloc(&drow, (size_t)(nm * nm + 1) * 4) != cudaSuccess ||
        cudaMalloc(&dcol, (size_t)(nnz > 0 ? nnz : 1) * 4) != cudaSuccess ||
        cudaMalloc(&dval, (size_t)(nnz > 0 ? nnz : 1) * 8) != cudaSuccess) {
        cudaGetLastError();
        if (dch) cudaFree(dch);
        if (drow) cudaFree(drow);
        if (dcol) cudaFree(dcol);
        if (dval) cudaFree(dval);
        return fail(C3D_ERR_OOM, "c3d_set_gaunt: device allocation failed");
    }
    cudaMemcpy(dch, ch.data(), ch.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(drow, rowPtr, (size_t)(nm * nm + 1) * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dcol, colInd, (size_t)nnz * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dval, val, (size_t)nnz * 8, cudaMemcpyHostToDevice);
    // compact chunks of the work-list engine: nm2 rows of M2, then the weights
    const size_t perC = (size_t)(nm2 + 1) * QCP;
    std::vector<double> chc((size_t)nch * perC, 0.0);
    for (int k = 0; k < nch; ++k)
        for (int qq = 0; qq < QC; ++qq) {
            int q = k * QC + qq;
            if (q >= nq)
                break;
            for (int r = 0; r < nm2; ++r)
                chc[k * perC + (size_t)r * QCP + qq] = M2[(size_t)q * nm2 + r];
            chc[k * perC + (size_t)nm2 * QCP + qq] = wh[q];
        }
    double *dchc = nullptr;
    if (cudaMalloc(&dchc, chc.size() * 8) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dch);
        cudaFree(drow);
        cudaFree(dcol);
        cudaFree(dval);
        return fail(C3D_ERR_OOM, "c3d_set_gaunt: device allocation failed");
    }
    cudaMemcpy(dchc, chc.data(), chc.size() * 8, cudaMemcpyHostToDevice);
    if (c->gChunksC) cudaFree(c->gChunksC);
    c->gChunksC = dchc;
    // assembly streams of the tiled Hessian (work-list engine). Thread t of the Newton
    // kernel's CTA owns the tile slots e = t + 128 i of the lower triangle of 8x8 tiles; its
    // stream lists, slot after slot, the CSR terms of beta for that slot's (row >= col)
    // element in the reference's order, the last one marked with the slot (a slot without
    // terms gets one zero term; identity padding slots one col = -1 entry). Streams are
    // padded to a common length with no-op entries and interleaved across threads
    // (entry s of thread t at s * 128 + t) so that a warp's loads coalesce.
    const int nt = (nm + 7) / 8, ls = 64 * nt * (nt + 1) / 2;
    std::vector<std::vector<GauntTerm>> lists(NEWTON_THREADS);
    for (int e = 0; e < ls; ++e) {
        std::vector<GauntTerm> &st = lists[e % NEWTON_THREADS];
        // storage offset e & 63 inside tile e >> 6 -> element (rr, cc), the inverse of toff
        const int t = e >> 6, rr = (e >> 3) & 7;
        const int cc = 2 * (((e >> 1) & 3) ^ ((rr >> 1) & 3)) + (e & 1);
        int ib = 0;
        while ((ib + 1) * (ib + 2) / 2 <= t)
            ++ib;
        const int jb = t - ib * (ib + 1) / 2;
        const int i = 8 * ib + rr, j = 8 * jb + cc;
        const size_t first = st.size();
        if (!(ib == jb && cc > rr)) {
            if (i >= nm || j >= nm) {
                if (i == j)
                    st.push_back(GauntTerm{1.0, -1, -1});
            } else {
                const int idx = j * nm + i;
                for (int k = rowPtr[idx]; k < rowPtr[idx + 1]; ++k)
                    st.push_back(GauntTerm{val[k], colInd[k], -1});
            }
        }
        if (st.size() == first)
            st.push_back(GauntTerm{0.0, 0, -1});
        st.back().slot = e;
    }
    size_t len = 0;
    for (auto &st : lists)
        len = st.size() > len ? st.size() : len;
    std::vector<GauntTerm> stream(len * NEWTON_THREADS, GauntTerm{0.0, 0, -1});
    for (int t = 0; t < NEWTON_THREADS; ++t)
        for (size_t k = 0; k < lists[t].size(); ++k)
            stream[k * NEWTON_THREADS + t] = lists[t][k];
    GauntTerm *dstream = nullptr;
    if (cudaMalloc(&dstream, stream.size() * sizeof(GauntTerm)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dch);
        cudaFree(drow);
        cudaFree(dcol);
        cudaFree(dval);
        return fail(C3D_ERR_OOM, "c3d_set_gaunt: device allocation failed");
    }
    cudaMemcpy(dstream, stream.data(), stream.size() * sizeof(GauntTerm), cudaMemcpyHostToDevice);
    C3D_CUDA(cudaDeviceSynchronize());
    if (c->gStream) cudaFree(c->gStream);
    c->gStream = dstream;
    c->gStreamLen = (int)len;
    if (c->gChunks) cudaFree(c->gChunks);
    if (c->gRow) cudaFree(c->gRow);
    if (c->gCol) cudaFree(c->gCol);
    if (c->gVal) cudaFree(c->gVal);
    c->gChunks = dch;
    c->gRow = drow;
    c->gCol = dcol;
    c->gVal = dval;
    c->gaunt = true;
    c->nm2 = nm2;
    c3d_status s = build_mixed_chunks(c, nm2, M2, wh);
    if (s != C3D_OK)
        return s;
    return build_certificate(c, nm2, M2, wh, rowPtr, colInd, val);
}

c3d_status c3d_set_precision(c3d_ctx *c, int mode, double condBf16, double condMixedMax,
                             int mixedIterMax, double polish)
{
    if (!c || mode < 0 || mode > 1)
        return fail(C3D_ERR_INVALID, "c3d_set_precision: mode must be 0 (FP64) or 1 (mixed)");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    if (mode == 1 && (!c->gaunt || c->engine != 0))
        return fail(C3D_ERR_INVALID,
                    "c3d_set_precision: the mixed closure needs the Gaunt form and engine 0");
    c->cp.mixed = mode;
    c->cp.condBf16 = condBf16 > 0 ? condBf16 : 1e4;
    c->cp.condMixMax = condMixedMax > 0 ? condMixedMax : 1e7;
    c->cp.mixIterMax = mixedIterMax > 0 ? mixedIterMax : 8;
    c->cp.mixPolish = polish > 0 ? polish : 1e3;
    // N <= 2 (at most 32 extended moments): the 128-row tensor-core tile would be mostly
    // padding and the FP64 moment pass is as cheap, so the Hessians stay FP64
    if (mode == 1 && closure_gaunt_nm2p(c->nm2) <= 32)
        c->cp.mixIterMax = 0;
    return C3D_OK;
}

c3d_status c3d_set_certificate(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_certificate: null context");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    c->certificate = on != 0;
    return C3D_OK;
}

c3d_status c3d_set_engine(c3d_ctx *c, int engine)
{
    if (!c || engine < 0 || engine > 1)
        return fail(C3D_ERR_INVALID, "c3d_set_engine: engine must be 0 (work list) or 1 (persistent)");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    c->engine = engine;
    if (engine != 0)
        c->cp.mixed = 0; // the persistent kernels are FP64 only
    return C3D_OK;
}

c3d_status c3d_set_graphs(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_graphs: null context");
    c->graphs = on != 0;
    return C3D_OK;
}

c3d_status c3d_set_ansatz_handoff(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_ansatz_handoff: null context");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    c->handoff = on != 0;
    if (!c->handoff)
        c->psiReady = false;
    return C3D_OK;
}

c3d_status c3d_set_limits(c3d_ctx *c, long long maxRounds, long long passBudget,
                          long long batch)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_limits: null context");
    c->maxRounds = maxRounds > 0 ? maxRounds : (1LL << 24);
    c->cp.passBudget = passBudget > 0 ? passBudget : (1LL << 40);
    c->maxBatch = batch > 0 ? batch : (1LL << 20);
    return C3D_OK;
}

c3d_status c3d_set_ghost_mirroring(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_ghost_mirroring: null context");
    c->mirror = on != 0;
    return C3D_OK;
}

c3d_status c3d_closure_vectors(c3d_ctx *c, long long n, double *u, double *alpha, int *iters,
                               int *iterGamma, int *regIndex, int *status)
{
    if (!c || !u || !alpha || n < 0)
        return fail(C3D_ERR_INVALID, "c3d_closure_vectors: bad argument");
    if (n == 0)
        return C3D_OK;
    return run_closure(c, n, u, alpha, iters, iterGamma, regIndex, status);
}

// Several contexts' standalone closures as parallel branches of one CUDA graph. cs: three
// capture streams per context (its closure, the round loop's body, the switch bodies) and an
// origin stream that forks to and joins the contexts' branches; the graph launches on the
// contexts' common stream.
struct c3d_group {
    std::vector<c3d_ctx *> ctx;
    std::vector<cudaStream_t> cs;
    cudaStream_t stream = nullptr;
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> launches; // per context: launches of one replay counted on the host
    // c3d_group_step's graph: every context's RK step as one branch
    std::vector<unsigned char> stepKey;
    cudaGraphExec_t stepExec = nullptr;
    std::vector<long long> stepLaunches;
};

static void group_streams_free(c3d_group *g)
{
    for (cudaStream_t &s : g->cs) {
        if (s)
            cudaStreamDestroy(s);
        s = nullptr;
    }
}

static cudaError_t group_streams_make(c3d_group *g)
{
    for (cudaStream_t &s : g->cs)
        if (!s) {
            cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (e != cudaSuccess)
                return e;
        }
    return cudaSuccess;
}

c3d_status c3d_group_create(int count, c3d_ctx *const *ctx, c3d_group **out)
{
    if (!out || !ctx || count < 1)
        return fail(C3D_ERR_INVALID, "c3d_group_create: bad argument");
    *out = nullptr;
    for (int k = 0; k < count; ++k) {
        if (!ctx[k] || ctx[k]->solver != 1)
            return fail(C3D_ERR_INVALID, "c3d_group_create: contexts must be M_N contexts");
        if (ctx[k]->stream != ctx[0]->stream)
            return fail(C3D_ERR_INVALID, "c3d_group_create: contexts must share one stream");
        for (int j = 0; j < k; ++j)
            if (ctx[j] == ctx[k])
                return fail(C3D_ERR_INVALID, "c3d_group_create: a context appears twice");
    }
    c3d_group *g = new c3d_group();
    g->ctx.assign(ctx, ctx + count);
    g->stream = ctx[0]->stream;
    g->cs.assign(3 * (size_t)count + 1, nullptr);
    g->launches.assign(count, 0);
    g->stepLaunches.assign(count, 0);
    cudaError_t e = group_streams_make(g);
    if (e != cudaSuccess) {
        group_streams_free(g);
        delete g;
        return fail(C3D_ERR_CUDA, std::string("c3d_group_create: ") + cudaGetErrorString(e));
    }
    *out = g;
    return C3D_OK;
}

void c3d_group_destroy(c3d_group *g)
{
    if (!g)
        return;
    cudaStreamSynchronize(g->stream); // a replay may still run
    if (g->exec)
        cudaGraphExecDestroy(g->exec);
    if (g->stepExec)
        cudaGraphExecDestroy(g->stepExec);
    group_streams_free(g);
    delete g;
}

c3d_status c3d_group_closure_vectors(c3d_group *g, const long long *n, double *const *u,
                                     double *const *alpha, int *const *iters,
                                     int *const *iterGamma, int *const *regIndex,
                                     int *const *status)
{
    if (!g || !n || !u || !alpha)
        return fail(C3D_ERR_INVALID, "c3d_group_closure_vectors: bad argument");
    const int K = (int)g->ctx.size();
    auto rec = [](int *const *a, int k) -> int * { return a ? a[k] : nullptr; };
    for (int k = 0; k < K; ++k) {
        const c3d_ctx *c = g->ctx[k];
        if (n[k] < 0 || (n[k] > 0 && (!u[k] || !alpha[k])))
            return fail(C3D_ERR_INVALID, "c3d_group_closure_vectors: bad vectors");
        if (c->engine != 0 || !c->graphs || c->timing)
            return fail(C3D_ERR_INVALID, "c3d_group_closure_vectors: the contexts need the "
                                         "work-list engine, graphs on and timing off");
    }
    // set-up of every closure (buffers are allocated here, never while capturing) and the
    // graph's key
    std::vector<RoundsLaunch> R(K);
    std::vector<unsigned char> key;
    for (int k = 0; k < K; ++k) {
        c3d_ctx *c = g->ctx[k];
        key.push_back((unsigned char)(n[k] > 0));
        if (n[k] == 0)
            continue;
        c3d_status s = rounds_setup(c, n[k], u[k], alpha[k], rec(iters, k), rec(iterGamma, k),
                                    rec(regIndex, k), rec(status, k), nullptr, false,
                                    g->cs[3 * k], R[k]);
        if (s != C3D_OK)
            return s;
        const std::vector<unsigned char> kk = rounds_graph_key(R[k], c->gaunt);
        key.insert(key.end(), kk.begin(), kk.end());
    }
    if (!g->exec || key != g->key) {
        std::lock_guard<std::mutex> lk(graph_build_mutex());
        if (g->exec) {
            C3D_CUDA(cudaStreamSynchronize(g->stream));
            cudaGraphExecDestroy(g->exec);
            g->exec = nullptr;
        }
        C3D_CUDA(group_streams_make(g));
        cudaStream_t o = g->cs[3 * K];
        std::vector<cudaEvent_t> ev(K + 1, nullptr);
        cudaError_t e = cudaSuccess;
        for (cudaEvent_t &x : ev)
            if (e == cudaSuccess)
                e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        cudaGraph_t top = nullptr;
        if (e == cudaSuccess)
            e = cudaGraphCreate(&top, 0);
        if (e == cudaSuccess) {
            e = cudaStreamBeginCaptureToGraph(o, top, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed);
            cudaError_t ec = e == cudaSuccess ? cudaEventRecord(ev[K], o) : e;
            for (int k = 0; k < K && ec == cudaSuccess; ++k) {
                c3d_ctx *c = g->ctx[k];
                g->launches[k] = 0;
                if (n[k] == 0)
                    continue;
                cudaStream_t *cs = &g->cs[3 * k];
                ec = cudaStreamWaitEvent(cs[0], ev[K], 0);
                if (ec != cudaSuccess)
                    break;
                R[k].stream = cs[0];
                R[k].captureTop = top;
                R[k].captureStreams = cs;
                const long long l0 = c->launches;
                ec = launch_closure_rounds(R[k], c->gaunt);
                g->launches[k] = c->launches - l0;
                c->launches = l0;
                if (ec == cudaSuccess)
                    ec = cudaEventRecord(ev[k], cs[0]);
                if (ec == cudaSuccess)
                    ec = cudaStreamWaitEvent(o, ev[k], 0);
            }
            if (e == cudaSuccess) {
                cudaGraph_t out = nullptr;
                e = cudaStreamEndCapture(o, &out);
                if (e == cudaSuccess)
                    e = ec;
            }
        }
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&g->exec, top, 0);
        if (top)
            cudaGraphDestroy(top);
        for (cudaEvent_t x : ev)
            if (x)
                cudaEventDestroy(x);
        if (e != cudaSuccess) {
            g->exec = nullptr;
            g->key.clear();
            group_streams_free(g); // streams left in a broken capture are replaced
            cudaGetLastError();
            return fail(C3D_ERR_CUDA, std::string("c3d_group_closure_vectors: group graph: ") +
                                          cudaGetErrorString(e));
        }
        g->key = key;
    }
    C3D_CUDA(cudaGraphLaunch(g->exec, g->stream));
    for (int k = 0; k < K; ++k) {
        g->ctx[k]->launches += g->launches[k];
        g->ctx[k]->psiReady = false;
    }
    return C3D_OK;
}

c3d_status c3d_flux_kinetic(c3d_ctx *c, int alphaIsU)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_flux_kinetic: null context");
    const size_t need = (size_t)c->qChunk * c->g.nall() * 8;
    if (!c->psi || c->psiAlloc < need) {
        if (c->psi)
            cudaFree(c->psi);
        c->psi = nullptr;
        c->psiAlloc = 0;
        C3D_CUDA(cudaMalloc(&c->psi, need));
        c->psiAlloc = need;
    }
    const double *a = alphaIsU ? c->u : c->alpha;
    int isPn = (c->solver == 0) ? 1 : 0;
    const bool ready = c->psiReady && !alphaIsU && isPn == 0 &&
                       c->psiAlloc >= (size_t)c->nq * c->g.nall() * 8;
    c->psiReady = false;
    if (!ready)
        psi_invalidate(c); // the ansatz kernel writes psi
    cudaEvent_t t0 = nullptr;
    timing_begin(c, &t0);
    C3D_CUDA(launch_kinetic_flux(c->g, a, c->mfA, c->mfP, c->xi, c->eta, c->nq, c->qChunk,
                                 c->runLen, c->theta, isPn, c->psi, ready, c->flux,
                                 c->errorFlag, nullptr, c->stream));
    timing_end(c, 1, t0);
    int nch = ceil_div(c->nq, c->qChunk);
    c->launches += ready ? 1 : 2 * nch;
    return C3D_OK;
}

// Flux autotuner: times the kinetic flux (one warm-up call, then the mean of two timed
// calls, CUDA events on the context's stream) for each direction chunk -- the largest the psi
// budget allows, and the balanced splits into 2 .. 4 more chunks -- and each z run length of
// the staged kernel (64 and 32 cells per CTA where nz allows), and keeps the fastest. The
// flux buffer is overwritten; the state is not touched.
c3d_status c3d_autotune(c3d_ctx *c, int *qChunk, int *runLen, double *msPerCall)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_autotune: null context");
    const int nq = c->nq;
    const long long nall = c->g.nall();
    long long byBudget = (long long)(c->psiBytes / ((size_t)nall * 8));
    int qmax = byBudget >= nq ? nq : (int)(byBudget / 32) * 32;
    if (qmax < 32)
        qmax = nq < 32 ? nq : 32;
    std::vector<int> qs{qmax};
    const int k0 = ceil_div(nq, qmax);
    for (int k = k0 + (qmax == nq ? 1 : 0); k <= k0 + 3; ++k) {
        int q = 32 * ceil_div(ceil_div(nq, k), 32);
        if (q < qmax && q >= 32 && std::find(qs.begin(), qs.end(), q) == qs.end())
            qs.push_back(q);
    }
    std::vector<int> ls{0};
    if (c->g.nz % 32 == 0 && c->g.nz > 32)
        ls.push_back(32);
    const int q0 = c->qChunk, l0 = c->runLen;
    const bool timing = c->timing;
    c->psiReady = false; // every timed call forms the ansatz
    c->timing = false;
    cudaEvent_t e0, e1;
    C3D_CUDA(cudaEventCreate(&e0));
    C3D_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    int bq = q0, bl = l0;
    for (int q : qs)
        for (int l : ls) {
            c->qChunk = q;
            c->runLen = l;
            c3d_status s = c3d_flux_kinetic(c, 0);
            if (s != C3D_OK) {
                c->qChunk = q0;
                c->runLen = l0;
                c->timing = timing;
                return s;
            }
            C3D_CUDA(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < 2; ++r)
                if ((s = c3d_flux_kinetic(c, 0)) != C3D_OK) {
                    c->qChunk = q0;
                    c->runLen = l0;
                    c->timing = timing;
                    return s;
                }
            C3D_CUDA(cudaEventRecord(e1, c->stream));
            C3D_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            C3D_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms / 2 < best) {
                best = ms / 2;
                bq = q;
                bl = l;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->timing = timing;
    c->qChunk = bq;
    c->runLen = bl;
    if (qChunk) *qChunk = bq;
    if (runLen) *runLen = bl;
    if (msPerCall) *msPerCall = best;
    return C3D_OK;
}

c3d_status c3d_flux_moment(c3d_ctx *c)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_flux_moment: null context");
    if (!c->pnops)
        return fail(C3D_ERR_INVALID, "c3d_flux_moment: no P_N operators in this context");
    C3D_CUDA(launch_moment_flux(c->g, c->u, c->pnops, c->dx, c->dy, c->dz, c->flux, c->stream));
    c->launches += 1;
    return C3D_OK;
}

c3d_status c3d_euler(c3d_ctx *c, double dt)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_euler: null context");
    cudaEvent_t t0 = nullptr;
    timing_begin(c, &t0);
    C3D_CUDA(launch_euler(c->g, c->u, c->flux, c->sigT, c->sigS, dt, c->numSMs, c->stream));
    timing_end(c, 3, t0);
    c->launches += 1;
    return C3D_OK;
}

// Sets an IF node's condition: mirrored closure when no face ghost's multipliers differ from
// its image's.
__global__ void mirror_if_kernel(const int *flag, cudaGraphConditionalHandle h)
{
    if (threadIdx.x == 0)
        cudaGraphSetConditional(h, *flag == 0 ? 1u : 0u);
}

// Whether a context's RK stages can run as CUDA graphs: the work-list engine with graphs on,
// and none of the options that need the stage launch by launch (timing events, the x-line
// log, re-projection) or the P_N solver.
static bool stage_graphs_usable(const c3d_ctx *c)
{
    return c->graphs && c->engine == 0 && !c->timing && c->lineCap == 0 && !c->reproject &&
           c->solver == 1;
}

// Buffers of a stage capture, allocated before it (nothing is allocated while capturing);
// *handoff: whether the closure hands its ansatz to the flux.
static c3d_status stage_prepare(c3d_ctx *c, bool *handoff)
{
    if (c->mirror && !c->xHaloExternal) {
        c3d_status sm = ensure_cellmap(c);
        if (sm != C3D_OK)
            return sm;
    }
    RoundsLaunch Rall;
    c3d_status s = rounds_setup(c, c->g.nall(), c->u, c->alpha, c->iters, c->iterGamma,
                                c->regIdx, c->status, nullptr, true, c->stream, Rall);
    if (s != C3D_OK)
        return s;
    if (!c->launchDev) {
        C3D_CUDA(cudaMalloc(&c->launchDev, sizeof(unsigned long long)));
        C3D_CUDA(cudaMemset(c->launchDev, 0, sizeof(unsigned long long)));
    }
    *handoff = Rall.psi != nullptr;
    if (!*handoff) {
        const size_t need = (size_t)c->qChunk * c->g.nall() * 8;
        if (!c->psi || c->psiAlloc < need) {
            if (c->psi)
                cudaFree(c->psi);
            c->psi = nullptr;
            c->psiAlloc = 0;
            C3D_CUDA(cudaMalloc(&c->psi, need));
            c->psiAlloc = need;
        }
    }
    for (cudaStream_t &x : c->sc)
        if (!x)
            C3D_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    return C3D_OK;
}

// What a captured stage depends on: equal keys, same graph.
static std::vector<unsigned char> stage_key(const c3d_ctx *c, int stage, double dt, bool handoff)
{
    std::vector<unsigned char> key;
    auto skey = [&key](const auto &v) {
        const unsigned char *b = reinterpret_cast<const unsigned char *>(&v);
        key.insert(key.end(), b, b + sizeof(v));
    };
    const bool mirrorPath = c->mirror && !c->xHaloExternal;
    skey(stage);
    skey(dt);
    skey(c->cp);
    skey(mirrorPath);
    skey(c->gaunt);
    skey(handoff);
    skey(c->qChunk);
    skey(c->runLen);
    skey(c->maxRounds);
    skey(c->rBatchUse);
    const void *ptrs[] = {c->psi, c->rState, c->rBuf, c->rListA, c->rCounts, c->cellMap,
                          c->gChunksC, c->chunks, c->gStream, c->mixF64, c->mixA[0],
                          c->mixA[1], c->g0, c->psiRefresh, c->launchDev, c->u, c->alpha};
    for (const void *p : ptrs)
        skey(p);
    return key;
}

// Appends one M_N RK stage of update() to the graph being captured on cs[0] (its top-level
// graph: top): [RK save,] ghost fill, the closure (with face-ghost mirroring: the mirror check
// picks, through an IF node, the mirrored closure with its ghost copies or the closure of
// every cell), the ansatz hand-off, the kinetic flux and the Euler stage[, RK average].
// Nothing in it waits for the host. cs[1] captures the IF bodies, cs[1..3] (mirrored) or
// cs[0..2] the closure's round loop and switch bodies. *launches: the kernels of one replay
// the host counts (the closure's device-side loop counts its own).
static cudaError_t stage_capture(c3d_ctx *c, int stage, double dt, bool handoff, cudaGraph_t top,
                                 cudaStream_t *cs, long long *launches)
{
    const bool mirrorPath = c->mirror && !c->xHaloExternal;
    // mirrored closure with the hand-off and the staged stencil: the face ghosts' psi is not
    // copied; the stencil reads their periodic images (the mirror flag tells it, on the device,
    // which closure body ran)
    const bool wrap = mirrorPath && handoff && kinetic_staged_used(c->g, c->runLen);
    const long long l0 = c->launches;
    long long n = 0;
    cudaStream_t s0 = cs[0];
    cudaError_t ec = cudaSuccess;
    if (stage == 0)
        ec = launch_rk(c->g, c->u, c->uOld, 0, c->numSMs, s0);
    if (ec == cudaSuccess)
        ec = launch_ghost_fill(c->g, c->u, c->numSMs, s0, c->xHaloExternal);
    n += (stage == 0) + 1;
    // the closure on stream cs[k] (its bodies on the next two) and what follows it
    auto closure = [&](bool mirrored, int k) -> cudaError_t {
        RoundsLaunch R;
        c3d_status rs = mirrored
                            ? rounds_setup(c, c->cellMapCount, c->u, c->alpha, c->iters,
                                           c->iterGamma, c->regIdx, c->status, c->cellMap, true,
                                           cs[k], R)
                            : rounds_setup(c, c->g.nall(), c->u, c->alpha, c->iters,
                                           c->iterGamma, c->regIdx, c->status, nullptr, true,
                                           cs[k], R);
        if (rs != C3D_OK)
            return cudaErrorInvalidValue;
        R.captureTop = top;
        R.captureStreams = &cs[k];
        cudaError_t er = launch_closure_rounds(R, c->gaunt);
        cudaStream_t sk = cs[k];
        if (er == cudaSuccess && mirrored) {
            er = launch_ghost_fill(c->g, c->alpha, c->numSMs, sk);
            if (er == cudaSuccess)
                er = launch_ghost_fill(c->g, c->u, c->numSMs, sk);
            for (int *a : {c->iters, c->iterGamma, c->regIdx, c->status})
                if (er == cudaSuccess)
                    er = launch_ghost_fill_int(c->g, a, c->numSMs, sk);
            for (double *a : {c->cellGamma, c->cellErr})
                if (er == cudaSuccess)
                    er = launch_ghost_fill_1(c->g, a, c->numSMs, sk);
            if (er == cudaSuccess)
                er = launch_ghost_stats(c->g, c->iters, c->iterGamma, c->regIdx, c->status,
                                        c->stats, c->numSMs, sk);
        }
        if (er == cudaSuccess && R.psi)
            er = launch_psi_handoff(c->g, c->nq, c->M, c->alpha, mirrored && !wrap, c->psiRefresh,
                                    c->psiRefreshCount, c->psi, c->psiValid, c->numSMs, sk);
        return er;
    };
    if (ec == cudaSuccess && mirrorPath) {
        ec = cudaMemsetAsync(c->mirrorFlag, 0, sizeof(int), s0);
        if (ec == cudaSuccess)
            ec = launch_ghost_mirror_check(c->g, c->alpha, c->mirrorFlag, c->numSMs, s0);
        cudaGraphConditionalHandle hIf;
        if (ec == cudaSuccess)
            ec = cudaGraphConditionalHandleCreate(&hIf, top, 0, cudaGraphCondAssignDefault);
        if (ec == cudaSuccess) {
            mirror_if_kernel<<<1, 32, 0, s0>>>(c->mirrorFlag, hIf);
            ec = cudaGetLastError();
        }
        cudaGraph_t *bodies = nullptr;
        if (ec == cudaSuccess)
            ec = capture_conditional(s0, hIf, cudaGraphCondTypeIf, 2, &bodies);
        for (int b = 0; b < 2 && ec == cudaSuccess; ++b) {
            ec = cudaStreamBeginCaptureToGraph(cs[1], bodies[b], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed);
            if (ec == cudaSuccess) {
                cudaError_t eb = closure(b == 0, 1);
                cudaGraph_t out = nullptr;
                ec = cudaStreamEndCapture(cs[1], &out);
                if (ec == cudaSuccess)
                    ec = eb;
            }
        }
        n += 3 + 9;
    } else if (ec == cudaSuccess) {
        ec = closure(false, 0);
    }
    if (ec == cudaSuccess && !handoff && c->psiValid) // the ansatz kernel writes psi
        ec = cudaMemsetAsync(c->psiValid, 0, sizeof(int), s0);
    if (ec == cudaSuccess)
        ec = launch_kinetic_flux(c->g, c->alpha, c->mfA, c->mfP, c->xi, c->eta, c->nq, c->qChunk,
                                 c->runLen, c->theta, 0, c->psi, handoff, c->flux, c->errorFlag,
                                 wrap ? c->mirrorFlag : nullptr, s0);
    if (ec == cudaSuccess)
        ec = launch_euler(c->g, c->u, c->flux, c->sigT, c->sigS, dt, c->numSMs, s0);
    if (ec == cudaSuccess && stage == 1)
        ec = launch_rk(c->g, c->u, c->uOld, 1, c->numSMs, s0);
    n += (handoff ? 1 + (wrap ? 1 : 2) : 2 * ceil_div(c->nq, c->qChunk)) + 1 + (stage == 1);
    *launches = n + (c->launches - l0); // the closure counted its round 0
    c->launches = l0;
    return ec;
}

// One M_N RK stage as a CUDA graph of its own, cached per configuration (stage_capture).
// *used is false when the context's options need the stage run launch by launch.
static c3d_status stage_graph(c3d_ctx *c, int stage, double dt, bool *used)
{
    *used = false;
    if (!stage_graphs_usable(c))
        return C3D_OK;
    bool handoff = false;
    c3d_status s = stage_prepare(c, &handoff);
    if (s != C3D_OK)
        return s;
    const std::vector<unsigned char> key = stage_key(c, stage, dt, handoff);
    c3d_ctx::StageGraph *Gp = nullptr;
    for (auto &g : c->sg)
        if (g.exec && g.key == key)
            Gp = &g;
    if (!Gp) {
        Gp = &c->sg[0];
        for (auto &g : c->sg)
            if (g.used < Gp->used)
                Gp = &g;
    }
    auto &G = *Gp;
    if (!G.exec || G.key != key) {
        std::lock_guard<std::mutex> lk(graph_build_mutex());
        if (G.exec) {
            // the previous graph may still run on the stream: it is destroyed once idle
            C3D_CUDA(cudaStreamSynchronize(c->stream));
            cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
        }
        cudaGraph_t top = nullptr;
        C3D_CUDA(cudaGraphCreate(&top, 0));
        long long launches = 0;
        cudaError_t e = cudaStreamBeginCaptureToGraph(c->sc[0], top, nullptr, nullptr, 0,
                                                      cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            const cudaError_t ec = stage_capture(c, stage, dt, handoff, top, c->sc, &launches);
            cudaGraph_t out = nullptr;
            e = cudaStreamEndCapture(c->sc[0], &out);
            if (e == cudaSuccess)
                e = ec;
        }
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&G.exec, top, 0);
        cudaGraphDestroy(top);
        G.launches = launches;
        if (e != cudaSuccess) {
            G.exec = nullptr;
            for (cudaStream_t &x : c->sc) {
                if (x)
                    cudaStreamDestroy(x);
                x = nullptr;
            }
            cudaGetLastError();
            return fail(C3D_ERR_CUDA, std::string("c3d_stage: stage graph: ") +
                                          cudaGetErrorString(e));
        }
        G.key = key;
    }
    G.used = ++c->sgTick;
    C3D_CUDA(cudaGraphLaunch(G.exec, c->stream));
    c->launches += G.launches;
    c->psiReady = false;
    *used = true;
    return C3D_OK;
}

c3d_status c3d_group_step(c3d_group *g, const double *dt)
{
    if (!g || !dt)
        return fail(C3D_ERR_INVALID, "c3d_group_step: bad argument");
    const int K = (int)g->ctx.size();
    for (int k = 0; k < K; ++k) {
        if (!stage_graphs_usable(g->ctx[k]))
            return fail(C3D_ERR_INVALID, "c3d_group_step: the contexts need the work-list "
                                         "engine, graphs on, timing, line log and re-projection "
                                         "off");
        if (!(dt[k] > 0.0))
            return fail(C3D_ERR_INVALID, "c3d_group_step: dt must be positive");
    }
    std::vector<unsigned char> key;
    std::vector<char> handoff(K, 0);
    for (int k = 0; k < K; ++k) {
        bool h = false;
        c3d_status s = stage_prepare(g->ctx[k], &h);
        if (s != C3D_OK)
            return s;
        handoff[k] = h;
        for (int stage = 0; stage < 2; ++stage) {
            const std::vector<unsigned char> kk = stage_key(g->ctx[k], stage, dt[k], h);
            key.insert(key.end(), kk.begin(), kk.end());
        }
    }
    if (!g->stepExec || key != g->stepKey) {
        std::lock_guard<std::mutex> lk(graph_build_mutex());
        if (g->stepExec) {
            C3D_CUDA(cudaStreamSynchronize(g->stream));
            cudaGraphExecDestroy(g->stepExec);
            g->stepExec = nullptr;
        }
        C3D_CUDA(group_streams_make(g));
        cudaStream_t o = g->cs[3 * K];
        std::vector<cudaEvent_t> ev(K + 1, nullptr);
        cudaError_t e = cudaSuccess;
        for (cudaEvent_t &x : ev)
            if (e == cudaSuccess)
                e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        cudaGraph_t top = nullptr;
        if (e == cudaSuccess)
            e = cudaGraphCreate(&top, 0);
        if (e == cudaSuccess) {
            e = cudaStreamBeginCaptureToGraph(o, top, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed);
            cudaError_t ec = e == cudaSuccess ? cudaEventRecord(ev[K], o) : e;
            // the contexts' steps one after another: each step fills the GPU with its own
            // kernels, and measured as parallel branches they ran slower than in sequence
            for (int k = 0; k < K && ec == cudaSuccess; ++k) {
                c3d_ctx *c = g->ctx[k];
                g->stepLaunches[k] = 0;
                ec = cudaStreamWaitEvent(c->sc[0], k == 0 ? ev[K] : ev[k - 1], 0);
                for (int stage = 0; stage < 2 && ec == cudaSuccess; ++stage) {
                    long long n = 0;
                    ec = stage_capture(c, stage, dt[k], handoff[k] != 0, top, c->sc, &n);
                    g->stepLaunches[k] += n;
                }
                if (ec == cudaSuccess)
                    ec = cudaEventRecord(ev[k], c->sc[0]);
            }
            if (ec == cudaSuccess)
                ec = cudaStreamWaitEvent(o, ev[K - 1], 0);
            if (e == cudaSuccess) {
                cudaGraph_t out = nullptr;
                e = cudaStreamEndCapture(o, &out);
                if (e == cudaSuccess)
                    e = ec;
            }
        }
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&g->stepExec, top, 0);
        if (top)
            cudaGraphDestroy(top);
        for (cudaEvent_t x : ev)
            if (x)
                cudaEventDestroy(x);
        if (e != cudaSuccess) {
            g->stepExec = nullptr;
            g->stepKey.clear();
            group_streams_free(g);
            for (c3d_ctx *c : g->ctx)
                for (cudaStream_t &x : c->sc) {
                    if (x)
                        cudaStreamDestroy(x);
                    x = nullptr;
                }
            cudaGetLastError();
            return fail(C3D_ERR_CUDA, std::string("c3d_group_step: group graph: ") +
                                          cudaGetErrorString(e));
        }
        g->stepKey = key;
    }
    C3D_CUDA(cudaGraphLaunch(g->stepExec, g->stream));
    for (int k = 0; k < K; ++k) {
        g->ctx[k]->launches += g->stepLaunches[k];
        g->ctx[k]->psiReady = false;
    }
    return C3D_OK;
}

c3d_status c3d_stage(c3d_ctx *c, int stage, double dt)
{
    if (!c || stage < 0 || stage > 1)
        return fail(C3D_ERR_INVALID, "c3d_stage: bad argument");
    c3d_status s;
    bool used = false;
    if ((s = stage_graph(c, stage, dt, &used)) != C3D_OK)
        return s;
    if (used)
        return C3D_OK;
    if (stage == 0) {
        C3D_CUDA(launch_rk(c->g, c->u, c->uOld, 0, c->numSMs, c->stream));
        c->launches += 1;
    }
    if ((s = c3d_ghost_fill(c)) != C3D_OK)
        return s;
    if (c->solver == 1) {
        if ((s = c3d_closure(c)) != C3D_OK)
            return s;
        if ((s = c3d_flux_kinetic(c, 0)) != C3D_OK)
            return s;
    } else if (!c->pnKinetic) {
        if ((s = c3d_flux_moment(c)) != C3D_OK)
            return s;
    } else {
        if ((s = c3d_flux_kinetic(c, 1)) != C3D_OK)
            return s;
    }
    if ((s = c3d_euler(c, dt)) != C3D_OK)
        return s;
    if (stage == 1) {
        C3D_CUDA(launch_rk(c->g, c->u, c->uOld, 1, c->numSMs, c->stream));
        c->launches += 1;
    }
    return C3D_OK;
}

// The cells of the x-slab split: x is the slowest index of the I3D layout, so each x-plane is
// a contiguous block of (ny+4)(nz+4) cells.
static c3d_status ensure_xsplit(c3d_ctx *c)
{
    if (c->xSplit[0])
        return C3D_OK;
    const long long P = (long long)c->g.nyg() * c->g.nzg();
    std::vector<int> part[2];
    part[0].reserve((size_t)(c->g.nx * P));
    part[1].reserve((size_t)(4 * P));
    for (int i = 0; i < c->g.nxg(); ++i) {
        const int w = (i < 2 || i >= c->g.nx + 2) ? 1 : 0;
        for (long long p = 0; p < P; ++p)
            part[w].push_back((int)(i * P + p));
    }
    for (int w = 0; w < 2; ++w) {
        if (cudaMalloc(&c->xSplit[w], part[w].size() * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            return fail(C3D_ERR_OOM, "c3d_stage_part: device allocation failed");
        }
        C3D_CUDA(cudaMemcpy(c->xSplit[w], part[w].data(), part[w].size() * sizeof(int),
                            cudaMemcpyHostToDevice));
        c->xSplitCount[w] = (long long)part[w].size();
    }
    return C3D_OK;
}

c3d_status c3d_stage_part(c3d_ctx *c, int stage, double dt, int part)
{
    if (!c || stage < 0 || stage > 1 || part < 0 || part > 1)
        return fail(C3D_ERR_INVALID, "c3d_stage_part: bad argument");
    if (c->solver != 1 || !c->xHaloExternal || c->engine != 0)
        return fail(C3D_ERR_INVALID, "c3d_stage_part: the split stage is for M_N slab contexts "
                                     "(c3d_set_x_halo_external) on the work-list engine");
    c3d_status s = ensure_xsplit(c);
    if (s != C3D_OK)
        return s;
    if (part == 0) {
        if (stage == 0) {
            C3D_CUDA(launch_rk(c->g, c->u, c->uOld, 0, c->numSMs, c->stream));
            c->launches += 1;
        }
        if ((s = c3d_ghost_fill(c)) != C3D_OK) // the y and z faces
            return s;
    }
    cudaEvent_t t0 = nullptr;
    timing_begin(c, &t0);
    s = run_closure(c, c->xSplitCount[part], c->u, c->alpha, c->iters, c->iterGamma, c->regIdx,
                    c->status, c->xSplit[part], true);
    if (s != C3D_OK)
        return s;
    if ((s = finish_handoff(c, false)) != C3D_OK)
        return s;
    if (part == 1) {
        if (c->lineLog && c->lineCount < c->lineCap) {
            C3D_CUDA(launch_line_log(c->g, c->cp, c->iters, c->iterGamma, c->regIdx,
                                     c->cellGamma, c->cellErr,
                                     c->lineLog + (size_t)c->lineCount * c->g.nx * 5, c->stream));
            c->lineCount++;
            c->launches += 1;
        }
        if (c->reproject) {
            C3D_CUDA(launch_reproject(c->g, c->u, c->alpha, c->mfA, c->mfP, c->nq, c->errorFlag,
                                      c->stream));
            c->launches += 1;
            psi_invalidate(c); // alpha_0 moved
        }
    }
    timing_end(c, 0, t0);
    if (part == 0)
        return C3D_OK;
    if ((s = c3d_flux_kinetic(c, 0)) != C3D_OK)
        return s;
    if ((s = c3d_euler(c, dt)) != C3D_OK)
        return s;
    if (stage == 1) {
        C3D_CUDA(launch_rk(c->g, c->u, c->uOld, 1, c->numSMs, c->stream));
        c->launches += 1;
    }
    return C3D_OK;
}

c3d_status c3d_step(c3d_ctx *c, double dt)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_step: null context");
    c3d_status s = c3d_stage(c, 0, dt);
    return s == C3D_OK ? c3d_stage(c, 1, dt) : s;
}

c3d_status c3d_set_x_halo_external(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_set_x_halo_external: null context");
    c->xHaloExternal = on != 0;
    return C3D_OK;
}

c3d_status c3d_copy_x_planes(c3d_ctx *c, int field, int i0, int count, void *buf, int toBuf,
                             int where)
{
    if (!c || !buf || field < 0 || field > 1 || count < 0 || i0 < 0 || i0 + count > c->g.nxg())
        return fail(C3D_ERR_INVALID, "c3d_copy_x_planes: bad argument");
    const size_t plane = (size_t)c->g.nyg() * c->g.nzg() * c->g.nm;
    double *a = (field == 0 ? c->u : c->alpha) + (size_t)i0 * plane;
    if (field == 1 && !toBuf) {
        c->psiReady = false;
        psi_invalidate(c);
    }
    const size_t bytes = (size_t)count * plane * sizeof(double);
    cudaMemcpyKind k = where ? cudaMemcpyDeviceToDevice
                             : (toBuf ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice);
    if (toBuf)
        C3D_CUDA(cudaMemcpyAsync(buf, a, bytes, k, c->stream));
    else
        C3D_CUDA(cudaMemcpyAsync(a, buf, bytes, k, c->stream));
    if (!where)
        C3D_CUDA(cudaStreamSynchronize(c->stream));
    return C3D_OK;
}

c3d_status c3d_sync(c3d_ctx *c)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_sync: null context");
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    int flag = 0;
    unsigned long long failed = 0;
    C3D_CUDA(cudaMemcpy(&flag, c->errorFlag, 4, cudaMemcpyDeviceToHost));
    C3D_CUDA(cudaMemcpy(&failed, c->failCount, 8, cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset(c->errorFlag, 0, 4);
        return fail(C3D_ERR_TIMEOUT, flag == 2 ? "closure: round limit exceeded"
                                               : "a bounded device wait gave up");
    }
    if (failed) {
        cudaMemset(c->failCount, 0, 8);
        return fail(C3D_ERR_CLOSURE, std::to_string(failed) +
                                         " cell(s) failed: u0 <= 0 or regularisation ladder exhausted");
    }
    return C3D_OK;
}

c3d_status c3d_closure_records(c3d_ctx *c, int *iters, int *iterGamma, int *regIndex, int *status)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_closure_records: null context");
    const size_t b = c->g.nall() * 4;
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    if (iters)
        C3D_CUDA(cudaMemcpy(iters, c->iters, b, cudaMemcpyDeviceToHost));
    if (iterGamma)
        C3D_CUDA(cudaMemcpy(iterGamma, c->iterGamma, b, cudaMemcpyDeviceToHost));
    if (regIndex)
        C3D_CUDA(cudaMemcpy(regIndex, c->regIdx, b, cudaMemcpyDeviceToHost));
    if (status)
        C3D_CUDA(cudaMemcpy(status, c->status, b, cudaMemcpyDeviceToHost));
    return C3D_OK;
}

c3d_status c3d_closure_records_fp(c3d_ctx *c, double *gamma, double *normG)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_closure_records_fp: null context");
    const size_t b = c->g.nall() * 8;
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    if (gamma)
        C3D_CUDA(cudaMemcpy(gamma, c->cellGamma, b, cudaMemcpyDeviceToHost));
    if (normG)
        C3D_CUDA(cudaMemcpy(normG, c->cellErr, b, cudaMemcpyDeviceToHost));
    return C3D_OK;
}

c3d_status c3d_line_stats_enable(c3d_ctx *c, int maxClosures)
{
    if (!c || maxClosures < 0)
        return fail(C3D_ERR_INVALID, "c3d_line_stats_enable: bad argument");
    psi_invalidate(c); // the closure may no longer hand its ansatz over
    if (c->lineLog) {
        cudaFree(c->lineLog);
        c->lineLog = nullptr;
    }
    c->lineCap = c->lineCount = 0;
    if (maxClosures == 0)
        return C3D_OK;
    C3D_CUDA(cudaMalloc(&c->lineLog, (size_t)maxClosures * c->g.nx * 5 * sizeof(double)));
    c->lineCap = maxClosures;
    return C3D_OK;
}

c3d_status c3d_line_stats_get(c3d_ctx *c, double *out, int *count)
{
    if (!c || !count)
        return fail(C3D_ERR_INVALID, "c3d_line_stats_get: null argument");
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    *count = c->lineCount;
    if (out && c->lineCount)
        C3D_CUDA(cudaMemcpy(out, c->lineLog, (size_t)c->lineCount * c->g.nx * 5 * sizeof(double),
                            cudaMemcpyDeviceToHost));
    return C3D_OK;
}

int c3d_timing_events(c3d_ctx *c, int *kinds, double *ms, int maxEvents)
{
    if (!c)
        return -1;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
        return -1;
    int n = 0;
    for (auto &e : c->events) {
        if (n >= maxEvents)
            break;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, e.second.first, e.second.second) != cudaSuccess)
            return -1;
        if (kinds)
            kinds[n] = e.first;
        if (ms)
            ms[n] = t;
        ++n;
    }
    return n;
}

c3d_status c3d_closure_stats_get(c3d_ctx *c, c3d_closure_stats *st)
{
    if (!c || !st)
        return fail(C3D_ERR_INVALID, "c3d_closure_stats_get: null argument");
    unsigned long long h[STAT_COUNT];
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    C3D_CUDA(cudaMemcpy(h, c->stats, sizeof(h), cudaMemcpyDeviceToHost));
    memset(st, 0, sizeof(*st));
    st->cells = (long long)h[STAT_CELLS];
    st->totalIters = (long long)h[STAT_ITERS];
    st->totalIterGamma = (long long)h[STAT_ITER_GAMMA];
    st->maxIter = (int)h[STAT_MAX_ITER];
    st->maxIterGamma = (int)h[STAT_MAX_ITER_GAMMA];
    st->failed = (long long)h[STAT_FAILED];
    st->trials = (long long)h[STAT_TRIALS];
    st->clkRefill = (long long)h[STAT_CLK_REFILL];
    st->clkPass = (long long)h[STAT_CLK_PASS];
    st->clkSerial = (long long)h[STAT_CLK_SERIAL];
    st->passes = (long long)h[STAT_PASSES];
    for (int i = 0; i < 16; ++i)
        st->regHist[i] = (long long)h[STAT_REG_HIST + i];
    for (int i = 0; i < 64; ++i)
        st->iterHist[i] = (long long)h[STAT_ITER_HIST + i];
    for (int i = 0; i < 8; ++i)
        st->clkNewton[i] = (long long)h[STAT_CLK_NEWTON + i];
    st->hessBf16 = (long long)h[STAT_H_BF16];
    st->hessTf32x3 = (long long)h[STAT_H_TF32X3];
    st->hessFp64 = (long long)h[STAT_H_FP64];
    st->escalated = (long long)h[STAT_ESCALATED];
    st->certified = (long long)h[STAT_CERTIFIED];
    st->hostSyncs = c->hostSyncs;
    return C3D_OK;
}

c3d_status c3d_closure_stats_reset(c3d_ctx *c)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_closure_stats_reset: null context");
    C3D_CUDA(cudaMemsetAsync(c->stats, 0, STAT_COUNT * 8, c->stream));
    return C3D_OK;
}

long long c3d_launch_count(c3d_ctx *c)
{
    if (!c)
        return 0;
    unsigned long long dev = 0;
    if (c->launchDev) {
        cudaStreamSynchronize(c->stream);
        cudaMemcpy(&dev, c->launchDev, sizeof(dev), cudaMemcpyDeviceToHost);
    }
    return c->launches + (long long)dev;
}

c3d_status c3d_timing_enable(c3d_ctx *c, int on)
{
    if (!c)
        return fail(C3D_ERR_INVALID, "c3d_timing_enable: null context");
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    timing_clear(c);
    c->timing = on != 0;
    return C3D_OK;
}

c3d_status c3d_timing_get(c3d_ctx *c, double *ms, long long *count)
{
    if (!c || !ms)
        return fail(C3D_ERR_INVALID, "c3d_timing_get: null argument");
    C3D_CUDA(cudaStreamSynchronize(c->stream));
    ms[0] = ms[1] = 0.0;
    long long n[2] = {0, 0};
    for (auto &e : c->events) {
        if (e.first > 1)
            continue;
        float t = 0.f;
        C3D_CUDA(cudaEventElapsedTime(&t, e.second.first, e.second.second));
        ms[e.first] += t;
        n[e.first]++;
    }
    if (count) {
        count[0] = n[0];
        count[1] = n[1];
    }
    return C3D_OK;
}

// ---------------------------------------------------------------- reference GPU entry points
// Process-wide state, as the reference keeps it (static device buffers set up on
// first use, src/cuda/cuda_flux_kinetic.cu:23-67, src/cuda/cuda_solveH.cu).

static std::mutex g_refMutex;
static struct {
    int nm = 0, nq = 0, nchunks = 0;
    double *chunks = nullptr, *alphas = nullptr, *hs = nullptr;
    long long cap = 0; // batch buffers hold cap vectors of up to capNm moments
    int capNm = 0;
    int *errorFlag = nullptr;
    // Gaunt form (solveHInit_cuda with useGaunt): staged chunks of M^T, M2^T and the weights,
    // dense beta transposed (betaT[k nm^2 + i nm + j]) and the CSR table of |beta| > 1e-13
    int nm2 = 0, nm2p = 0, gnchunks = 0;
    double *gchunks = nullptr, *betaT = nullptr, *betaVal = nullptr;
    int *betaRow = nullptr, *betaCol = nullptr;
} g_h;

static void ref_free(void *&p)
{
    if (p)
        cudaFree(p);
    p = nullptr;
}

// Host staging for a device table; returns false (and prints) on a CUDA error.
static bool ref_upload(void **dst, const void *src, size_t bytes, const char *what)
{
    void *d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes > 0 ? bytes : 1);
    if (e == cudaSuccess && bytes > 0)
        e = cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (d)
            cudaFree(d);
        cudaGetLastError();
        fprintf(stderr, "[c3d_b200] solveHInit_cuda: %s: %s\n", what, cudaGetErrorString(e));
        return false;
    }
    *dst = d;
    return true;
}

void solveHInit_cuda(int nm, int nm2, int nq, int batchSize, double *w, double *p, double *p2,
                     double *beta, double *betaVal, int *betaColInd, int *betaRowPtr, int useGaunt)
{
    std::lock_guard<std::mutex> lk(g_refMutex);
    if (nm < 1 || nm > 64 || nq < 1 || !w || !p) {
        fprintf(stderr, "[c3d_b200] solveHInit_cuda: unsupported sizes nm=%d nq=%d\n", nm, nq);
        return;
    }
    // direct form: chunks of M^T and the weights
    std::vector<double> ch = build_chunks(nm, nq, p, w);
    ref_free((void *&)g_h.chunks);
    g_h.nm = g_h.nq = 0;
    if (!ref_upload((void **)&g_h.chunks, ch.data(), ch.size() * 8, "basis"))
        return;
    g_h.nchunks = ceil_div(nq, QC);
    if (!g_h.errorFlag) {
        if (cudaMalloc(&g_h.errorFlag, 4) != cudaSuccess || cudaMemset(g_h.errorFlag, 0, 4) != cudaSuccess) {
            cudaGetLastError();
            g_h.errorFlag = nullptr;
            fprintf(stderr, "[c3d_b200] solveHInit_cuda: device allocation failed\n");
            return;
        }
    }
    long long cap = batchSize > 0 ? batchSize : 1;
    if (cap > g_h.cap || nm > g_h.capNm) {
        ref_free((void *&)g_h.alphas);
        ref_free((void *&)g_h.hs);
        g_h.cap = 0;
        g_h.capNm = 0;
        if (cudaMalloc(&g_h.alphas, cap * nm * 8) != cudaSuccess ||
            cudaMalloc(&g_h.hs, cap * nm * nm * 8) != cudaSuccess) {
            cudaGetLastError();
            ref_free((void *&)g_h.alphas);
            ref_free((void *&)g_h.hs);
            fprintf(stderr, "[c3d_b200] solveHInit_cuda: device allocation of the batch failed\n");
            return;
        }
        g_h.cap = cap;
        g_h.capNm = nm;
    }
    // Gaunt form (src/cuda/cuda_solveH.cu:44-104 takes the same tables)
    ref_free((void *&)g_h.gchunks);
    ref_free((void *&)g_h.betaT);
    ref_free((void *&)g_h.betaVal);
    ref_free((void *&)g_h.betaRow);
    ref_free((void *&)g_h.betaCol);
    g_h.nm2 = g_h.nm2p = g_h.gnchunks = 0;
    if (useGaunt) {
        const int nm2p = 8 * ceil_div(nm2, 8);
        if (nm2 < 1 || !p2 || gaunt_batch_smem(nm, nm2p) == 0) {
            fprintf(stderr, "[c3d_b200] solveHInit_cuda: unsupported Gaunt sizes nm=%d nm2=%d\n",
                    nm, nm2);
            return;
        }
        const int rows = nm + nm2p + 1, nch = ceil_div(nq, QC);
        std::vector<double> gch((size_t)nch * rows * QCP, 0.0);
        for (int k = 0; k < nch; ++k)
            for (int qq = 0; qq < QC && k * QC + qq < nq; ++qq) {
                const int q = k * QC + qq;
                double *c = gch.data() + (size_t)k * rows * QCP;
                for (int i = 0; i < nm; ++i)
                    c[i * QCP + qq] = p[(size_t)q * nm + i];
                for (int i = 0; i < nm2; ++i)
                    c[(nm + i) * QCP + qq] = p2[(size_t)q * nm2 + i];
                c[(nm + nm2p) * QCP + qq] = w[q];
            }
        if (!ref_upload((void **)&g_h.gchunks, gch.data(), gch.size() * 8, "Gaunt basis"))
            return;
        if (beta) {
            const size_t nmm = (size_t)nm * nm;
            std::vector<double> bt(nmm * nm2);
            for (size_t ij = 0; ij < nmm; ++ij)
                for (int k = 0; k < nm2; ++k)
                    bt[(size_t)k * nmm + ij] = beta[ij * nm2 + k];
            if (!ref_upload((void **)&g_h.betaT, bt.data(), bt.size() * 8, "dense beta"))
                return;
        }
        if (betaVal && betaColInd && betaRowPtr) {
            const int nnz = betaRowPtr[nm * nm];
            if (!ref_upload((void **)&g_h.betaRow, betaRowPtr, (size_t)(nm * nm + 1) * 4, "beta rows") ||
                !ref_upload((void **)&g_h.betaCol, betaColInd, (size_t)nnz * 4, "beta columns") ||
                !ref_upload((void **)&g_h.betaVal, betaVal, (size_t)nnz * 8, "beta values"))
                return;
        }
        g_h.nm2 = nm2;
        g_h.nm2p = nm2p;
        g_h.gnchunks = nch;
    }
    g_h.nm = nm;
    g_h.nq = nq;
}

// Fills hs with NaN so that a failed call cannot pass for a computed batch.
static void ref_poison(double *hs, long long count)
{
    if (hs && count > 0)
        std::fill(hs, hs + count, std::nan(""));
}

void solveH_cuda(int nm, int nm2, int nq, int batchSize, double *alphas, double *hs, int useGaunt,
                 int useGauntSparse)
{
    std::lock_guard<std::mutex> lk(g_refMutex);
    const long long count = batchSize > 0 ? (long long)batchSize * nm * nm : 0;
    if (batchSize <= 0)
        return;
    bool ready = g_h.chunks && nm == g_h.nm && nq == g_h.nq && batchSize <= g_h.cap && alphas && hs;
    if (ready && useGaunt)
        ready = g_h.gchunks && nm2 == g_h.nm2 && (useGauntSparse ? g_h.betaVal != nullptr
                                                                 : g_h.betaT != nullptr);
    if (!ready) {
        fprintf(stderr, "[c3d_b200] solveH_cuda: not initialised for nm=%d nm2=%d nq=%d batch=%d "
                        "useGaunt=%d sparse=%d (call solveHInit_cuda with the same sizes and "
                        "tables); hs set to NaN\n",
                nm, nm2, nq, batchSize, useGaunt, useGauntSparse);
        ref_poison(hs, count);
        return;
    }
    cudaError_t e = cudaMemcpy(g_h.alphas, alphas, (size_t)batchSize * nm * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (useGaunt)
            e = launch_gaunt_batch(nm, g_h.nm2, g_h.nm2p, g_h.gnchunks, g_h.gchunks, g_h.alphas,
                                   batchSize, g_h.betaT, g_h.betaRow, g_h.betaCol, g_h.betaVal,
                                   useGauntSparse ? 1 : 0, g_h.hs, g_h.errorFlag, 0);
        else
            e = launch_hessian_batch(nm, g_h.nchunks, g_h.chunks, g_h.alphas, batchSize, g_h.hs,
                                     g_h.errorFlag, 0);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(hs, g_h.hs, (size_t)count * 8, cudaMemcpyDeviceToHost);
    int flag = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(&flag, g_h.errorFlag, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "[c3d_b200] solveH_cuda: %s; hs set to NaN\n", cudaGetErrorString(e));
        ref_poison(hs, count);
        return;
    }
    if (flag) {
        cudaMemset(g_h.errorFlag, 0, 4);
        fprintf(stderr, "[c3d_b200] solveH_cuda: a bounded device wait gave up; hs set to NaN\n");
        ref_poison(hs, count);
    }
}

static struct {
    c3d_ctx *ctx = nullptr;
    int nx = 0, ny = 0, nz = 0, nm = 0, nq = 0, isPn = -1;
    double dx = 0.0, dy = 0.0, dz = 0.0;
} g_f;

void solveFluxKinetic_cuda(int nx, int ny, int nz, int nm, int nq, double dx, double dy, double dz,
                           double *alpha, double *flux, double *xi, double *eta, double *mu,
                           double *w, double *p, int isPn)
{
    std::lock_guard<std::mutex> lk(g_refMutex);
    if (nx < 5 || ny < 5 || nz < 5) {
        fprintf(stderr, "[c3d_b200] solveFluxKinetic_cuda: grid (with ghosts) too small\n");
        return;
    }
    // the flux fragments carry cosine x weight / spacing: a new spacing needs a new context
    if (!g_f.ctx || g_f.nx != nx || g_f.ny != ny || g_f.nz != nz || g_f.nm != nm || g_f.nq != nq ||
        g_f.isPn != isPn || g_f.dx != dx || g_f.dy != dy || g_f.dz != dz) {
        if (g_f.ctx)
            c3d_destroy(g_f.ctx);
        g_f.ctx = nullptr;
        c3d_params P{};
        P.nx = nx - 4;
        P.ny = ny - 4;
        P.nz = nz - 4;
        P.nm = nm;
        P.nq = nq;
        P.dx = dx;
        P.dy = dy;
        P.dz = dz;
        P.theta = 2.0; // the reference's GPU flux hard-codes theta (src/cuda/cuda_flux_kinetic.cu:82)
        P.solver = isPn ? 0 : 1;
        P.pnUseKineticFlux = 1;
        P.mnBatched = 1;
        P.mnMaxIter = 100;
        P.mnTol = 1e-8;
        P.mnTolGamma = 1.1;
        P.mnCondHMax = 1e10;
        P.nreg = 1;
        if (c3d_create(&P, p, w, xi, eta, mu, nullptr, nullptr, &g_f.ctx) != C3D_OK) {
            fprintf(stderr, "[c3d_b200] solveFluxKinetic_cuda: %s\n", c3d_last_error());
            g_f.ctx = nullptr;
            return;
        }
        g_f.nx = nx; g_f.ny = ny; g_f.nz = nz; g_f.nm = nm; g_f.nq = nq; g_f.isPn = isPn;
        g_f.dx = dx; g_f.dy = dy; g_f.dz = dz;
    }
    c3d_ctx *c = g_f.ctx;
    size_t vb = c->g.nall() * nm * 8;
    cudaMemcpyAsync(c->alpha, alpha, vb, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(c->flux, 0, vb, c->stream);
    if (c3d_flux_kinetic(c, 0) != C3D_OK) {
        fprintf(stderr, "[c3d_b200] solveFluxKinetic_cuda: %s\n", c3d_last_error());
        return;
    }
    cudaMemcpyAsync(flux, c->flux, vb, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess)
        fprintf(stderr, "[c3d_b200] solveFluxKinetic_cuda: %s\n", cudaGetErrorString(e));
}

} // extern "C"
