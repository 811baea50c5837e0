// Allocation-free standalone closure (c3d_closure_vectors_noalloc, include/c3d_b200.h).
//
// Some callers cannot call cudaMalloc: an application that hands this library
// device memory out of its own pre-reserved pool (so that a stray cudaMalloc
// either fails for lack of free memory or breaks the application's accounting),
// or a caller on a latency-critical path that must not risk the implicit
// device-wide synchronisation cudaMalloc/cudaFree may perform. For them this
// entry point solves n independent moment vectors with the persistent FP64
// closure kernel while allocating nothing: the caller passes every input and
// output, and the kernel's scratch -- the work-queue counter, the failure and
// statistics counters and the chunked copy of the quadrature basis that the
// kernel bulk-copies into shared memory -- lives in the file-scope array below.
//
// The array is C3D_NOALLOC_SCRATCH_BYTES (1.15 MiB) per GPU; every GPU that loads
// the library holds it until the process exits. It bounds the sizes this entry
// point accepts: nm <= 64 moments and nq <= 2048 directions.
//
// All calls share the one array and it keeps the last call's contents: each call
// clears the counters it needs and rewrites the basis table before its kernel.
// Calls that overlap on the GPU (for example on two streams) race on the array;
// callers must order them, e.g. by issuing them on one stream.
#include "../../include/c3d_b200.h"
#include "c3d_common.cuh"

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

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
void set_last_error(const std::string &msg); // reported by c3d_last_error (api.cu)
} // namespace c3d

using namespace c3d;

namespace {

constexpr int NOALLOC_MAX_NM = 64;
constexpr int NOALLOC_MAX_NQ = 2048;
constexpr size_t NOALLOC_HEADER = 4096;                          // counters
constexpr size_t NOALLOC_CHUNK_MAX = (size_t)(64 + 1) * QCP * 8; // one basis chunk at nm = 64
constexpr size_t NOALLOC_BYTES =
    NOALLOC_HEADER + (size_t)((NOALLOC_MAX_NQ + QC - 1) / QC) * NOALLOC_CHUNK_MAX;
static_assert(NOALLOC_BYTES == C3D_NOALLOC_SCRATCH_BYTES, "header and implementation disagree");

// Header layout (byte offsets): counter, failCount, errorFlag, statistics.
constexpr size_t OFF_COUNTER = 0, OFF_FAIL = 8, OFF_ERROR = 16, OFF_STATS = 64;
constexpr size_t OFF_CHUNKS = NOALLOC_HEADER;

} // namespace

// The scratch array. Host code must not use its name as an address: it is looked up
// once per device with cudaGetSymbolAddress (noalloc_scratch_ptr below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Chunked, transposed basis in the layout the closure kernel bulk-copies (the same as
// build_chunks in api.cu, but built on the device from the caller's M and w).
__global__ void noalloc_build_chunks(int nm, int nmp, int nq, int nchunks,
                                     const double *__restrict__ M, const double *__restrict__ w,
                                     double *__restrict__ chunks)
{
    const long long per = (long long)(nmp + 1) * QCP;
    const long long total = per * nchunks;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int k = (int)(e / per);
        int r = (int)((e % per) / QCP), qq = (int)(e % QCP);
        int q = k * QC + qq;
        double v = 0.0;
        if (qq < QC && q < nq) {
            if (r < nm)
                v = M[(long long)q * nm + r];
            else if (r == nmp)
                v = w[q];
        }
        chunks[e] = v;
    }
}

namespace {

std::mutex g_mu;
void *g_ptr[64];      // per device: device address of g_noalloc_scratch
int g_sms[64];

// Set-up on first use per device, with that device current: the symbol's device
// address (a plain cudaGetSymbolAddress; it allocates nothing).
c3d_status noalloc_scratch_ptr(unsigned char **out, int *numSMs)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_last_error("c3d_closure_vectors_noalloc: no usable current device");
        return C3D_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("c3d_closure_vectors_noalloc: cudaGetSymbolAddress: ") +
                    cudaGetErrorString(e));
            return C3D_ERR_CUDA;
        }
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_ptr[dev] = p;
        g_sms[dev] = sms > 0 ? sms : 1;
    }
    *out = static_cast<unsigned char *>(g_ptr[dev]);
    *numSMs = g_sms[dev];
    return C3D_OK;
}

} // namespace

extern "C" {

c3d_status c3d_closure_vectors_noalloc(int nm, int nq, const double *M, const double *w,
                                       long long n, double *u, double *alpha, int *iters,
                                       int *status, const c3d_closure_opts *opts, void *stream)
{
    if (!M || !w || !u || !alpha || !opts || n < 0) {
        set_last_error("c3d_closure_vectors_noalloc: null pointer or negative count");
        return C3D_ERR_INVALID;
    }
    if (nm < 1 || nm > NOALLOC_MAX_NM || nq < 1 || nq > NOALLOC_MAX_NQ) {
        set_last_error("c3d_closure_vectors_noalloc: nm must be in [1, 64] and nq in [1, 2048] (the "
                "static scratch holds the basis for at most these sizes)");
        return C3D_ERR_INVALID;
    }
    if (opts->nreg < 1 || opts->nreg > MAX_REG) {
        set_last_error("c3d_closure_vectors_noalloc: ladder length must be in [1, 16]");
        return C3D_ERR_INVALID;
    }
    // Without these checks a cell would run to the pass budget (maxIter < 1) or never meet
    // its stopping test (tol <= 0), and the caller would only see status -1 or 3.
    auto positive = [](double v) { return std::isfinite(v) && v > 0.0; };
    if (opts->maxIter < 1 || !positive(opts->tol) || !positive(opts->condHMax) ||
        (opts->batched && !positive(opts->tolGamma))) {
        set_last_error("c3d_closure_vectors_noalloc: maxIter must be >= 1 and tol, tolGamma and "
                       "condHMax positive and finite");
        return C3D_ERR_INVALID;
    }
    if (n == 0)
        return C3D_OK;
    unsigned char *base = nullptr;
    int numSMs = 1;
    c3d_status s = noalloc_scratch_ptr(&base, &numSMs);
    if (s != C3D_OK)
        return s;
    cudaStream_t st = (cudaStream_t)stream;
    const int nmp = closure_fp64_nmp(nm);
    const int nchunks = ceil_div(nq, QC);
    double *chunks = reinterpret_cast<double *>(base + OFF_CHUNKS);

    ClosureParams P{};
    P.nm = nm;
    P.nq = nq;
    P.nchunks = nchunks;
    P.batched = opts->batched ? 1 : 0;
    P.maxIter = opts->maxIter;
    P.nreg = opts->nreg;
    P.tol = opts->tol;
    P.tolGamma = opts->batched ? opts->tolGamma : 1.1;
    P.condHMax = opts->condHMax;
    for (int i = 0; i < opts->nreg; ++i)
        P.reg[i] = opts->reg[i];
    P.passBudget = 1LL << 40;

    // start from zero: failure count, error flag and statistics (the work counter is
    // reset by the closure launch itself); unsolved cells report status -1
    cudaError_t e = cudaMemsetAsync(base + OFF_FAIL, 0, OFF_CHUNKS - OFF_FAIL, st);
    if (e == cudaSuccess && status)
        e = cudaMemsetAsync(status, 0xff, (size_t)n * sizeof(int), st);
    if (e == cudaSuccess) {
        long long total = (long long)(nmp + 1) * QCP * nchunks;
        int blocks = (int)((total + 255) / 256);
        noalloc_build_chunks<<<blocks, 256, 0, st>>>(nm, nmp, nq, nchunks, M, w, chunks);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        ClosureLaunch L{};
        L.P = &P;
        L.chunks = chunks;
        L.ncells = n;
        L.counter = reinterpret_cast<unsigned long long *>(base + OFF_COUNTER);
        L.u = u;
        L.alpha = alpha;
        L.iters = iters;
        L.iterGamma = nullptr;
        L.regIdx = nullptr;
        L.status = status;
        L.failCount = reinterpret_cast<unsigned long long *>(base + OFF_FAIL);
        L.stats = reinterpret_cast<unsigned long long *>(base + OFF_STATS);
        L.errorFlag = reinterpret_cast<int *>(base + OFF_ERROR);
        L.numSMs = numSMs;
        L.stream = st;
        e = launch_closure_fp64(L);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("c3d_closure_vectors_noalloc: ") + cudaGetErrorString(e));
        return C3D_ERR_CUDA;
    }
    return C3D_OK;
}

// Outcome of the last c3d_closure_vectors_noalloc call on this device: synchronises the
// stream, then reads the kernel's error flag and failure count out of the static array
// (cudaMemcpyFromSymbol into host variables; nothing is allocated) and clears both.
c3d_status c3d_closure_vectors_noalloc_check(void *stream, long long *failed)
{
    if (failed)
        *failed = 0;
    unsigned char *base = nullptr;
    int numSMs = 1;
    c3d_status s = noalloc_scratch_ptr(&base, &numSMs);
    if (s != C3D_OK)
        return s;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    int flag = 0;
    unsigned long long nfail = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyFromSymbol(&flag, g_noalloc_scratch, sizeof(int), OFF_ERROR,
                                 cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpyFromSymbol(&nfail, g_noalloc_scratch, sizeof(nfail), OFF_FAIL,
                                 cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && (flag || nfail)) {
        const unsigned char zero[16] = {};
        e = cudaMemcpyToSymbol(g_noalloc_scratch, zero, sizeof(zero), OFF_FAIL,
                               cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("c3d_closure_vectors_noalloc_check: ") + cudaGetErrorString(e));
        return C3D_ERR_CUDA;
    }
    if (failed)
        *failed = (long long)nfail;
    if (flag) {
        set_last_error("c3d_closure_vectors_noalloc: a bounded device wait gave up; cells whose "
                       "status is -1 were not solved");
        return C3D_ERR_TIMEOUT;
    }
    if (nfail) {
        set_last_error("c3d_closure_vectors_noalloc: " + std::to_string(nfail) +
                       " cell(s) failed: u0 <= 0 or regularisation ladder exhausted");
        return C3D_ERR_CLOSURE;
    }
    return C3D_OK;
}

} // extern "C"
