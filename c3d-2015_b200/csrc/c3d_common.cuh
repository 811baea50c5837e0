// Shared device-side definitions for the B200 M_N step kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace c3d {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int MAX_REG = 16;

// Quadrature chunk staged per bulk copy: QC directions, row stride QCP doubles
// (QCP = QC + 4 keeps the 8x4 DMMA fragment loads and the lane-per-direction
// exponent loads free of shared-memory bank conflicts).
constexpr int QC = 32;
constexpr int QCP = 36;

// Per-cell status codes written by the closure (0 = converged).
enum CellStatus : int {
    CELL_OK = 0,
    CELL_NONPOSITIVE_U0 = 1,   // u0 <= 0 (reference aborts, src/opt/opt.cpp:343-346)
    CELL_LADDER_EXHAUSTED = 2, // "Max regularization achieved" (src/opt/opt.cpp:261-266)
    CELL_PASS_BUDGET = 3,      // safety bound on passes per cell exceeded
};

// Layout of the device-side closure counters (accumulated until reset).
enum StatSlot : int {
    STAT_CELLS = 0,
    STAT_ITERS = 1,
    STAT_ITER_GAMMA = 2,
    STAT_MAX_ITER = 3,
    STAT_MAX_ITER_GAMMA = 4,
    STAT_FAILED = 5,
    STAT_TRIALS = 6,     // line-search trial passes
    STAT_CERTIFIED = 7,  // first visits ended by the probe's convergence certificate
    STAT_REG_HIST = 8,   // 16 bins
    STAT_CLK_REFILL = 24, // SM clocks summed over warps: queue refill + cell set-up
    STAT_CLK_PASS = 25,   // passes over the staged basis
    STAT_CLK_SERIAL = 26, // per-cell Newton logic after each pass
    STAT_PASSES = 27,     // passes (per CTA)
    STAT_H_BF16 = 28,     // mixed-precision closure: Hessian visits with BF16 moments,
    STAT_H_TF32X3 = 29,   //   with 3xTF32 split moments,
    STAT_H_FP64 = 30,     //   with FP64 moments,
    STAT_ESCALATED = 31,  //   and visits redone in FP64 (factorisation failed or non-finite)
    STAT_ITER_HIST = 32, // 64 bins (last: >= 63)
    STAT_CLK_NEWTON = 96, // 8 slots, builds with C3D_NEWTON_CLOCKS only: SM clocks of the
                          // work-list Newton kernel's phases (c3d_closure_stats.clkNewton)
    STAT_COUNT = 104,
};

// Closure options (the MN_* deck keys, src/init.cpp:252-258).
struct ClosureParams {
    int nm;          // moments
    int nq;          // quadrature points
    int nchunks;     // ceil(nq / QC)
    int batched;     // 1: src/opt/optBatch.cpp rules; 0: src/opt/opt.cpp rules
    int maxIter;
    int nreg;
    double tol;
    double tolGamma; // 1.1 for the unbatched rules (src/update.cpp:57)
    double condHMax;
    double reg[MAX_REG];
    long long passBudget; // safety bound on H/line-search passes per cell
    // mixed-precision closure (work-list engine, Gaunt form): the Hessian's extended moments
    // in BF16 (condition estimate <= condBf16) or 3xTF32 split products (<= condMixMax) with
    // FP32 accumulation; FP64 moments beyond, after mixIterMax iterations at one
    // regularisation level, and for the rest of the closure once a reduced-precision
    // factorisation fails. Gradient, objective and line search stay FP64.
    int mixed;
    int mixIterMax;
    double condBf16;
    double condMixMax;
    double mixPolish;  // > 0: a reduced-precision visit whose gradient norm lies in
                       // (rtol, mixPolish * rtol] is redone with FP64 moments, so that the
                       // steps that end the iteration are FP64 Newton steps
    // convergence certificate of a cell's first Hessian visit (work-list engine, Gaunt form):
    // a probe pass computes the first-order moments and the extreme values of e^{alpha.m}
    // over the quadrature; H >= e_min G with G = sum_q w_q m_q m_q^T, whose eigenvalues lie
    // in [gramLo, gramHi] (Gershgorin), bounds the condition estimate and |d| = |H^-1 g|,
    // so a cell whose visit would end converged is finalized without H (see after_probe)
    int probe;
    double gramLo, gramHi;
};

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// One entry of the Gaunt-form Hessian assembly stream (src/opt/fobj.cpp:81-99): the
// running H element += v * moment[col] (col = -1: the element is 1, an identity padding
// slot); slot >= 0 ends tile slot `slot`, which then receives the element.
struct __align__(16) GauntTerm {
    double v;
    int col;
    int slot;
};

// Threads of the work-list Newton kernel (4 cells of one warp each); the Gaunt assembly
// streams are laid out for this many threads.
constexpr int NEWTON_THREADS = 128;

// Grid with two ghost layers per face; cell (i,j,k) with k fastest (src/global.h:15).
struct GridDims {
    int nx, ny, nz; // interior cells
    int nm;
    __host__ __device__ int nxg() const { return nx + 4; }
    __host__ __device__ int nyg() const { return ny + 4; }
    __host__ __device__ int nzg() const { return nz + 4; }
    __host__ __device__ long long cell(int i, int j, int k) const
    {
        return (long long)k + (long long)nzg() * ((long long)j + (long long)nyg() * i);
    }
    __host__ __device__ long long nall() const { return (long long)nxg() * nyg() * nzg(); }
    __host__ __device__ long long ninterior() const { return (long long)nx * ny * nz; }
};

// Interior-cell index (k fastest) -> grid cell index.
__host__ __device__ inline long long interior_cell(const GridDims &g, long long n)
{
    int k = (int)(n % g.nz);
    long long r = n / g.nz;
    int j = (int)(r % g.ny);
    int i = (int)(r / g.ny);
    return g.cell(i + 2, j + 2, k + 2);
}

// Face ghost cells: 2 layers per face over the interior ranges of the other two axes (no
// edges or corners), f in [0, 4 (ny nz + nx nz + nx ny)). dst is the ghost cell, src its
// periodic image inside the domain (src/comm.cpp:281-323).
__host__ __device__ inline long long ghost_faces(const GridDims &g)
{
    return 4LL * g.ny * g.nz + 4LL * g.nx * g.nz + 4LL * g.nx * g.ny;
}
__host__ __device__ inline void ghost_pair(const GridDims &g, long long f, long long &dst,
                                           long long &src)
{
    const long long fx = 4LL * g.ny * g.nz, fy = 4LL * g.nx * g.nz;
    if (f < fx) {
        int side = (int)(f / (2LL * g.ny * g.nz)); // 0: low ghosts, 1: high ghosts
        long long r = f % (2LL * g.ny * g.nz);
        int l = (int)(r / ((long long)g.ny * g.nz));
        long long r2 = r % ((long long)g.ny * g.nz);
        int j = 2 + (int)(r2 / g.nz), k = 2 + (int)(r2 % g.nz);
        dst = side == 0 ? g.cell(l, j, k) : g.cell(g.nx + 2 + l, j, k);
        src = side == 0 ? g.cell(g.nx + l, j, k) : g.cell(2 + l, j, k);
    } else if (f < fx + fy) {
        f -= fx;
        int side = (int)(f / (2LL * g.nx * g.nz));
        long long r = f % (2LL * g.nx * g.nz);
        int l = (int)(r / ((long long)g.nx * g.nz));
        long long r2 = r % ((long long)g.nx * g.nz);
        int i = 2 + (int)(r2 / g.nz), k = 2 + (int)(r2 % g.nz);
        dst = side == 0 ? g.cell(i, l, k) : g.cell(i, g.ny + 2 + l, k);
        src = side == 0 ? g.cell(i, g.ny + l, k) : g.cell(i, 2 + l, k);
    } else {
        f -= fx + fy;
        int side = (int)(f / (2LL * g.nx * g.ny));
        long long r = f % (2LL * g.nx * g.ny);
        int l = (int)(r / ((long long)g.nx * g.ny));
        long long r2 = r % ((long long)g.nx * g.ny);
        int i = 2 + (int)(r2 / g.ny), j = 2 + (int)(r2 % g.ny);
        dst = side == 0 ? g.cell(i, j, l) : g.cell(i, j, g.nz + 2 + l);
        src = side == 0 ? g.cell(i, j, g.nz + l) : g.cell(i, j, 2 + l);
    }
}


} // namespace c3d
