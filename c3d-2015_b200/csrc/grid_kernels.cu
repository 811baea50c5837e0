// Grid kernels of the M_N / P_N time step:
//   ghost fill        src/comm.cpp:281-323 (serial periodic communicateBoundaries)
//   kinetic flux      src/flux_kinetic.cpp:20-198
//   P_N moment flux   src/flux_moment.cpp:15-104
//   Euler stage       src/update.cpp:21-37
//   RK copy / average src/update.cpp:206-212, :268-274
//
// Layout: the reference's, cell-major with the moment index fastest, cells
// (i,j,k) with k fastest and two ghost layers per face; arrays cover all
// (nx+4)(ny+4)(nz+4) cells.
//
// Elementwise stages (ghost fill, Euler, average) reproduce the reference's
// arithmetic bit for bit (unfused operations in its order). The kinetic flux runs its
// two contractions (exponents alpha.m_q, projection onto the moments) on the FP64 tensor
// pipe, so its sums are reordered against the reference's (agreement to ~1e-15 relative).
#include "c3d_common.cuh"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace c3d {


// ---------------------------------------------------------------- ghost fill

// Two periodic ghost layers per face over interior ranges of the other two axes
// (no edges or corners). The three face groups read only interior cells, so
// they run as one launch. T: double state arrays (ncomp = nm) or int per-cell records.
// f0 > 0 skips the first f0 faces: f0 = 4 ny nz leaves the x faces to the caller (x-slab
// decomposition, whose x ghosts come from the neighbouring slabs).
template <typename T>
__global__ void ghost_fill_kernel(GridDims g, T *__restrict__ u, int ncomp, long long f0)
{
    const long long total = (ghost_faces(g) - f0) * ncomp;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = (int)(e % ncomp);
        long long dst, src;
        ghost_pair(g, f0 + e / ncomp, dst, src);
        u[dst * ncomp + m] = u[src * ncomp + m];
    }
}

// Closure statistics of the face ghosts whose records a mirrored closure copied from their
// images: the same counters a solve adds (finalize, closure_core.cuh), so that the totals
// equal those of solving every cell.
__global__ void ghost_stats_kernel(GridDims g, const int *__restrict__ iters,
                                   const int *__restrict__ iterGamma,
                                   const int *__restrict__ regIdx, const int *__restrict__ status,
                                   unsigned long long *stats)
{
    // the CTA's counters in shared memory, added to the context's once per CTA
    __shared__ unsigned long long sStat[STAT_COUNT];
    for (int q = threadIdx.x; q < STAT_COUNT; q += blockDim.x)
        sStat[q] = 0;
    __syncthreads();
    const long long total = ghost_faces(g);
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < total;
         f += (long long)gridDim.x * blockDim.x) {
        long long dst, src;
        ghost_pair(g, f, dst, src);
        const unsigned long long it = (unsigned long long)iters[dst];
        const unsigned long long ig = (unsigned long long)iterGamma[dst];
        atomicAdd(&sStat[STAT_CELLS], 1ull);
        atomicAdd(&sStat[STAT_ITERS], it);
        atomicAdd(&sStat[STAT_ITER_GAMMA], ig);
        atomicMax(&sStat[STAT_MAX_ITER], it);
        atomicMax(&sStat[STAT_MAX_ITER_GAMMA], ig);
        if (status[dst] != CELL_OK)
            atomicAdd(&sStat[STAT_FAILED], 1ull);
        atomicAdd(&sStat[STAT_REG_HIST + (regIdx[dst] & 15)], 1ull);
        atomicAdd(&sStat[STAT_ITER_HIST + (it < 63 ? it : 63)], 1ull);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < STAT_COUNT; q += blockDim.x) {
        const unsigned long long v = sStat[q];
        if (v == 0)
            continue;
        if (q == STAT_MAX_ITER || q == STAT_MAX_ITER_GAMMA)
            atomicMax(&stats[q], v);
        else
            atomicAdd(&stats[q], v);
    }
}

// One closure's records along the x-line (i, (ny+3)/2, (nz+3)/2) of interior cells:
// {r, iter, iterGamma, gamma, normG} per cell (src/update.cpp:66-75 unbatched,
// :147-155 batched, where the stored gamma is the gamma-iteration count).
__global__ void line_log_kernel(GridDims g, ClosureParams P, const int *__restrict__ iters,
                                const int *__restrict__ iterGamma, const int *__restrict__ regIdx,
                                const double *__restrict__ gamma, const double *__restrict__ normG,
                                double *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nx)
        return;
    const long long c = g.cell(2 + i, (g.ny + 3) / 2, (g.nz + 3) / 2);
    double *o = out + (size_t)i * 5;
    o[0] = P.reg[regIdx[c] & 15];
    o[1] = (double)iters[c];
    o[2] = (double)iterGamma[c];
    o[3] = P.batched ? (double)iterGamma[c] : gamma[c];
    o[4] = normG[c];
}

// *flag = 1 if any face ghost of a differs (bitwise) from its periodic image.
__global__ void ghost_mirror_check_kernel(GridDims g, const double *__restrict__ a, int ncomp,
                                          int *flag)
{
    const long long total = ghost_faces(g) * ncomp;
    const unsigned long long *b = reinterpret_cast<const unsigned long long *>(a);
    bool diff = false;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = (int)(e % ncomp);
        long long dst, src;
        ghost_pair(g, e / ncomp, dst, src);
        diff |= b[dst * ncomp + m] != b[src * ncomp + m];
    }
    if (__syncthreads_or(diff) && threadIdx.x == 0)
        atomicExch(flag, 1);
}

// ---------------------------------------------------------------- ansatz hand-off from the closure

// psi[q nall + ghost] = psi[q nall + image] for every face ghost and direction: the closure
// copied the face ghosts' multipliers from their periodic images, so their ansatz values are
// the images' too (the probe pass wrote the solved cells' values). Grid x: one thread per x-
// or y-face ghost (consecutive threads hold consecutive cells of a z line, so a warp's copies
// per direction are contiguous runs) or per z-face pair (the two ghost layers k = 0, 1 or
// nz+2, nz+3 of one (i, j) line, contiguous, copied as one 16-byte access when nz is even);
// grid y: blocks of qPer directions.
__global__ void psi_face_copy_kernel(GridDims g, int nq, int qPer, double *__restrict__ psi)
{
    const long long fxy = 4LL * g.ny * g.nz + 4LL * g.nx * g.nz;
    const long long nxy = (long long)g.nx * g.ny, nall = g.nall();
    const long long total = fxy + 2 * nxy;
    const int q0 = blockIdx.y * qPer, q1 = min(nq, q0 + qPer);
    const bool vec = (g.nz & 1) == 0; // then every z-face pair and nall are even
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < fxy) {
            long long dst, src;
            ghost_pair(g, t, dst, src);
            const double *sp = psi + src;
            double *dp = psi + dst;
#pragma unroll 4
            for (int q = q0; q < q1; ++q)
                dp[(long long)q * nall] = sp[(long long)q * nall];
        } else {
            const long long r = t - fxy;
            const int side = (int)(r / nxy);
            const long long r2 = r % nxy;
            const int i = 2 + (int)(r2 / g.ny), j = 2 + (int)(r2 % g.ny);
            const long long dst = g.cell(i, j, side == 0 ? 0 : g.nz + 2);
            const long long src = g.cell(i, j, side == 0 ? g.nz : 2);
            if (vec) {
                const double2 *sp = reinterpret_cast<const double2 *>(psi + src);
                double2 *dp = reinterpret_cast<double2 *>(psi + dst);
                const long long step = nall / 2;
#pragma unroll 4
                for (int q = q0; q < q1; ++q)
                    dp[(long long)q * step] = sp[(long long)q * step];
            } else {
#pragma unroll 4
                for (int q = q0; q < q1; ++q) {
                    psi[(long long)q * nall + dst] = psi[(long long)q * nall + src];
                    psi[(long long)q * nall + dst + 1] = psi[(long long)q * nall + src + 1];
                }
            }
        }
    }
}

// psi[q nall + c] = exp(alpha_c . m_q) for the *count cells c of list (one warp per cell,
// directions over the lanes; exponent summed in the reference's order, unfused): the cells
// whose multipliers the closure changed after its probe pass had written their psi.
__global__ void psi_refresh_kernel(GridDims g, int nq, const double *__restrict__ M,
                                   const double *__restrict__ alpha, const int *__restrict__ list,
                                   const unsigned int *__restrict__ count, double *__restrict__ psi)
{
    const int nm = g.nm;
    const long long nall = g.nall();
    const unsigned int n = *count;
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = w0; i < n; i += nw) {
        const long long c = list[i];
        const double *a = alpha + c * nm;
        for (int q = lane; q < nq; q += 32) {
            const double *m = M + (size_t)q * nm;
            double z = 0.0;
            for (int k = 0; k < nm; ++k)
                z = __dadd_rn(z, __dmul_rn(a[k], m[k]));
            psi[(long long)q * nall + c] = exp(z);
        }
    }
}

// ---------------------------------------------------------------- Euler / RK

__device__ __forceinline__ bool interior(const GridDims &g, long long c, int &i, int &j, int &k)
{
    k = (int)(c % g.nzg());
    long long r = c / g.nzg();
    j = (int)(r % g.nyg());
    i = (int)(r / g.nyg());
    return i >= 2 && i < g.nx + 2 && j >= 2 && j < g.ny + 2 && k >= 2 && k < g.nz + 2;
}


__global__ void euler_kernel(GridDims g, double *__restrict__ u, const double *__restrict__ flux,
                             const double *__restrict__ sigT, const double *__restrict__ sigS,
                             double dt)
{
    const int nm = g.nm;
    const long long total = g.ninterior() * nm;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = (int)(e % nm);
        long long c = interior_cell(g, e / nm);
        long long x = c * nm + m;
        double st = sigT[c];
        double v;
        if (m == 0) {
            double fac = __dsub_rn(__dadd_rn(1.0, __dmul_rn(dt, sigS[c])), __dmul_rn(dt, st));
            v = __dsub_rn(__dmul_rn(u[x], fac), __dmul_rn(dt, flux[x]));
        } else {
            v = __dsub_rn(__dmul_rn(u[x], __dsub_rn(1.0, __dmul_rn(dt, st))), __dmul_rn(dt, flux[x]));
        }
        u[x] = v;
    }
}

// mode 0: uOld <- u ; mode 1: u <- 0.5 (u + uOld)   (interior cells only)
__global__ void rk_kernel(GridDims g, double *__restrict__ u, double *__restrict__ uOld, int mode)
{
    const int nm = g.nm;
    const long long total = g.ninterior() * nm;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long x = interior_cell(g, e / nm) * nm + (e % nm);
        if (mode == 0)
            uOld[x] = u[x];
        else
            u[x] = __dmul_rn(0.5, __dadd_rn(u[x], uOld[x]));
    }
}

// ---------------------------------------------------------------- kinetic flux on the tensor pipe
//
// Directions come in tiles of 32. Per tile the host prepares (c3d_create) two copies of the
// basis in m8n8k4 fragment order, so that a warp reads each fragment as 32 consecutive
// doubles and a CTA stages a tile with one bulk copy:
//   ansatz     [j 0..3][k-step 0..2NT-1][lane]  M[32t + 8j + lane/4][4k + lane%4]   (B of Z = A M^T)
//   projection [k-step 0..7][j 0..NT-1][lane]   M[32t + 4k + lane%4][8j + lane/4]   (B of F += S M)
//              followed by c_x = (xi w)/dx, c_y = (eta w)/dy, c_z = (mu w)/dz and w of the
//              tile's 32 directions (a direction's limited differences along each axis are
//              weighted by c, whose sign is the cosine's).
// Directions past nq and moments past nm are zero.

constexpr int FLUX_STAGES = 2;

__device__ __forceinline__ void dmma_g(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void fbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)));
}
__device__ __forceinline__ void fbar_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Two bulk copies completing one phase of a barrier initialised for one arrival: a single
// arrive.expect_tx with the combined byte count, then both copies.
__device__ __forceinline__ void fbar_load2(void *dst0, const void *src0, uint32_t bytes0, void *dst1,
                                           const void *src1, uint32_t bytes1, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
                 "r"(bytes0 + bytes1)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst0)),
                 "l"(src0), "r"(bytes0), "r"(smem_addr(bar))
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst1)),
                 "l"(src1), "r"(bytes1), "r"(smem_addr(bar))
                 : "memory");
}
// false if the phase did not complete within the iteration limit
__device__ __forceinline__ bool fbar_wait(uint64_t *bar, uint32_t parity)
{
    for (int it = 0; it < (1 << 26); ++it) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(smem_addr(bar)), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

// psi[(q - q0) nall + c] = exp(alpha_c . m_q) (M_N) or alpha_c . m_q (P_N) for the directions
// q0 <= q < q0 + nqc, q0 a multiple of 32. A CTA owns 64 cells (warp w: 8w..8w+7), keeps
// their multipliers as A fragments in registers and walks the direction tiles of the chunk
// (double-buffered bulk copies of the ansatz fragments): 8 NT DMMAs per 8 x 8 block.
template <int NT>
__global__ void __launch_bounds__(256)
    ansatz_dmma_kernel(GridDims g, const double *__restrict__ alpha, const double *__restrict__ mfA,
                       int q0, int nqc, int isPn, double *__restrict__ psi, int *errorFlag)
{
    constexpr int KS = 2 * NT;
    constexpr int TILE = 4 * KS * 32;
    __shared__ __align__(128) double sB[FLUX_STAGES][TILE];
    __shared__ uint64_t bar[FLUX_STAGES];
    __shared__ int sAbort;
    const int nm = g.nm;
    const long long nall = g.nall();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long c = (long long)blockIdx.x * 64 + 8 * warp + (lane >> 2);
    const int t0 = q0 >> 5, nt = (nqc + 31) >> 5;
    if (tid == 0) {
        sAbort = 0;
        for (int s = 0; s < FLUX_STAGES; ++s)
            fbar_init(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        for (int s = 0; s < FLUX_STAGES && s < nt; ++s)
            fbar_load(sB[s], mfA + (size_t)(t0 + s) * TILE, TILE * 8, &bar[s]);
    }
    double a[KS];
#pragma unroll
    for (int kk = 0; kk < KS; ++kk) {
        int k = 4 * kk + (lane & 3);
        a[kk] = (c < nall && k < nm) ? alpha[c * nm + k] : 0.0;
    }
    __syncthreads();
    for (int t = 0; t < nt; ++t) {
        const int s = t % FLUX_STAGES;
        if (!fbar_wait(&bar[s], (t / FLUX_STAGES) & 1))
            sAbort = 1;
        if (__syncthreads_or(sAbort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *B = sB[s];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double z0 = 0.0, z1 = 0.0;
#pragma unroll
            for (int kk = 0; kk < KS; ++kk)
                dmma_g(z0, z1, a[kk], B[(j * KS + kk) * 32 + lane]);
            const int ql = 32 * t + 8 * j + 2 * (lane & 3); // direction within the chunk
            if (c < nall) {
                if (ql < nqc)
                    psi[(long long)ql * nall + c] = isPn ? z0 : exp(z0);
                if (ql + 1 < nqc)
                    psi[(long long)(ql + 1) * nall + c] = isPn ? z1 : exp(z1);
            }
        }
        __syncthreads();
        if (tid == 0 && t + FLUX_STAGES < nt)
            fbar_load(sB[s], mfA + (size_t)(t0 + t + FLUX_STAGES) * TILE, TILE * 8, &bar[s]);
    }
}

// minmod of src/flux_kinetic.cpp:45-50 as a select: the same value (x when |x| < |y|, else
// y, for operands of one sign; 0 otherwise), except possibly for the sign of a zero and for
// operands whose product underflows.
__device__ __forceinline__ double minmod_sel(double x, double y)
{
    return (x * y > 0.0) ? (fabs(x) < fabs(y) ? x : y) : 0.0;
}

// Limited upwind difference along one axis for either sign of the direction weight c (the
// cosine's sign), src/flux_kinetic.cpp:130-189. With h = +1/2 (c > 0: values k1..k4 at offsets
// -2..1) or h = -1/2 (c <= 0: offsets -1..2),
//   f = ((k3 + h s(k2,k3,k4)) - k2) - h s(k1,k2,k3),  s(l,c,r) = slopefit (src/flux_kinetic.cpp:56-61)
//     = minmod(th (r - c), minmod((r - l) / 2, th (c - l))).
// Here s' = 2 s = minmod(2th (r - c), minmod(r - l, 2th (c - l))) and h s = (h/2) s': scaling by
// powers of two commutes with rounding and with the minmod's comparisons, so f rounds as the
// reference's expression with two multiplications fewer per axis (th2 = 2 th).
__device__ __forceinline__ double axis_flux_bf(double c, double th2, const double *pc,
                                               long long st)
{
    const bool pos = c > 0;
    const double *b = pos ? pc - 2 * st : pc - st;
    const double k1 = b[0], k2 = b[st], k3 = b[2 * st], k4 = b[3 * st];
    const double q = pos ? 0.25 : -0.25; // h / 2
    const double t32 = th2 * (k3 - k2);
    const double s1 = minmod_sel(th2 * (k4 - k3), minmod_sel(k4 - k2, t32));
    const double s2 = minmod_sel(t32, minmod_sel(k3 - k1, th2 * (k2 - k1)));
    return fma(-q, s2, fma(q, s1, k3) - k2);
}

// flux(c) (+)= sum_q m_q (c_x fx + c_y fy + c_z fz) (c = cosine x weight / spacing of the
// direction, fx.. the limited differences) for 64 interior cells per CTA (consecutive
// in the interior numbering). Per direction tile: the limited upwind differences S[q][cell]
// of the CTA (each thread 8 (cell, direction) pairs, loads issued two pairs at a time) go to
// shared memory, then F += S^T M on the FP64 tensor pipe (warp w: cells 8w..8w+7, all moment
// tiles), with the projection fragments and direction cosines staged by bulk copies.
template <int NT>
__global__ void __launch_bounds__(256)
    kinetic_dmma_kernel(GridDims g, const double *__restrict__ psi, const double *__restrict__ mfP,
                        int q0, int nqc, double theta, int accumulate, double *__restrict__ flux,
                        int *errorFlag)
{
    constexpr int TILE = 8 * NT * 32 + 128;
    constexpr int CS = 68; // S tile row stride (cells)
    const double th2 = 2.0 * theta;
    extern __shared__ __align__(128) double kinSmem[]; // sB[FLUX_STAGES][TILE], sS[32 * CS]
    double(*sB)[TILE] = reinterpret_cast<double(*)[TILE]>(kinSmem);
    double *sS = kinSmem + FLUX_STAGES * TILE;
    __shared__ long long sCell[64];
    __shared__ uint64_t bar[FLUX_STAGES];
    __shared__ int sAbort;
    const int nm = g.nm;
    const long long nall = g.nall(), nint = g.ninterior();
    const long long n0 = (long long)blockIdx.x * 64;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long sx = (long long)g.nyg() * g.nzg(), sy = g.nzg(), sz = 1;
    const int t0 = q0 >> 5, nt = (nqc + 31) >> 5;
    if (tid == 0) {
        sAbort = 0;
        for (int s = 0; s < FLUX_STAGES; ++s)
            fbar_init(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        for (int s = 0; s < FLUX_STAGES && s < nt; ++s)
            fbar_load(sB[s], mfP + (size_t)(t0 + s) * TILE, TILE * 8, &bar[s]);
    }
    if (tid < 64)
        sCell[tid] = (n0 + tid < nint) ? interior_cell(g, n0 + tid) : -1;
    __syncthreads();
    const long long myc = sCell[8 * warp + (lane >> 2)];
    double acc[NT][2];
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * j + 2 * (lane & 3) + e2;
            acc[j][e2] = (accumulate && myc >= 0 && m < nm) ? flux[myc * nm + m] : 0.0;
        }
    const int cl = tid & 63;
    const long long c = sCell[cl];
    for (int t = 0; t < nt; ++t) {
        const int s = t % FLUX_STAGES;
        if (!fbar_wait(&bar[s], (t / FLUX_STAGES) & 1))
            sAbort = 1;
        if (__syncthreads_or(sAbort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *dirs = sB[s] + 8 * NT * 32; // c_x, c_y, c_z, w per direction
#pragma unroll 2
        for (int i = 0; i < 8; ++i) {
            const int qq = (tid >> 6) + 4 * i;
            const int ql = 32 * t + qq;
            double sv = 0.0;
            if (c >= 0 && ql < nqc) {
                const double *pc = psi + (long long)ql * nall + c;
                const double cx = dirs[qq], cy = dirs[qq + 32], cz = dirs[qq + 64];
                const double fx = axis_flux_bf(cx, th2, pc, sx);
                const double fy = axis_flux_bf(cy, th2, pc, sy);
                const double fz = axis_flux_bf(cz, th2, pc, sz);
                sv = fx * cx + fy * cy + fz * cz;
            }
            sS[qq * CS + cl] = sv;
        }
        __syncthreads();
        const double *B = sB[s];
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const double a = sS[(4 * kk + (lane & 3)) * CS + 8 * warp + (lane >> 2)];
#pragma unroll
            for (int j = 0; j < NT; ++j)
                dmma_g(acc[j][0], acc[j][1], a, B[(kk * NT + j) * 32 + lane]);
        }
        __syncthreads();
        if (tid == 0 && t + FLUX_STAGES < nt)
            fbar_load(sB[s], mfP + (size_t)(t0 + t + FLUX_STAGES) * TILE, TILE * 8, &bar[s]);
    }
    if (myc < 0)
        return;
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * j + 2 * (lane & 3) + e2;
            if (m < nm)
                flux[myc * nm + m] = acc[j][e2];
        }
}

// minmod(p, minmod(q, s)) of src/flux_kinetic.cpp:45-61 is symmetric in its three operands:
// sign * min(|p|, |q|, |s|) when all three have one sign, else 0 (the reference's nested form
// gives exactly that: its MIN/MAX select operands without rounding). Here the operand of
// smallest magnitude is chosen by two FP64 compares of absolute values and kept when the sign
// bits of the three high words agree: the same value as the nested form, except possibly for
// the sign of a zero. (On sm_100a this beat the nested selects by 10% in the staged flux, and
// an integer-pipe form and an fmin/fmax form by 8% and 30%.)
__device__ __forceinline__ double minmod3(double p, double q, double s)
{
    double m = fabs(q) < fabs(p) ? q : p;
    m = fabs(s) < fabs(m) ? s : m;
    const bool same =
        ((__double2hiint(p) ^ __double2hiint(q)) | (__double2hiint(q) ^ __double2hiint(s))) >= 0;
    return same ? m : 0.0;
}

// The limited upwind difference along one axis of src/flux_kinetic.cpp:130-189 from the four
// stencil values k1..k4 (offsets -2..1 with h = 1/2 for a positive cosine, -1..2 with h = -1/2
// otherwise): f = ((k3 + h s(k2,k3,k4)) - k2) - h s(k1,k2,k3), s = slopefit
// (src/flux_kinetic.cpp:56-61), evaluated as in axis_flux_bf: s' = 2 s from 2 th (th2) and
// unscaled centred differences, q = h / 2, so f rounds as the reference's expression.
__device__ __forceinline__ double axis_flux_m3(double q, double th2, double k1, double k2,
                                               double k3, double k4)
{
    const double t32 = th2 * (k3 - k2);
    const double s1 = minmod3(th2 * (k4 - k3), k4 - k2, t32);
    const double s2 = minmod3(t32, k3 - k1, th2 * (k2 - k1));
    return fma(-q, s2, fma(q, s1, k3) - k2);
}

// The kinetic flux of kinetic_dmma_kernel with psi staged in shared memory. A CTA owns one
// run of L consecutive interior cells along z (i, j, k0 .. k0 + L - 1; L = min(64, nz), L
// even, nz a multiple of L) and walks its direction chunk in sub-stages of KDS = 8
// directions, two in flight. Per direction a sub-stage holds seven contiguous runs of psi,
// brought in by 1-D bulk copies: the cell run with two halo cells on either side (L + 4
// values) and the three x- and three y-neighbour lines the upwind stencil of that direction
// reads (offsets -2, -1, +1 for a positive cosine, -1, +1, +2 otherwise; L values each), and
// the sub-stage's two projection k-steps and its directions' cosines and weights; warp d
// copies direction d (warp 0 also the projection data), each warp arriving on the stage's
// mbarrier with its bytes. Each thread forms the limited differences of the two (cell,
// direction) pairs whose values it holds in the DMMA A fragments of the sub-stage's two
// k-steps (cell 8 warp + lane / 4, direction 4 k + lane % 4), from shared memory and
// branch-free (the staged slots put the stencil values of either sign of the cosine at fixed
// places; the limiter is the three-operand minmod), then projects them onto the moments with
// DMMAs straight from its registers (k-steps 2v, 2v + 1 of the 32-direction fragment tile, in
// order), so the flux has the same values as kinetic_dmma_kernel's. One barrier per sub-stage,
// before its buffers are refilled.
constexpr int KDS = 8;                      // directions per sub-stage
constexpr int KRUN = 64;                    // longest cell run per CTA
// doubles staged per direction: the runs back to back (KPER = 4 mod 16, so the four directions
// a warp reads at once, one DMMA k-step, start a quarter of the banks apart; a padding to
// 8 mod 16 measured 2% slower)
constexpr int KPER = (KRUN + 4) + 6 * KRUN;
template <int NT> struct KinStage {
    static constexpr int FRAG = 2 * NT * 32;                    // two projection k-steps
    static constexpr int DOUBLES = KDS * KPER + FRAG + 4 * KDS; // + c_x, c_y, c_z, w of KDS dirs
};
template <int NT>
__global__ void __launch_bounds__(256, 3)
    kinetic_staged_kernel(GridDims g, const double *__restrict__ psi, const double *__restrict__ mfP,
                          const double *__restrict__ xiAll, const double *__restrict__ etaAll,
                          int q0, int nqc, int L, double theta, int accumulate,
                          double *__restrict__ flux, int *errorFlag, const int *wrapFlag)
{
    constexpr int TILE = 8 * NT * 32 + 128; // one 32-direction tile of mfP
    constexpr int SD = KinStage<NT>::DOUBLES, FRAG = KinStage<NT>::FRAG;
    static_assert((SD * 8) % 16 == 0 && (KPER * 8) % 16 == 0, "stage alignment");
    static_assert(KDS * 32 == 256, "one warp per direction of a sub-stage");
    extern __shared__ __align__(128) double kinSmem[];
    __shared__ uint64_t pbar[2];
    __shared__ long long sRun[9];
    const double th2 = 2.0 * theta;
    const int nm = g.nm;
    const long long nall = g.nall();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // block order: z run index slowest; the (i, j) lines in tiles of 16 x 16 (row-major,
    // partial tiles at the edges), so that CTAs running at the same time stage each other's
    // neighbour lines from L2
    int i, j, kb;
    {
        constexpr int TI = 16, TJ = 16;
        const long long lines = (long long)g.nx * g.ny;
        kb = (int)(blockIdx.x / lines);
        const long long r = blockIdx.x % lines, rowBlock = (long long)TI * g.ny;
        const int ti = (int)(r / rowBlock);
        const long long r2 = r % rowBlock;
        const int hi = min(TI, g.nx - ti * TI);
        const int tj = (int)(r2 / ((long long)hi * TJ));
        const int r3 = (int)(r2 % ((long long)hi * TJ));
        const int wj = min(TJ, g.ny - tj * TJ);
        i = 2 + ti * TI + r3 / wj;
        j = 2 + tj * TJ + r3 % wj;
    }
    const int k0 = 2 + kb * L;
    const int t0 = q0 >> 5, nu = (nqc + KDS - 1) / KDS;
    // start cell of run r: 0 the cell run with its z halo, 1-4 x offsets -2, -1, +1, +2,
    // 5-8 y offsets -2, -1, +1, +2
    // wrap (the closure copied the face ghosts from their periodic images and their psi was
    // not copied): stencil values of face ghosts are read at the images instead -- the x and
    // y neighbour lines of the periodic grid, and the z halo pairs of runs at either end
    const bool wrap = wrapFlag && *wrapFlag == 0;
    const bool lowB = wrap && k0 == 2, highB = wrap && k0 + L == g.nz + 2;
    if (tid < 9) {
        const int r = tid, o = (r - 1) & 3, d = o < 2 ? o - 2 : o - 1;
        auto per = [&](int a, int n) { return !wrap ? a : a < 2 ? a + n : a >= n + 2 ? a - n : a; };
        sRun[r] = r == 0    ? g.cell(i, j, k0 - 2)
                  : r <= 4 ? g.cell(per(i + d, g.nx), j, k0)
                           : g.cell(i, per(j + d, g.ny), k0);
    }
    const uint32_t perDir = (uint32_t)((L + 4) + 6 * L) * 8;
    // a direction's stage: the cell run, then x slots 0-2, then y slots 0-2 (offsets -2, -1,
    // +1 for a positive cosine, -1, +1, +2 otherwise)
    auto issue = [&](int u) {
        const int nd = min(KDS, nqc - KDS * u), d = warp;
        double *st = kinSmem + (u & 1) * SD;
        uint64_t *b = &pbar[u & 1];
        uint32_t bytes = d < nd ? perDir : 0u;
        if (d == 0)
            bytes += (FRAG + 4 * KDS) * 8;
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                             smem_addr(b)),
                         "r"(bytes)
                         : "memory");
        __syncwarp();
        const double *src = nullptr;
        double *dst = nullptr;
        uint32_t nb = 0;
        if (d < nd && lane < 7) {
            const int ql = KDS * u + d;
            int r = 0, off = 0;
            if (lane >= 1 && lane <= 3) {
                const int sl = lane - 1;
                r = (xiAll[q0 + ql] > 0 ? 1 : 2) + sl; // runs 1-4: offsets -2, -1, +1, +2
                off = (L + 4) + sl * L;
            } else if (lane >= 4) {
                const int sl = lane - 4;
                r = (etaAll[q0 + ql] > 0 ? 5 : 6) + sl;
                off = (L + 4) + (3 + sl) * L;
            }
            src = psi + (long long)ql * nall + sRun[r];
            dst = st + d * KPER + off;
            nb = (uint32_t)(r == 0 ? L + 4 : L) * 8;
            if (r == 0 && (lowB || highB)) {
                // the run without the halo pairs that lanes 12 and 13 bring from the images
                src += lowB ? 2 : 0;
                dst += lowB ? 2 : 0;
                nb -= (uint32_t)(2 * lowB + 2 * highB) * 8;
            }
        } else if (d < nd && ((lane == 12 && lowB) || (lane == 13 && highB))) {
            // z halo pair of a run at the low end (ghosts k = 0, 1 = images nz, nz + 1) or the
            // high end (k = nz + 2, nz + 3 = images 2, 3); 16-byte aligned: nz and L are even
            const int ql = KDS * u + d;
            src = psi + (long long)ql * nall + g.cell(i, j, lane == 12 ? g.nz : 2);
            dst = st + d * KPER + (lane == 12 ? 0 : L + 2);
            nb = 16;
        } else if (d == 0 && lane >= 7 && lane <= 11) {
            const int ql = KDS * u;
            const double *tile = mfP + (size_t)(t0 + (ql >> 5)) * TILE;
            const int v = (ql & 31) / KDS;
            if (lane == 7) {
                src = tile + v * FRAG;
                dst = st + KDS * KPER;
                nb = FRAG * 8;
            } else {
                src = tile + 8 * NT * 32 + 32 * (lane - 8) + KDS * v; // c_x, c_y, c_z, w
                dst = st + KDS * KPER + FRAG + KDS * (lane - 8);
                nb = KDS * 8;
            }
        }
        if (nb)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                             smem_addr(dst)),
                         "l"(src), "r"(nb), "r"(smem_addr(b))
                         : "memory");
    };
    if (tid == 0) {
        for (int s = 0; s < 2; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(&pbar[s])),
                         "r"(KDS));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    for (int u = 0; u < 2 && u < nu; ++u)
        issue(u);
    const int cw = 8 * warp + (lane >> 2); // the warp's projection cells
    const long long myc = cw < L ? g.cell(i, j, k0 + cw) : -1;
    double acc[NT][2];
#pragma unroll
    for (int jj = 0; jj < NT; ++jj)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * jj + 2 * (lane & 3) + e2;
            acc[jj][e2] = (accumulate && myc >= 0 && m < nm) ? flux[myc * nm + m] : 0.0;
        }
    for (int u = 0; u < nu; ++u) {
        const double *st = kinSmem + (u & 1) * SD;
        // a timed-out wait is agreed on at the barrier after the stencil (the data of that
        // sub-stage are then not used)
        const bool ok = fbar_wait(&pbar[u & 1], (u >> 1) & 1);
        const double *dirs = st + KDS * KPER + FRAG; // c_x[KDS], c_y[KDS], c_z[KDS], w[KDS]
        double afr[2]; // the thread's own A fragments of the sub-stage's two k-steps
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            // cell 8 warp + lane / 4, direction 4 r + lane % 4: the element of the DMMA A
            // fragment (k-step r) the thread holds
            const int cl = cw, d = 4 * r + (lane & 3);
            const int ql = KDS * u + d;
            double sv = 0.0;
            if (cl < L && ql < nqc) {
                const double *P = st + d * KPER;
                const double *xr = P + (L + 4), *yr = xr + 3 * L;
                const double c0 = P[cl + 2];
                // the direction's weights c = cosine x w / spacing per axis
                const double ox = dirs[d], oy = dirs[KDS + d], oz = dirs[2 * KDS + d];
                // branch-free: the staged x and y slots hold offsets (-2, -1, +1) for a positive
                // cosine and (-1, +1, +2) otherwise, so k1 and k4 always come from slots 0 and 2
                // and the cell's own value is k3 or k2; the z run holds offsets -2 .. +2
                const bool px = ox > 0, py = oy > 0, pz = oz > 0;
                const double ax = xr[L + cl], ay = yr[L + cl];
                const double fx = axis_flux_m3(px ? 0.25 : -0.25, th2, xr[cl], px ? ax : c0,
                                               px ? c0 : ax, xr[2 * L + cl]);
                const double fy = axis_flux_m3(py ? 0.25 : -0.25, th2, yr[cl], py ? ay : c0,
                                               py ? c0 : ay, yr[2 * L + cl]);
                const double *zb = P + cl + (pz ? 0 : 1);
                const double fz = axis_flux_m3(pz ? 0.25 : -0.25, th2, zb[0], zb[1], zb[2], zb[3]);
                sv = fx * ox + fy * oy + fz * oz;
            }
            afr[r] = sv;
        }
        // projection straight from the registers; one barrier per sub-stage (before its stage
        // is refilled), where a timed-out wait is agreed on
        const double *B = st + KDS * KPER;
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int jj = 0; jj < NT; ++jj)
                dmma_g(acc[jj][0], acc[jj][1], afr[h], B[(h * NT + jj) * 32 + lane]);
        if (__syncthreads_or(!ok)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        if (u + 2 < nu)
            issue(u + 2);
    }
    if (myc < 0)
        return;
#pragma unroll
    for (int jj = 0; jj < NT; ++jj)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * jj + 2 * (lane & 3) + e2;
            if (m < nm)
                flux[myc * nm + m] = acc[jj][e2];
        }
}

// ---------------------------------------------------------------- P_N moment flux

// One CTA handles CPB interior cells; phase 1 forms the six 4-point differences per
// cell, phase 2 applies the six half-range operators row by row in the order of
// mvProduct (src/flux_moment.cpp:15-24, :57-101).
__global__ void moment_flux_kernel(GridDims g, const double *__restrict__ u,
                                   const double *__restrict__ ops, double dx, double dy, double dz,
                                   int cellsPerBlock, double *__restrict__ flux)
{
    extern __shared__ double sh[];
    const int nm = g.nm;
    double *T = sh; // cellsPerBlock x 6 x nm
    const long long nint = g.ninterior();
    long long n0 = (long long)blockIdx.x * cellsPerBlock;
    const long long sx = (long long)g.nyg() * g.nzg(), sy = g.nzg(), sz = 1;
    for (int e = threadIdx.x; e < cellsPerBlock * nm; e += blockDim.x) {
        int cl = e / nm, m = e % nm;
        long long n = n0 + cl;
        if (n >= nint)
            continue;
        long long c = interior_cell(g, n);
        const long long st[3] = {sx, sy, sz};
        for (int ax = 0; ax < 3; ++ax) {
            long long s = st[ax];
#define UU(o) u[(c + (o) * s) * nm + m]
            double tp = __dadd_rn(__dsub_rn(__dadd_rn(__dmul_rn(0.25, UU(1)), __dmul_rn(0.75, UU(0))),
                                            __dmul_rn(1.25, UU(-1))),
                                  __dmul_rn(0.25, UU(-2)));
            double tm = __dsub_rn(__dsub_rn(__dadd_rn(__dmul_rn(-0.25, UU(2)), __dmul_rn(1.25, UU(1))),
                                            __dmul_rn(0.75, UU(0))),
                                  __dmul_rn(0.25, UU(-1)));
#undef UU
            T[(cl * 6 + 2 * ax + 0) * nm + m] = tp;
            T[(cl * 6 + 2 * ax + 1) * nm + m] = tm;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < cellsPerBlock * nm; e += blockDim.x) {
        int cl = e / nm, i = e % nm;
        long long n = n0 + cl;
        if (n >= nint)
            continue;
        long long c = interior_cell(g, n);
        double axf[3];
        for (int ax = 0; ax < 3; ++ax) {
            const double *Ap = ops + (2 * ax + 0) * (long long)nm * nm + (long long)i * nm;
            const double *Am = ops + (2 * ax + 1) * (long long)nm * nm + (long long)i * nm;
            const double *tp = T + (cl * 6 + 2 * ax + 0) * nm;
            const double *tm = T + (cl * 6 + 2 * ax + 1) * nm;
            double b = 0.0;
            for (int j = 0; j < nm; ++j)
                b = __dadd_rn(b, __dmul_rn(__ldg(Ap + j), tp[j]));
            for (int j = 0; j < nm; ++j)
                b = __dadd_rn(b, __dmul_rn(__ldg(Am + j), tm[j]));
            axf[ax] = b;
        }
        flux[c * nm + i] = __dadd_rn(__dadd_rn(__ddiv_rn(axf[0], dx), __ddiv_rn(axf[1], dy)),
                                     __ddiv_rn(axf[2], dz));
    }
}

// ---------------------------------------------------------------- launchers

static int grid_for(long long n, int threads, int numSMs)
{
    long long b = (n + threads - 1) / threads;
    long long cap = (long long)numSMs * 16;
    if (b > cap)
        b = cap;
    return b < 1 ? 1 : (int)b;
}

cudaError_t launch_ghost_fill(const GridDims &g, double *u, int numSMs, cudaStream_t st,
                              bool skipX)
{
    const long long f0 = skipX ? 4LL * g.ny * g.nz : 0;
    ghost_fill_kernel<double><<<grid_for((ghost_faces(g) - f0) * g.nm, 256, numSMs), 256, 0, st>>>(
        g, u, g.nm, f0);
    return cudaGetLastError();
}

cudaError_t launch_ghost_fill_int(const GridDims &g, int *a, int numSMs, cudaStream_t st)
{
    ghost_fill_kernel<int><<<grid_for(ghost_faces(g), 256, numSMs), 256, 0, st>>>(g, a, 1, 0);
    return cudaGetLastError();
}

cudaError_t launch_ghost_fill_1(const GridDims &g, double *a, int numSMs, cudaStream_t st)
{
    ghost_fill_kernel<double><<<grid_for(ghost_faces(g), 256, numSMs), 256, 0, st>>>(g, a, 1, 0);
    return cudaGetLastError();
}

cudaError_t launch_line_log(const GridDims &g, const ClosureParams &P, const int *iters,
                            const int *iterGamma, const int *regIdx, const double *gamma,
                            const double *normG, double *out, cudaStream_t st)
{
    line_log_kernel<<<(g.nx + 127) / 128, 128, 0, st>>>(g, P, iters, iterGamma, regIdx, gamma,
                                                         normG, out);
    return cudaGetLastError();
}

cudaError_t launch_ghost_stats(const GridDims &g, const int *iters, const int *iterGamma,
                               const int *regIdx, const int *status, unsigned long long *stats,
                               int numSMs, cudaStream_t st)
{
    ghost_stats_kernel<<<grid_for(ghost_faces(g), 256, numSMs), 256, 0, st>>>(
        g, iters, iterGamma, regIdx, status, stats);
    return cudaGetLastError();
}

cudaError_t launch_ghost_mirror_check(const GridDims &g, const double *a, int *flag, int numSMs,
                                      cudaStream_t st)
{
    ghost_mirror_check_kernel<<<grid_for(ghost_faces(g) * g.nm, 256, numSMs), 256, 0, st>>>(
        g, a, g.nm, flag);
    return cudaGetLastError();
}

// The refresh comes first: a face ghost copies its image's final psi, and the image may be
// one of the refreshed cells.
// psiValid (may be null): set once psi holds every non-face-ghost cell's ansatz for the final
// multipliers, so that the next closure's probe pass need not write it again.
cudaError_t launch_psi_handoff(const GridDims &g, int nq, const double *M, const double *alpha,
                               bool faceCopy, const int *refresh, const unsigned int *refreshCount,
                               double *psi, int *psiValid, int numSMs, cudaStream_t st)
{
    psi_refresh_kernel<<<2 * numSMs, 256, 0, st>>>(g, nq, M, alpha, refresh, refreshCount, psi);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && psiValid)
        e = cudaMemsetAsync(psiValid, 1, sizeof(int), st);
    if (e != cudaSuccess || !faceCopy)
        return e;
    constexpr int QPER = 64;
    const long long threads = 4LL * g.ny * g.nz + 4LL * g.nx * g.nz + 2LL * g.nx * g.ny;
    const dim3 grid((unsigned)((threads + 255) / 256), (unsigned)ceil_div(nq, QPER));
    psi_face_copy_kernel<<<grid, 256, 0, st>>>(g, nq, QPER, psi);
    return cudaGetLastError();
}

cudaError_t launch_euler(const GridDims &g, double *u, const double *flux, const double *sigT,
                         const double *sigS, double dt, int numSMs, cudaStream_t st)
{
    euler_kernel<<<grid_for(g.ninterior() * g.nm, 256, numSMs), 256, 0, st>>>(g, u, flux, sigT, sigS,
                                                                              dt);
    return cudaGetLastError();
}

cudaError_t launch_rk(const GridDims &g, double *u, double *uOld, int mode, int numSMs,
                      cudaStream_t st)
{
    rk_kernel<<<grid_for(g.ninterior() * g.nm, 256, numSMs), 256, 0, st>>>(g, u, uOld, mode);
    return cudaGetLastError();
}

// Robustness re-projection after the closure (the note in the reference's readme.txt:
// "one should calculate a new u^n so that u^n = <m exp(m^T alpha^n)> exactly ... and scale
// u^n and alpha^n so that u_0^n does not change"): per cell u' = sum_q w_q m_q e^{alpha.m_q};
// with s = u_0 / u'_0, u <- (u_0, s u'_1, ..., s u'_{nm-1}) and alpha_0 <- alpha_0 + log(s)/m_0
// (m_0 = 1/(2 sqrt(pi)); e^{alpha.m} s = e^{alpha'.m}). A CTA owns 64 cells: per direction
// tile the exponents (DMMA, multipliers as A fragments), c = w e^{z} into shared memory, then
// the moments (DMMA with the projection fragments) -- the ansatz and projection layouts of
// the kinetic flux.
template <int NT>
__global__ void __launch_bounds__(256)
    reproject_kernel(GridDims g, double *__restrict__ u, double *__restrict__ alpha,
                     const double *__restrict__ mfA, const double *__restrict__ mfP, int nq,
                     int *errorFlag)
{
    constexpr int KS = 2 * NT;
    constexpr int TA = 4 * KS * 32, TP = 8 * NT * 32 + 128;
    constexpr int CS = 68;
    extern __shared__ __align__(128) double rpSmem[]; // sA[2][TA], sP[2][TP], sC[32][CS]
    double(*sA)[TA] = reinterpret_cast<double(*)[TA]>(rpSmem);
    double(*sP)[TP] = reinterpret_cast<double(*)[TP]>(rpSmem + FLUX_STAGES * TA);
    double *sC = rpSmem + FLUX_STAGES * (TA + TP);
    __shared__ uint64_t bar[FLUX_STAGES];
    __shared__ int sAbort;
    const int nm = g.nm;
    const long long nall = g.nall();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long c = (long long)blockIdx.x * 64 + 8 * warp + (lane >> 2);
    const int nt = (nq + 31) >> 5;
    if (tid == 0) {
        sAbort = 0;
        for (int st = 0; st < FLUX_STAGES; ++st)
            fbar_init(&bar[st]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        for (int st = 0; st < FLUX_STAGES && st < nt; ++st)
            fbar_load2(sA[st], mfA + (size_t)st * TA, TA * 8, sP[st], mfP + (size_t)st * TP,
                       TP * 8, &bar[st]);
    }
    double a[KS];
#pragma unroll
    for (int kk = 0; kk < KS; ++kk) {
        int k = 4 * kk + (lane & 3);
        a[kk] = (c < nall && k < nm) ? alpha[c * nm + k] : 0.0;
    }
    double acc[NT][2];
#pragma unroll
    for (int j = 0; j < NT; ++j)
        acc[j][0] = acc[j][1] = 0.0;
    __syncthreads();
    for (int t = 0; t < nt; ++t) {
        const int st = t % FLUX_STAGES;
        if (!fbar_wait(&bar[st], (t / FLUX_STAGES) & 1))
            sAbort = 1;
        if (__syncthreads_or(sAbort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *w = sP[st] + 8 * NT * 32 + 96;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double z0 = 0.0, z1 = 0.0;
#pragma unroll
            for (int kk = 0; kk < KS; ++kk)
                dmma_g(z0, z1, a[kk], sA[st][(j * KS + kk) * 32 + lane]);
            const int qq = 8 * j + 2 * (lane & 3);
            sC[qq * CS + 8 * warp + (lane >> 2)] = w[qq] * exp(z0);
            sC[(qq + 1) * CS + 8 * warp + (lane >> 2)] = w[qq + 1] * exp(z1);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const double av = sC[(4 * kk + (lane & 3)) * CS + 8 * warp + (lane >> 2)];
#pragma unroll
            for (int j = 0; j < NT; ++j)
                dmma_g(acc[j][0], acc[j][1], av, sP[st][(kk * NT + j) * 32 + lane]);
        }
        __syncthreads();
        if (tid == 0 && t + FLUX_STAGES < nt)
            fbar_load2(sA[st], mfA + (size_t)(t + FLUX_STAGES) * TA, TA * 8, sP[st],
                       mfP + (size_t)(t + FLUX_STAGES) * TP, TP * 8, &bar[st]);
    }
    // lane 4r holds moment 0 of cell r of the warp's tile
    const double un0 = __shfl_sync(0xffffffffu, acc[0][0], lane & ~3);
    if (c >= nall)
        return;
    const double u0 = u[c * nm];
    const double sc = u0 / un0;
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * j + 2 * (lane & 3) + e2;
            if (m > 0 && m < nm)
                u[c * nm + m] = sc * acc[j][e2];
        }
    if ((lane & 3) == 0)
        alpha[c * nm] += 2.0 * sqrt(M_PI) * log(sc);
}

template <int NT>
static cudaError_t reproject_t(const GridDims &g, double *u, double *alpha, const double *mfA,
                               const double *mfP, int nq, int *errorFlag, cudaStream_t st)
{
    constexpr int KS = 2 * NT;
    const size_t smem =
        (size_t)(FLUX_STAGES * (4 * KS * 32 + 8 * NT * 32 + 128) + 32 * 68) * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(reproject_kernel<NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    reproject_kernel<NT><<<(unsigned)((g.nall() + 63) / 64), 256, smem, st>>>(g, u, alpha, mfA,
                                                                             mfP, nq, errorFlag);
    return cudaGetLastError();
}

cudaError_t launch_reproject(const GridDims &g, double *u, double *alpha, const double *mfA,
                             const double *mfP, int nq, int *errorFlag, cudaStream_t st)
{
    switch ((g.nm + 7) / 8) {
    case 1: return reproject_t<1>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 2: return reproject_t<2>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 3: return reproject_t<3>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 4: return reproject_t<4>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 5: return reproject_t<5>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 6: return reproject_t<6>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 7: return reproject_t<7>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    case 8: return reproject_t<8>(g, u, alpha, mfA, mfP, nq, errorFlag, st);
    default: return cudaErrorInvalidValue;
    }
}

// Fragment-order copies of the basis for the flux kernels (layouts above); nt = ceil(nq/32)
// tiles each.
size_t flux_frag_doubles(int nm, int nq, int which)
{
    const int NT = (nm + 7) / 8, nt = (nq + 31) / 32;
    return (size_t)nt * (which == 0 ? 4 * 2 * NT * 32 : 8 * NT * 32 + 128);
}

void flux_frags(int nm, int nq, const double *M, const double *w, const double *xi,
                const double *eta, const double *mu, double rdx, double rdy, double rdz,
                double *mfA, double *mfP)
{
    const int NT = (nm + 7) / 8, KS = 2 * NT, nt = (nq + 31) / 32;
    auto m = [&](int q, int k) { return (q < nq && k < nm) ? M[(size_t)q * nm + k] : 0.0; };
    for (int t = 0; t < nt; ++t) {
        double *A = mfA + (size_t)t * 4 * KS * 32;
        for (int j = 0; j < 4; ++j)
            for (int kk = 0; kk < KS; ++kk)
                for (int l = 0; l < 32; ++l)
                    A[(j * KS + kk) * 32 + l] = m(32 * t + 8 * j + l / 4, 4 * kk + l % 4);
        double *P = mfP + (size_t)t * (8 * NT * 32 + 128);
        for (int kk = 0; kk < 8; ++kk)
            for (int j = 0; j < NT; ++j)
                for (int l = 0; l < 32; ++l)
                    P[(kk * NT + j) * 32 + l] = m(32 * t + 4 * kk + l % 4, 8 * j + l / 4);
        double *D = P + 8 * NT * 32;
        for (int qq = 0; qq < 32; ++qq) {
            int q = 32 * t + qq;
            D[qq] = q < nq ? (xi[q] * w[q]) * rdx : 0.0;
            D[32 + qq] = q < nq ? (eta[q] * w[q]) * rdy : 0.0;
            D[64 + qq] = q < nq ? (mu[q] * w[q]) * rdz : 0.0;
            D[96 + qq] = q < nq ? w[q] : 0.0;
        }
    }
}

template <int NT>
static cudaError_t kinetic_t(const GridDims &g, const double *alpha, const double *mfA,
                             const double *mfP, const double *xi, const double *eta, int nq,
                             int qChunk, int runLen, double theta, int isPn, double *psi,
                             bool psiReady, double *flux, int *errorFlag, const int *wrapFlag,
                             cudaStream_t st)
{
    if (psiReady)
        qChunk = nq; // psi of every direction is in place: the stencil alone, in one pass
    for (int q0 = 0; q0 < nq; q0 += qChunk) {
        int nqc = nq - q0 < qChunk ? nq - q0 : qChunk;
        if (!psiReady)
            ansatz_dmma_kernel<NT><<<(unsigned)((g.nall() + 63) / 64), 256, 0, st>>>(
                g, alpha, mfA, q0, nqc, isPn, psi, errorFlag);
        // staged psi when the z lines split into even runs of at most 64 cells (runLen: the
        // run length chosen by the autotuner, 0 for min(64, nz))
        const int L = runLen > 0 ? runLen : (g.nz < KRUN ? g.nz : KRUN);
        if (L % 2 == 0 && L <= KRUN && g.nz % L == 0) {
            const size_t smem = (size_t)(2 * KinStage<NT>::DOUBLES) * 8;
            auto kern = kinetic_staged_kernel<NT>;
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess)
                return e;
            kern<<<(unsigned)((long long)g.nx * g.ny * (g.nz / L)), 256, smem, st>>>(
                    g, psi, mfP, xi, eta, q0, nqc, L, theta, q0 > 0 ? 1 : 0, flux, errorFlag,
                    wrapFlag);
            e = cudaGetLastError();
            if (e != cudaSuccess)
                return e;
            continue;
        }
        if (wrapFlag) // the global-load form reads the face ghosts themselves
            return cudaErrorInvalidValue;
        const size_t kinSmem = (size_t)(FLUX_STAGES * (8 * NT * 32 + 128) + 32 * 68) * 8;
        // opt in above the 48 KB default for the dynamic part plus the ~1.3 KB static part
        if (kinSmem > 46 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kinetic_dmma_kernel<NT>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)kinSmem);
            if (e != cudaSuccess)
                return e;
        }
        kinetic_dmma_kernel<NT><<<(unsigned)((g.ninterior() + 63) / 64), 256, kinSmem, st>>>(
            g, psi, mfP, q0, nqc, theta, q0 > 0 ? 1 : 0, flux, errorFlag);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// qChunk: a multiple of 32 unless it covers all of nq.
// psiReady: psi[q nall + c] already holds the ansatz of every direction (handed off by the
// closure), so only the stencil and projection run.
// wrapFlag (staged stencil only, else null): a device flag; when it reads 0 the face ghosts'
// psi is not in place and their stencil values are read at their periodic images.
bool kinetic_staged_used(const GridDims &g, int runLen)
{
    const int L = runLen > 0 ? runLen : (g.nz < KRUN ? g.nz : KRUN);
    return L % 2 == 0 && L <= KRUN && g.nz % L == 0;
}

cudaError_t launch_kinetic_flux(const GridDims &g, const double *alpha, const double *mfA,
                                const double *mfP, const double *xi, const double *eta, int nq,
                                int qChunk, int runLen, double theta, int isPn, double *psi,
                                bool psiReady, double *flux, int *errorFlag, const int *wrapFlag,
                                cudaStream_t st)
{
    if (qChunk < nq && (qChunk & 31))
        return cudaErrorInvalidValue;
#define C3D_NT_CASE(NT)                                                                            \
    case NT:                                                                                       \
        return kinetic_t<NT>(g, alpha, mfA, mfP, xi, eta, nq, qChunk, runLen, theta, isPn, psi,  \
                             psiReady, flux, errorFlag, wrapFlag, st);
    switch ((g.nm + 7) / 8) {
        C3D_NT_CASE(1)
        C3D_NT_CASE(2)
        C3D_NT_CASE(3)
        C3D_NT_CASE(4)
        C3D_NT_CASE(5)
        C3D_NT_CASE(6)
        C3D_NT_CASE(7)
        C3D_NT_CASE(8)
    default:
        return cudaErrorInvalidValue;
    }
#undef C3D_NT_CASE
}

cudaError_t launch_moment_flux(const GridDims &g, const double *u, const double *ops, double dx,
                               double dy, double dz, double *flux, cudaStream_t st)
{
    int cpb = 256 / g.nm;
    if (cpb < 1)
        cpb = 1;
    size_t sm = (size_t)cpb * 6 * g.nm * sizeof(double);
    long long blocks = (g.ninterior() + cpb - 1) / cpb;
    moment_flux_kernel<<<(int)blocks, 256, sm, st>>>(g, u, ops, dx, dy, dz, cpb, flux);
    return cudaGetLastError();
}

} // namespace c3d
