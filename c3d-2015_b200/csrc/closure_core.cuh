// Device-side building blocks of the M_N dual solve shared by the closure engines
// (closure_fp64.cu: persistent kernels; closure_rounds.cu: work-list rounds):
// warp utilities, the FP64 DMMA, mbarrier/bulk-copy helpers, the per-warp Cholesky,
// condition estimate and substitutions, and the per-cell Newton state machine of
// src/opt/optBatch.cpp:143-344 / src/opt/opt.cpp:139-355 (see closure_fp64.cu).
#pragma once
#include "c3d_common.cuh"

#include <cfloat>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace c3d {
namespace {

constexpr int STAGES = 3;
constexpr int GSTAGES = 2; // stages of the (larger) Gaunt chunks
constexpr int CST = 12;    // row stride of the coefficient tile (bank-conflict-free B fragments)
constexpr double EPS_HALF = DBL_EPSILON / 2;

enum Need : int { NEED_NONE = 0, NEED_H = 1, NEED_TRIAL = 2, NEED_PROBE = 3 };

// Phase clocks of the per-cell Newton logic (profiling builds only).
#ifdef C3D_NEWTON_CLOCKS
#define C3D_NCLK_DECL long long nclk_ = clock64();
#define C3D_NCLK(stats, slot, lane)                                                                \
    do {                                                                                           \
        long long t_ = clock64();                                                                  \
        if ((lane) == 0 && (stats))                                                                \
            atomicAdd(&(stats)[STAT_CLK_NEWTON + (slot)], (unsigned long long)(t_ - nclk_));       \
        nclk_ = t_;                                                                                \
    } while (0)
#else
#define C3D_NCLK_DECL
#define C3D_NCLK(stats, slot, lane)
#endif

struct SlotScalars {
    long long cell;
    long long passes;
    double u0, alphaScale, rtol, f, t, maxFactor, gd, fquad, r, gamma, err;
    int need, iter, totalIter, iterGamma, regIndex, maxIter, status, exhausted;
    // mixed precision: condition estimate of the last Hessian (-1: none yet; +inf: the
    // factorisation failed), FP64 moments forced for the rest of the closure, and the binary
    // exponent of the largest w_q e^{alpha.m_q} of the last reduced-precision pass (the
    // per-cell shift of the next one)
    double cnd;
    int fp64, cshift;
    int hprec; // precision of the last Hessian: 0 FP64, 1 BF16, 2 3xTF32
};

// Largest moment count (N+1)^2 whose padding to 8 gives NT tiles.
__host__ __device__ constexpr int max_nm_for(int nt)
{
    return nt == 1 ? 4 : nt == 2 ? 16 : nt == 4 ? 25 : nt == 5 ? 36 : nt == 7 ? 49 : 8 * nt;
}

template <int NT> struct Cfg {
    static constexpr int NMP = 8 * NT;
    static constexpr int NML = max_nm_for(NT);
    static constexpr int NPK = NML * (NML + 1) / 2;
    static constexpr int ROWS = NMP + 1; // basis rows + weight row
    static constexpr int CHUNK = ROWS * QCP;
    static constexpr int NTILE = NT * (NT + 1) / 2;
};

__host__ __device__ constexpr int pidx(int i, int j) { return (i * (i + 1)) / 2 + j; }

// Tile (ib, jb), ib >= jb, of the lower triangle of 8x8 tiles, in row order.
__host__ __device__ constexpr int tix(int ib, int jb) { return ib * (ib + 1) / 2 + jb; }

// Offset of element (r, c) inside a tile: row-major by pairs of columns, the pair index of
// row r XOR-ed with (r / 2) & 3. A pair (r, 2q), (r, 2q + 1) stays 16-byte aligned (the
// Cholesky and DMMA accumulator accesses), and the 8 elements of a column land in 8
// distinct 8-byte bank groups (the substitutions and row norms read columns).
__host__ __device__ constexpr int toff(int r, int c)
{
    return 8 * r + 2 * ((c >> 1) ^ ((r >> 1) & 3)) + (c & 1);
}
// Offset of the pair lane l holds in the m8n8 accumulator layout (row l / 4, pair l % 4).
__host__ __device__ constexpr int tpair(int l) { return toff(l >> 2, 2 * (l & 3)); }

// Per-warp state of one cell. The lower triangle of H (then of its Cholesky factor L) is
// either packed row by row (TILED = false) or stored as the lower triangle of 8x8 tiles of
// the matrix padded to 8 NT rows (TILED = true): tile (ib, jb) at 64 tix(ib, jb), inside the
// tile element (r, c) at toff(r, c); lane l of the m8n8k4 DMMA accumulator layout holds the
// pair at tpair(l). Padding rows are those of the identity. 16-byte alignment keeps
// L of every slot in an array aligned for the double2 tile accesses.
template <int NT, bool TILED = false> struct alignas(16) Slot {
    static constexpr int NMP = Cfg<NT>::NMP;
    static constexpr int NTILES = NT * (NT + 1) / 2;
    static constexpr int LSIZE = TILED ? 64 * NTILES : Cfg<NT>::NPK;
    static constexpr bool tiled = TILED;
    static constexpr int nt = NT;
    double u[NMP], alpha[NMP], alpha0[NMP], uOrig[NMP], g[NMP], d[NMP], alphaOld[NMP], rinv[NMP];
    double L[LSIZE];
    SlotScalars s;
    // g, d, alphaOld and rinv as one array of 4 NMP doubles (scratch between Hessian visits),
    // addressed through the slot object so that it may span the four vectors
    __device__ __forceinline__ double *scratch()
    {
        return reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(this) +
                                          4 * NMP * sizeof(double));
    }
    // offset of element (i, j), i >= j
    __device__ static __forceinline__ int lx(int i, int j)
    {
        if (TILED)
            return 64 * tix(i >> 3, j >> 3) + toff(i & 7, j & 7);
        return pidx(i, j);
    }
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

// First index of the largest |x| (LAPACK idamax semantics).
__device__ __forceinline__ int warp_iamax(double a0, double a1, int lane, int n)
{
    double best = (lane < n) ? fabs(a0) : -1.0;
    int bi = lane;
    if (lane + 32 < n) {
        double b = fabs(a1);
        if (b > best) {
            best = b;
            bi = lane + 32;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(FULL_MASK, best, o);
        int oi = __shfl_xor_sync(FULL_MASK, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    return bi;
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ---------------------------------------------------------------- mbarrier / bulk copy

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Returns false if the phase did not complete within the iteration limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t addr = smem_u32(bar);
    for (int it = 0; it < (1 << 26); ++it) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(addr), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------- per-warp linear algebra

// In-place right-looking Cholesky of the packed lower triangle; returns LAPACK info.
template <class S>
__device__ int warp_cholesky_packed(S &sl, int n, int lane)
{
    double *P = sl.L;
    for (int j = 0; j < n; ++j) {
        double ajj = P[pidx(j, j)];
        if (!(ajj > 0.0))
            return j + 1;
        double ljj = sqrt(ajj);
        double r = 1.0 / ljj;
        __syncwarp();
        if (lane == 0)
            P[pidx(j, j)] = ljj;
        for (int i = j + 1 + lane; i < n; i += 32)
            P[pidx(i, j)] *= r;
        __syncwarp();
        // trailing update P(i,k) -= L(i,j) L(k,j), j < k <= i < n, flattened over the warp
        int m = n - j - 1;
        int total = m * (m + 1) / 2;
        int ii = 0, kk = lane;
        while (kk > ii) { // locate element number `lane` in row-major triangle order
            kk -= ii + 1;
            ++ii;
        }
        for (int e = lane; e < total; e += 32) {
            int i = j + 1 + ii, k = j + 1 + kk;
            P[pidx(i, k)] = fma(-P[pidx(i, j)], P[pidx(k, j)], P[pidx(i, k)]);
            kk += 32;
            while (kk > ii) {
                kk -= ii + 1;
                ++ii;
            }
        }
        __syncwarp();
    }
    return 0;
}

// Blocked Cholesky of the tiled lower triangle (Slot<NT, true>); returns LAPACK info.
// Per tile column kb: the 8 columns of the panel (diagonal tile and the tiles below it,
// in registers, lane l holding elements 2l, 2l+1 of each) are factored right-looking with
// warp shuffles; the trailing tiles (ib, jb), kb < jb <= ib, then receive
// -L(ib,kb) L(jb,kb)^T as two m8n8k4 DMMAs each (the panel tiles in operand layout:
// lane l holds L[l/4][4s + l%4] for k-step s, which is the A fragment of L(ib,kb) and the
// B fragment of L(jb,kb)^T).
template <class S>
__device__ int warp_cholesky_tiled(S &sl, int n, int lane)
{
    constexpr int T = S::nt;
    static_assert(sizeof(S) % 16 == 0 && (8 * 8 * S::NMP) % 16 == 0,
                  "tiles must be 16-byte aligned in every slot");
    double *A = sl.L;
    const int r = lane >> 2, q = lane & 3;
    const int c0 = 2 * q, c1 = 2 * q + 1;
    int info = 0;
#pragma unroll
    for (int kb = 0; kb < T; ++kb) {
        double p0[T], p1[T];
#pragma unroll
        for (int t = kb; t < T; ++t) {
            double2 v = *reinterpret_cast<const double2 *>(&A[64 * tix(t, kb) + tpair(lane)]);
            p0[t] = v.x;
            p1[t] = v.y;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            // padding columns (identity rows, zero couplings) would leave their entries
            // unchanged: skip them (warp-uniform)
            if (8 * kb + j >= n)
                break;
            const int src = 4 * j + (j >> 1);
            double ajj = __shfl_sync(FULL_MASK, (j & 1) ? p1[kb] : p0[kb], src);
            // warp-uniform; padding pivots are 1. The loops run to the end (and then hold
            // NaNs) so that they unroll completely and the panel stays in registers.
            if (!(ajj > 0.0) && info == 0)
                info = 8 * kb + j + 1;
            double ljj = sqrt(ajj);
            double rj = 1.0 / ljj;
            // column j: the pivot, then the rows below it scaled by 1/L_jj
            if (q == (j >> 1)) {
                double &dv = (j & 1) ? p1[kb] : p0[kb];
                if (r == j)
                    dv = ljj;
                else if (r > j)
                    dv *= rj;
#pragma unroll
                for (int t = kb + 1; t < T; ++t) {
                    double &v = (j & 1) ? p1[t] : p0[t];
                    v *= rj;
                }
            }
            // L(c, j) of the diagonal tile for this lane's columns c0, c1
            double lc0 = __shfl_sync(FULL_MASK, (j & 1) ? p1[kb] : p0[kb], 4 * c0 + (j >> 1));
            double lc1 = __shfl_sync(FULL_MASK, (j & 1) ? p1[kb] : p0[kb], 4 * c1 + (j >> 1));
#pragma unroll
            for (int t = kb; t < T; ++t) {
                double lrj = __shfl_sync(FULL_MASK, (j & 1) ? p1[t] : p0[t], 4 * r + (j >> 1));
                bool ok0 = c0 > j && (t > kb || c0 <= r);
                bool ok1 = c1 > j && (t > kb || c1 <= r);
                if (ok0)
                    p0[t] = fma(-lrj, lc0, p0[t]);
                if (ok1)
                    p1[t] = fma(-lrj, lc1, p1[t]);
            }
        }
        double f0[T], f1[T];
#pragma unroll
        for (int t = kb; t < T; ++t) {
            *reinterpret_cast<double2 *>(&A[64 * tix(t, kb) + tpair(lane)]) =
                make_double2(p0[t], p1[t]);
            double x0 = __shfl_sync(FULL_MASK, p0[t], 4 * r + (q >> 1));
            double x1 = __shfl_sync(FULL_MASK, p1[t], 4 * r + (q >> 1));
            double y0 = __shfl_sync(FULL_MASK, p0[t], 4 * r + 2 + (q >> 1));
            double y1 = __shfl_sync(FULL_MASK, p1[t], 4 * r + 2 + (q >> 1));
            f0[t] = (q & 1) ? x1 : x0;
            f1[t] = (q & 1) ? y1 : y0;
        }
#pragma unroll
        for (int jb = kb + 1; jb < T; ++jb)
#pragma unroll
            for (int ib = jb; ib < T; ++ib) {
                double2 *cp = reinterpret_cast<double2 *>(&A[64 * tix(ib, jb) + tpair(lane)]);
                double2 c = *cp;
                dmma(c.x, c.y, -f0[ib], f0[jb]);
                dmma(c.x, c.y, -f1[ib], f1[jb]);
                *cp = c;
            }
        __syncwarp();
    }
    return info;
}

template <class S>
__device__ __forceinline__ int warp_cholesky(S &sl, int n, int lane)
{
    if constexpr (S::tiled)
        return warp_cholesky_tiled(sl, n, lane);
    else
        return warp_cholesky_packed(sl, n, lane);
}

// x <- (L L^T)^{-1} x, x distributed as x0 = x[lane], x1 = x[lane+32]; column-oriented
// substitution (the order of the reference BLAS dtrsv and of src/utils.cpp:71-86).
// exactDiv selects division by L_kk (as the reference's own dpotrs) instead of the
// precomputed reciprocal.
template <class S>
__device__ __forceinline__ void warp_apply_inverse_tiled(const S &sl, int lane, double &x0,
                                                         double &x1, double r0, double r1);

template <class S>
__device__ void warp_apply_inverse(const S &sl, int n, int lane, double &x0, double &x1,
                                   bool exactDiv, double r0 = 0.0, double r1 = 0.0)
{
    if constexpr (S::tiled) {
        // the reciprocals serve both the estimate and the direction here: the blocked
        // factor already rounds differently from the reference's unblocked one
        (void)n;
        (void)exactDiv;
        warp_apply_inverse_tiled(sl, lane, x0, x1, r0, r1);
        return;
    }
    const double *P = sl.L;
    for (int k = 0; k < n; ++k) {
        double v = (k < 32) ? x0 : x1;
        double xk = __shfl_sync(FULL_MASK, v, k & 31);
        xk = exactDiv ? xk / P[S::lx(k, k)] : xk * sl.rinv[k];
        if (lane == (k & 31)) {
            if (k < 32)
                x0 = xk;
            else
                x1 = xk;
        }
        if (lane > k && lane < n)
            x0 = fma(-P[S::lx(lane, k)], xk, x0);
        if (lane + 32 > k && lane + 32 < n)
            x1 = fma(-P[S::lx(lane + 32, k)], xk, x1);
    }
    for (int k = n - 1; k >= 0; --k) {
        double v = (k < 32) ? x0 : x1;
        double xk = __shfl_sync(FULL_MASK, v, k & 31);
        xk = exactDiv ? xk / P[S::lx(k, k)] : xk * sl.rinv[k];
        if (lane == (k & 31)) {
            if (k < 32)
                x0 = xk;
            else
                x1 = xk;
        }
        if (lane < k && lane < n)
            x0 = fma(-P[S::lx(k, lane)], xk, x0);
        if (lane + 32 < k && lane + 32 < n)
            x1 = fma(-P[S::lx(k, lane + 32)], xk, x1);
    }
}

// x <- (L L^T)^{-1} x on the tiled factor: tile-blocked substitution. Inside the diagonal
// tile the steps are those of the column-oriented form with the reciprocal pivots r0, r1
// of this lane's rows (lane, lane + 32), held in registers: the row's owner scales it and
// broadcasts the result;
// the tiles off the diagonal act as 8-column mat-vec updates of the rows below (forward) or
// above (backward). Padding rows (L = I there, reciprocal 1) keep finite values and never feed
// the real rows.
template <class S>
__device__ __forceinline__ void warp_apply_inverse_tiled(const S &sl, int lane, double &x0,
                                                         double &x1, double r0, double r1)
{
    constexpr int T = S::nt;
    constexpr int NMP = S::NMP;
    const double *A = sl.L;
#pragma unroll
    for (int kb = 0; kb < T; ++kb) {
        const double *D = A + 64 * tix(kb, kb);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = 8 * kb + i;
            const double xi = __shfl_sync(FULL_MASK, row < 32 ? x0 * r0 : x1 * r1, row & 31);
            if (lane == (row & 31)) {
                if (row < 32)
                    x0 = xi;
                else
                    x1 = xi;
            }
            if (lane > row && lane < 8 * kb + 8)
                x0 = fma(-D[toff(lane - 8 * kb, i)], xi, x0);
            if (lane + 32 > row && lane + 32 < 8 * kb + 8)
                x1 = fma(-D[toff(lane + 32 - 8 * kb, i)], xi, x1);
        }
        if (kb + 1 < T) {
            double y[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                y[c] = __shfl_sync(FULL_MASK, 8 * kb + c < 32 ? x0 : x1, (8 * kb + c) & 31);
            if (lane >= 8 * kb + 8 && lane < NMP) {
                const double *Lt = A + 64 * tix(lane >> 3, kb);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    x0 = fma(-Lt[toff(lane & 7, c)], y[c], x0);
            }
            if (lane + 32 >= 8 * kb + 8 && lane + 32 < NMP) {
                const double *Lt = A + 64 * tix((lane + 32) >> 3, kb);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    x1 = fma(-Lt[toff(lane & 7, c)], y[c], x1);
            }
        }
    }
#pragma unroll
    for (int kb = T - 1; kb >= 0; --kb) {
        const double *D = A + 64 * tix(kb, kb);
#pragma unroll
        for (int i = 7; i >= 0; --i) {
            const int row = 8 * kb + i;
            const double xi = __shfl_sync(FULL_MASK, row < 32 ? x0 * r0 : x1 * r1, row & 31);
            if (lane == (row & 31)) {
                if (row < 32)
                    x0 = xi;
                else
                    x1 = xi;
            }
            if (lane >= 8 * kb && lane < row)
                x0 = fma(-D[toff(i, lane - 8 * kb)], xi, x0);
            if (lane + 32 >= 8 * kb && lane + 32 < row)
                x1 = fma(-D[toff(i, lane + 32 - 8 * kb)], xi, x1);
        }
        if (kb > 0) {
            double y[8];
#pragma unroll
            for (int c = 0; c < 8; ++c)
                y[c] = __shfl_sync(FULL_MASK, 8 * kb + c < 32 ? x0 : x1, (8 * kb + c) & 31);
            if (lane < 8 * kb) {
                const double *Lt = A + 64 * tix(kb, lane >> 3);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    x0 = fma(-Lt[toff(c, lane & 7)], y[c], x0);
            }
            if (lane + 32 < 8 * kb) {
                const double *Lt = A + 64 * tix(kb, (lane + 32) >> 3);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    x1 = fma(-Lt[toff(c, lane & 7)], y[c], x1);
            }
        }
    }
}

__device__ __forceinline__ double vsum_abs(double x0, double x1, int lane, int n)
{
    double s = (lane < n ? fabs(x0) : 0.0) + (lane + 32 < n ? fabs(x1) : 0.0);
    return warp_sum(s);
}

// Hager/Higham 1-norm estimate of (L L^T)^{-1} (N. J. Higham, ACM TOMS 14 (1988)
// 381-396, Alg. 4.1 -- the algorithm of LAPACK's dlacn2 as driven by dpocon).
// Returns 1/rcond with rcond = (1/est)/anorm.
template <class S>
__device__ double warp_condest(const S &sl, int n, int lane, double anorm, double r0 = 0.0,
                               double r1 = 0.0)
{
    if (anorm == 0.0)
        return 1.0 / 0.0;
    double x0 = 1.0 / (double)n, x1 = 1.0 / (double)n;
    warp_apply_inverse(sl, n, lane, x0, x1, false, r0, r1);
    double est;
    if (n == 1) {
        est = fabs(__shfl_sync(FULL_MASK, x0, 0));
    } else {
        est = vsum_abs(x0, x1, lane, n);
        int s0 = x0 >= 0.0 ? 1 : -1, s1 = x1 >= 0.0 ? 1 : -1;
        x0 = (double)s0;
        x1 = (double)s1;
        warp_apply_inverse(sl, n, lane, x0, x1, false, r0, r1);
        int j = warp_iamax(x0, x1, lane, n);
        int iter = 2;
        for (;;) {
            x0 = (lane == j) ? 1.0 : 0.0;
            x1 = (lane + 32 == j) ? 1.0 : 0.0;
            warp_apply_inverse(sl, n, lane, x0, x1, false, r0, r1);
            double estold = est;
            est = vsum_abs(x0, x1, lane, n);
            bool diff = (lane < n && (x0 >= 0.0 ? 1 : -1) != s0) ||
                        (lane + 32 < n && (x1 >= 0.0 ? 1 : -1) != s1);
            bool same = !__any_sync(FULL_MASK, diff);
            if (same || est <= estold)
                break;
            s0 = x0 >= 0.0 ? 1 : -1;
            s1 = x1 >= 0.0 ? 1 : -1;
            x0 = (double)s0;
            x1 = (double)s1;
            warp_apply_inverse(sl, n, lane, x0, x1, false, r0, r1);
            int jlast = j;
            j = warp_iamax(x0, x1, lane, n);
            double xjl = __shfl_sync(FULL_MASK, jlast < 32 ? x0 : x1, jlast & 31);
            double xj = fabs(__shfl_sync(FULL_MASK, j < 32 ? x0 : x1, j & 31));
            if (xjl != xj && iter < 5) {
                ++iter;
                continue;
            }
            break;
        }
        x0 = ((lane & 1) ? -1.0 : 1.0) * (1.0 + (double)lane / (double)(n - 1));
        x1 = (((lane + 32) & 1) ? -1.0 : 1.0) * (1.0 + (double)(lane + 32) / (double)(n - 1));
        warp_apply_inverse(sl, n, lane, x0, x1, false, r0, r1);
        double temp = 2.0 * (vsum_abs(x0, x1, lane, n) / (double)(3 * n));
        if (temp > est)
            est = temp;
    }
    if (est == 0.0)
        return 1.0 / 0.0;
    double rcond = (1.0 / est) / anorm;
    return 1.0 / rcond;
}

__device__ __forceinline__ double warp_nrm2(const double *v, int n, int lane)
{
    double s = 0.0;
    if (lane < n)
        s = v[lane] * v[lane];
    if (lane + 32 < n)
        s = fma(v[lane + 32], v[lane + 32], s);
    return sqrt(warp_sum(s));
}

// ---------------------------------------------------------------- Newton state machine

struct Outputs {
    double *u, *alpha;
    int *iters, *iterGamma, *regIdx, *status;
    unsigned long long *failCount; // cells finishing with a non-zero status
    unsigned long long *stats;     // running counters, layout STAT_* (may be null)
    double *gamma, *normG;         // final gamma and |g| per cell (may be null)
    float *cond;                   // condition estimate of the last Hessian per cell, read at
                                   // set-up as the mixed closure's first precision hint (may be null)
};

template <class S>
__device__ void finalize(S &sl, const ClosureParams &P, const Outputs &O, int lane)
{
    const int nm = P.nm;
    long long c = sl.s.cell;
    __syncwarp();
    if (sl.s.status != CELL_NONPOSITIVE_U0) {
        // postProcess: rescale (src/opt/optBatch.cpp:334-344, src/opt/opt.cpp:352-354)
        for (int i = lane; i < nm; i += 32) {
            O.u[c * nm + i] = sl.u[i] * sl.s.u0;
            double a = sl.alpha[i];
            if (i == 0)
                a = a + sl.s.alphaScale;
            O.alpha[c * nm + i] = a;
        }
    }
    if (lane == 0) {
        if (O.iters) O.iters[c] = sl.s.totalIter;
        if (O.iterGamma) O.iterGamma[c] = sl.s.iterGamma < 0 ? 0 : sl.s.iterGamma;
        if (O.regIdx) O.regIdx[c] = sl.s.regIndex;
        if (O.status) O.status[c] = sl.s.status;
        if (O.gamma) O.gamma[c] = sl.s.gamma;
        if (O.normG) O.normG[c] = sl.s.err;
        if (O.cond) O.cond[c] = (float)sl.s.cnd;
        if (sl.s.status != CELL_OK && O.failCount)
            atomicAdd(O.failCount, 1ull);
        if (O.stats) {
            unsigned long long it = (unsigned long long)sl.s.totalIter;
            unsigned long long ig = (unsigned long long)(sl.s.iterGamma < 0 ? 0 : sl.s.iterGamma);
            atomicAdd(&O.stats[STAT_CELLS], 1ull);
            atomicAdd(&O.stats[STAT_ITERS], it);
            atomicAdd(&O.stats[STAT_ITER_GAMMA], ig);
            atomicMax(&O.stats[STAT_MAX_ITER], it);
            atomicMax(&O.stats[STAT_MAX_ITER_GAMMA], ig);
            if (sl.s.status != CELL_OK)
                atomicAdd(&O.stats[STAT_FAILED], 1ull);
            atomicAdd(&O.stats[STAT_REG_HIST + (sl.s.regIndex & 15)], 1ull);
            atomicAdd(&O.stats[STAT_ITER_HIST + (it < 63 ? it : 63)], 1ull);
        }
        sl.s.need = NEED_NONE;
        sl.s.cell = -1;
    }
    __syncwarp();
}

// Regularise (src/opt/opt.cpp:251-279). Returns false if the ladder is exhausted.
template <class S>
__device__ bool regularize(S &sl, const ClosureParams &P, int lane)
{
    const int nm = P.nm;
    __syncwarp();
    if (sl.s.regIndex >= P.nreg - 1)
        return false;
    int ri = sl.s.regIndex + 1;
    double r = P.reg[ri];
    for (int i = lane; i < nm; i += 32)
        sl.u[i] = (i == 0) ? 1.0 : sl.uOrig[i] * (1.0 - r);
    __syncwarp();
    double rt = P.batched ? P.tol : warp_nrm2(sl.u, nm, lane) * P.tol;
    for (int i = lane; i < nm; i += 32)
        sl.alpha[i] = sl.alpha0[i];
    __syncwarp();
    if (lane == 0) {
        sl.s.regIndex = ri;
        sl.s.r = r;
        sl.s.rtol = rt;
        sl.s.iterGamma = 0;
        sl.s.iter = 0;
        sl.s.t = 1.0;
        if (!P.batched && ri == P.nreg - 1)
            sl.s.maxIter = 10 * sl.s.maxIter;
    }
    __syncwarp();
    return true;
}

// Starts the next Newton iteration. When the iteration is bound to regularise
// whatever H turns out to be (t == 0 after a failed line search, or the
// iteration cap reached), the regularisation is applied here without the H pass.
template <class S>
__device__ void begin_iteration(S &sl, const ClosureParams &P, const Outputs &O, int lane)
{
    for (;;) {
        __syncwarp();
        int maxIterEff = sl.s.maxIter;
        if (P.batched && sl.s.regIndex == P.nreg - 1)
            maxIterEff = 10 * P.maxIter;
        int iter = sl.s.iter + 1, total = sl.s.totalIter + 1;
        long long passes = sl.s.passes + 1;
        __syncwarp();
        if (lane == 0) {
            sl.s.iter = iter;
            sl.s.totalIter = total;
            sl.s.passes = passes;
        }
        __syncwarp();
        if (passes > P.passBudget) {
            if (lane == 0)
                sl.s.status = CELL_PASS_BUDGET;
            finalize(sl, P, O, lane);
            return;
        }
        if (total > 1 && (sl.s.t == 0.0 || iter >= maxIterEff)) {
            if (!regularize(sl, P, lane)) {
                if (lane == 0)
                    sl.s.status = CELL_LADDER_EXHAUSTED;
                finalize(sl, P, O, lane);
                return;
            }
            continue;
        }
        if (lane == 0)
            sl.s.need = (P.probe && total == 1) ? NEED_PROBE : NEED_H;
        __syncwarp();
        return;
    }
}

template <class S>
__device__ void load_cell(S &sl, const ClosureParams &P, const Outputs &O, long long c,
                          int lane)
{
    const int nm = P.nm;
    constexpr int NMP = S::NMP;
    double u0 = O.u[c * nm];
    double alphaScale = log(u0) * 2.0 * sqrt(M_PI);
    for (int i = lane; i < NMP; i += 32) {
        double ui = 0.0, ai = 0.0;
        if (i < nm) {
            ui = O.u[c * nm + i] / u0;
            ai = O.alpha[c * nm + i];
            if (i == 0)
                ai = ai - alphaScale;
        }
        sl.u[i] = ui;
        sl.uOrig[i] = ui;
        sl.alpha[i] = ai;
        sl.alpha0[i] = ai;
        sl.g[i] = 0.0;
        sl.d[i] = 0.0;
    }
    __syncwarp();
    double rt = P.batched ? P.tol : warp_nrm2(sl.u, nm, lane) * P.tol;
    if (lane == 0) {
        sl.s.cell = c;
        sl.s.passes = 0;
        sl.s.u0 = u0;
        sl.s.alphaScale = alphaScale;
        sl.s.rtol = rt;
        sl.s.t = 1.0;
        sl.s.r = 0.0;
        sl.s.gamma = 0.0;
        sl.s.err = 0.0;
        sl.s.iter = 0;
        sl.s.totalIter = 0;
        sl.s.iterGamma = 0;
        sl.s.regIndex = 0;
        sl.s.maxIter = P.maxIter;
        sl.s.status = CELL_OK;
        sl.s.cnd = O.cond ? (double)O.cond[c] : -1.0;
        sl.s.fp64 = 0;
        sl.s.cshift = 0;
        sl.s.hprec = 0;
    }
    __syncwarp();
    if (u0 <= 0) {
        if (lane == 0)
            sl.s.status = CELL_NONPOSITIVE_U0;
        finalize(sl, P, O, lane);
        return;
    }
    begin_iteration(sl, P, O, lane);
}

// Sets alpha = alphaOld + t d and requests a trial pass, or gives up with t = 0.
template <class S>
__device__ void next_trial(S &sl, const ClosureParams &P, const Outputs &O, int lane);

template <class S>
__device__ void next_trial(S &sl, const ClosureParams &P, const Outputs &O, int lane)
{
    const int nm = P.nm;
    double t = sl.s.t;
    __syncwarp();
    if (t * sl.s.maxFactor > EPS_HALF) {
        for (int i = lane; i < nm; i += 32)
            sl.alpha[i] = __dadd_rn(sl.alphaOld[i], __dmul_rn(t, sl.d[i]));
        __syncwarp();
        if (lane == 0) {
            sl.s.need = NEED_TRIAL;
            if (O.stats)
                atomicAdd(&O.stats[STAT_TRIALS], 1ull);
        }
        __syncwarp();
    } else {
        // backtracked all the way (src/opt/linesearch.cpp:76-78)
        for (int i = lane; i < nm; i += 32)
            sl.alpha[i] = sl.alphaOld[i];
        __syncwarp();
        // mixed precision: a direction from a reduced-precision Hessian is not the reference's
        // Newton direction; the iteration is redone from alphaOld with FP64 moments instead of
        // regularising
        const bool redo = P.mixed && sl.s.hprec != 0;
        if (lane == 0) {
            sl.s.t = redo ? 1.0 : 0.0;
            if (redo) {
                sl.s.fp64 = 1;
                if (O.stats)
                    atomicAdd(&O.stats[STAT_ESCALATED], 1ull);
            }
        }
        __syncwarp();
        begin_iteration(sl, P, O, lane);
    }
}

// A reduced-precision Hessian visit is redone with FP64 moments (same iteration); the cell
// keeps FP64 moments for the rest of the closure.
template <class S>
__device__ void escalate_fp64(S &sl, const Outputs &O, int lane)
{
    __syncwarp();
    if (lane == 0) {
        sl.s.fp64 = 1;
        sl.s.passes += 1;
        sl.s.need = NEED_H;
        if (O.stats)
            atomicAdd(&O.stats[STAT_ESCALATED], 1ull);
    }
    __syncwarp();
}

// gext (mixed precision): the FP64 moments <m_i e^{alpha.m}> and fqext = <e^{alpha.m}> of
// the pass, from which g and f are formed instead of from row 0 of the reduced-precision H.
template <class S>
__device__ void after_hessian(S &sl, const ClosureParams &P, const Outputs &O, int lane,
                              double m0, const double *gext = nullptr, double fqext = 0.0)
{
    const int nm = P.nm;
    C3D_NCLK_DECL
    // g_i = H_i0 / m_0 - u_i ; f = H_00 / m_0^2 - alpha.u  (src/opt/fobj.cpp:121-129)
    for (int i = lane; i < nm; i += 32)
        sl.g[i] = gext ? __dsub_rn(gext[i], sl.u[i]) : sl.L[S::lx(i, 0)] / m0 - sl.u[i];
    __syncwarp();
    if (gext && P.mixPolish > 0.0) {
        const double e0 = warp_nrm2(sl.g, nm, lane);
        if (e0 > sl.s.rtol && e0 <= P.mixPolish * sl.s.rtol) {
            escalate_fp64(sl, O, lane);
            return;
        }
    }
    double f = 0.0;
    if (lane == 0) {
        f = gext ? fqext : sl.L[0] / (m0 * m0);
        for (int i = 0; i < nm; ++i)
            f = __dsub_rn(f, __dmul_rn(sl.alpha[i], sl.u[i]));
    }
    f = __shfl_sync(FULL_MASK, f, 0);
    // 1-norm: max row sum of |H| (src/utils.cpp:35-49)
    double rs = 0.0, gmin = 1.0 / 0.0;
    for (int i = lane; i < nm; i += 32) {
        double s = 0.0;
        if constexpr (S::tiled) {
            // row i = the row segments of tiles (ib, jb <= ib) and the column segments of
            // tiles (ib' > ib, ib); padding entries are 0
            const int ib = i >> 3, r = i & 7;
            for (int jb = 0; jb < ib; ++jb) {
                const double *Lt = sl.L + 64 * tix(ib, jb);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    s += fabs(Lt[toff(r, c)]);
            }
            const double *D = sl.L + 64 * tix(ib, ib);
#pragma unroll
            for (int c = 0; c < 8; ++c)
                s += fabs(c <= r ? D[toff(r, c)] : D[toff(c, r)]);
            for (int ib2 = ib + 1; ib2 < S::nt; ++ib2) {
                const double *Lt = sl.L + 64 * tix(ib2, ib);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    s += fabs(Lt[toff(c, r)]);
            }
        } else {
            for (int j = 0; j < nm; ++j)
                s += fabs(j <= i ? sl.L[S::lx(i, j)] : sl.L[S::lx(j, i)]);
        }
        rs = fmax(rs, s);
        gmin = fmin(gmin, 2.0 * sl.L[S::lx(i, i)] - s); // Gershgorin: H_ii - sum_{j!=i} |H_ij|
    }
    double norm1 = warp_max(rs);
    gmin = -warp_max(-gmin);
    // All eigenvalues of H are >= gmin, so when gmin > 0, ||H^-1||_1 <= sqrt(n)/gmin and the
    // 1-norm condition number is at most norm1 sqrt(n)/gmin. The Hager estimate can only be
    // smaller, so if this bound is below condHMax/2 the reference's test `condest > condHMax`
    // is false whatever the estimate; the estimate is then skipped.
    bool condSure = gmin > 0.0 && norm1 * sqrt((double)nm) / gmin <= 0.5 * P.condHMax;
    if (lane == 0) // the condition record: the Gershgorin bound, or the estimate below
        sl.s.cnd = condSure ? norm1 * sqrt((double)nm) / gmin : 0.0;
    __syncwarp();
    C3D_NCLK(O.stats, 1, lane);
    int info = warp_cholesky(sl, nm, lane);
    C3D_NCLK(O.stats, 2, lane);
    double cond = 0.0;
    double r0 = 1.0, r1 = 1.0; // tiled: reciprocal pivots of rows lane, lane + 32
    if (info == 0) {
        if constexpr (S::tiled) {
            if (lane < S::NMP)
                r0 = 1.0 / sl.L[S::lx(lane, lane)];
            if (lane + 32 < S::NMP)
                r1 = 1.0 / sl.L[S::lx(lane + 32, lane + 32)];
        } else {
            for (int i = lane; i < nm; i += 32)
                sl.rinv[i] = 1.0 / sl.L[S::lx(i, i)];
        }
        __syncwarp();
        if (!condSure)
            cond = warp_condest(sl, nm, lane, norm1, r0, r1);
    }
    __syncwarp();
    C3D_NCLK(O.stats, 3, lane);

    if (lane == 0 && (info != 0 || !condSure))
        sl.s.cnd = info != 0 ? 1.0 / 0.0 : cond;
    bool bad = (info != 0) || (cond > P.condHMax);
    if (gext && bad) {
        escalate_fp64(sl, O, lane);
        return;
    }
    if (sl.s.totalIter == 1 && bad) {
        // isotropic restart (src/opt/opt.cpp:236-247)
        double rt = P.batched ? P.tol : warp_nrm2(sl.u, nm, lane) * P.tol;
        for (int i = lane; i < nm; i += 32) {
            double a = (i == 0) ? 2.0 * sqrt(M_PI) * log(0.5 / sqrt(M_PI)) : 0.0;
            sl.alpha0[i] = a;
            sl.alpha[i] = a;
        }
        __syncwarp();
        if (lane == 0) {
            sl.s.rtol = rt;
            sl.s.iter = 0;
            sl.s.iterGamma = 0;
            sl.s.t = 1.0;
        }
        __syncwarp();
        begin_iteration(sl, P, O, lane);
        return;
    }
    int maxIterEff = sl.s.maxIter;
    if (P.batched && sl.s.regIndex == P.nreg - 1)
        maxIterEff = 10 * P.maxIter;
    if (sl.s.iter >= maxIterEff || bad || sl.s.t == 0.0) {
        if (!regularize(sl, P, lane)) {
            if (lane == 0)
                sl.s.status = CELL_LADDER_EXHAUSTED;
            finalize(sl, P, O, lane);
            return;
        }
        begin_iteration(sl, P, O, lane);
        return;
    }
    // d = -H^{-1} g
    double x0 = lane < nm ? sl.g[lane] : 0.0;
    double x1 = lane + 32 < nm ? sl.g[lane + 32] : 0.0;
    warp_apply_inverse(sl, nm, lane, x0, x1, true, r0, r1);
    if (lane < nm)
        sl.d[lane] = -x0;
    if (lane + 32 < nm)
        sl.d[lane + 32] = -x1;
    __syncwarp();
    C3D_NCLK(O.stats, 4, lane);
    double err = warp_nrm2(sl.g, nm, lane);
    double d1 = vsum_abs(x0, x1, lane, nm);
    int pnOrder = (int)floor(sqrt((double)nm)) + 1;
    double minf = sqrt((2 * pnOrder + 1) / (2 * M_PI));
    double gamma = exp(2.0 * d1 * minf);
    double tolEff = sl.s.rtol;
    if (lane == 0) {
        sl.s.err = err;
        sl.s.gamma = gamma;
    }
    __syncwarp();
    if (err <= tolEff && gamma <= P.tolGamma) {
        finalize(sl, P, O, lane);
        return;
    }
    // line search set-up (src/opt/linesearch.cpp:41-54)
    double mf = 0.0;
    for (int i = lane; i < nm; i += 32) {
        sl.alphaOld[i] = sl.alpha[i];
        mf = fmax(mf, fabs(sl.d[i]) / (fabs(sl.alpha[i]) + 1e-100));
    }
    mf = warp_max(mf);
    double gd = 0.0;
    __syncwarp();
    if (lane == 0) {
        for (int i = 0; i < nm; ++i)
            gd = __dadd_rn(gd, __dmul_rn(sl.g[i], sl.d[i]));
        if (err <= tolEff)
            sl.s.iterGamma += 1;
        sl.s.f = f;
        sl.s.maxFactor = mf;
        sl.s.gd = gd;
        sl.s.t = 1.0;
    }
    __syncwarp();
    next_trial(sl, P, O, lane);
}

// First visit of a cell after the probe pass. pm: the probe's entry -- the first-order
// moments mom_i (i < NMP, rows of M2 = the basis), then f's sum, e_min and e_max of
// e^{alpha.m_q}. g is formed as the full visit would form it: FP64 closure, from the Gaunt
// terms of the Hessian's column 0 (g0: g0n terms per row in the reference's CSR order, col
// -2 padding; H_i0 = sum_t v_t mom_col_t, g_i = H_i0 / m_0 - u_i, src/opt/fobj.cpp:121-129);
// mixed closure (g0 null), g_i = mom_i - u_i. The full visit ends the cell converged
// (src/opt/optBatch.cpp:185-250) when info = 0, cond <= condHMax, |g| <= rtol and
// gamma = exp(2 minf |d|_1) <= tolGamma. With lambda_min(H) >= e_min gramLo and
// lambda_max(H) <= e_max gramHi (exact arithmetic; halved for rounding): the 1-norm condition
// estimate is at most nm kappa_2 <= nm e_max gramHi / (e_min gramLo), kept below condHMax / 4
// (Cholesky of such an H succeeds); |d|_1 <= sqrt(nm) |g|_2 / lambda_min, and the gamma
// exponent is kept below half of log(tolGamma). A cell meeting these is finalized with the
// same multipliers, moments and counts as the full visit would give (its gamma record is the
// bound); any other goes on to the Hessian pass of the same iteration.
template <class S>
__device__ void after_probe(S &sl, const ClosureParams &P, const Outputs &O, int lane, double m0,
                            const double *pm, const GauntTerm *g0, int g0n)
{
    const int nm = P.nm;
    constexpr int NMP = S::NMP;
    for (int i = lane; i < nm; i += 32) {
        double gi;
        if (g0) {
            double h = 0.0;
            for (int t = 0; t < g0n; ++t) {
                const GauntTerm e = g0[i * g0n + t];
                if (e.col >= 0)
                    h = __dadd_rn(h, __dmul_rn(pm[e.col], e.v));
            }
            gi = h / m0 - sl.u[i];
        } else {
            gi = __dsub_rn(pm[i], sl.u[i]);
        }
        sl.g[i] = gi;
    }
    __syncwarp();
    const double err = warp_nrm2(sl.g, nm, lane);
    const double emin = pm[NMP + 1], emax = pm[NMP + 2];
    int maxIterEff = sl.s.maxIter;
    if (P.batched && sl.s.regIndex == P.nreg - 1)
        maxIterEff = 10 * P.maxIter;
    bool ok = err <= sl.s.rtol && sl.s.iter < maxIterEff && sl.s.t != 0.0 && P.tolGamma > 1.0 &&
              emin > 0.0 && emax < 1.0 / 0.0 && P.gramLo > 0.0;
    double k1 = 0.0, gexp = 0.0;
    if (ok) {
        const double lam = 0.5 * emin * P.gramLo;
        k1 = nm * (emax * P.gramHi) / lam;
        const int pnOrder = (int)floor(sqrt((double)nm)) + 1;
        const double minf = sqrt((2 * pnOrder + 1) / (2 * M_PI));
        gexp = 2.0 * minf * sqrt((double)nm) * err / lam;
        ok = k1 <= 0.25 * P.condHMax && gexp <= 0.5 * log(P.tolGamma);
    }
    __syncwarp();
    if (ok) {
        if (lane == 0) {
            sl.s.err = err;
            sl.s.gamma = exp(gexp);
            sl.s.cnd = k1;
            if (O.stats)
                atomicAdd(&O.stats[STAT_CERTIFIED], 1ull);
        }
        __syncwarp();
        finalize(sl, P, O, lane);
        return;
    }
    if (lane == 0) {
        sl.s.passes += 1;
        sl.s.need = NEED_H;
        // mixed precision: a gradient already within the polish range would make the
        // reduced-precision Hessian visit of this iteration escalate (after_hessian); the cell
        // goes to the FP64 visit directly, with the same permanent FP64 routing
        if (P.mixed && P.mixPolish > 0.0 && err > sl.s.rtol && err <= P.mixPolish * sl.s.rtol)
            sl.s.fp64 = 1;
    }
    __syncwarp();
}

template <class S>
__device__ void after_trial(S &sl, const ClosureParams &P, const Outputs &O, int lane,
                            double fquad)
{
    const int nm = P.nm;
    double fnew = 0.0;
    if (lane == 0) {
        fnew = fquad;
        for (int i = 0; i < nm; ++i)
            fnew = __dsub_rn(fnew, __dmul_rn(sl.alpha[i], sl.u[i]));
    }
    fnew = __shfl_sync(FULL_MASK, fnew, 0);
    double t = sl.s.t;
    bool accept = fnew <= __dadd_rn(sl.s.f, __dmul_rn(__dmul_rn(1e-3, t), sl.s.gd));
    __syncwarp();
    if (accept) {
        begin_iteration(sl, P, O, lane);
        return;
    }
    if (lane == 0)
        sl.s.t = 0.5 * t;
    __syncwarp();
    next_trial(sl, P, O, lane);
}

} // namespace

} // namespace c3d
