// Plain FP64 M_N dual solve (the drop-in form) as one persistent kernel.
//
// Algorithm: the per-cell Newton iteration of ckrisgarrett/C3D-2015,
//   src/opt/opt.cpp:139-355 (unbatched rules) and
//   src/opt/optBatch.cpp:143-344 (batched rules: absolute MN_TOL, MN_TOL_GAMMA),
// with f, g from row 0 of H (src/opt/fobj.cpp:118-131), Cholesky + 1-norm
// condition estimate (dpotrf_/dpocon_), isotropic restart, regularisation
// ladder, direction by forward/back substitution (src/utils.cpp:71-86),
// gamma = modcfl (src/opt/opt.cpp:117-132) and Armijo backtracking
// (src/opt/linesearch.cpp:29-79).
//
// B200 design:
// * Persistent CTAs, one cell per warp ("slot"); warps pull cells from a
//   device counter, so cells that need more iterations, line-search trials
//   or regularisation never hold up other cells.
// * Every quadrature sum is a "pass" over the basis M in chunks of QC
//   directions, staged into shared memory by the bulk-copy (TMA) engine with
//   an mbarrier pipeline of STAGES buffers; all warps of a CTA share each
//   chunk. In one pass a warp either accumulates its cell's Hessian or its
//   line-search objective, whatever its Newton state needs.
// * H = M^T diag(w e^{M alpha}) M is accumulated on the FP64 tensor pipe
//   (mma.m8n8k4 f64): lower-triangle 8x8 tiles per warp, A = c-scaled basis
//   fragment, B = basis fragment, K = 4 directions per instruction.
// * The exponent alpha.m_q is summed in the reference's order (moment index
//   ascending) with unfused multiply and add.
// * Cholesky, condition estimate and solves run per warp in shared memory
//   (packed lower triangle) with warp shuffles.
#include "c3d_common.cuh"

#include <cfloat>
#include <cstdio>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace c3d {

namespace {

constexpr int STAGES = 3;
constexpr double EPS_HALF = DBL_EPSILON / 2;

enum Need : int { NEED_NONE = 0, NEED_H = 1, NEED_TRIAL = 2 };

struct SlotScalars {
    long long cell;
    long long passes;
    double u0, alphaScale, rtol, f, t, maxFactor, gd, fquad, r, gamma, err;
    int need, iter, totalIter, iterGamma, regIndex, maxIter, status, exhausted;
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

template <int NT> struct Slot {
    static constexpr int NMP = Cfg<NT>::NMP;
    double u[NMP], alpha[NMP], alpha0[NMP], uOrig[NMP], g[NMP], d[NMP], alphaOld[NMP], rinv[NMP];
    double L[Cfg<NT>::NPK];
    SlotScalars s;
};

__device__ __forceinline__ int pidx(int i, int j) { return (i * (i + 1)) / 2 + j; }

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
template <int NT>
__device__ int warp_cholesky(Slot<NT> &sl, int n, int lane)
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

// x <- (L L^T)^{-1} x, x distributed as x0 = x[lane], x1 = x[lane+32]; column-oriented
// substitution (the order of the reference BLAS dtrsv and of src/utils.cpp:71-86).
// exactDiv selects division by L_kk (as the reference's own dpotrs) instead of the
// precomputed reciprocal.
template <int NT>
__device__ void warp_apply_inverse(const Slot<NT> &sl, int n, int lane, double &x0, double &x1,
                                   bool exactDiv)
{
    const double *P = sl.L;
    for (int k = 0; k < n; ++k) {
        double v = (k < 32) ? x0 : x1;
        double xk = __shfl_sync(FULL_MASK, v, k & 31);
        xk = exactDiv ? xk / P[pidx(k, k)] : xk * sl.rinv[k];
        if (lane == (k & 31)) {
            if (k < 32)
                x0 = xk;
            else
                x1 = xk;
        }
        if (lane > k && lane < n)
            x0 = fma(-P[pidx(lane, k)], xk, x0);
        if (lane + 32 > k && lane + 32 < n)
            x1 = fma(-P[pidx(lane + 32, k)], xk, x1);
    }
    for (int k = n - 1; k >= 0; --k) {
        double v = (k < 32) ? x0 : x1;
        double xk = __shfl_sync(FULL_MASK, v, k & 31);
        xk = exactDiv ? xk / P[pidx(k, k)] : xk * sl.rinv[k];
        if (lane == (k & 31)) {
            if (k < 32)
                x0 = xk;
            else
                x1 = xk;
        }
        if (lane < k && lane < n)
            x0 = fma(-P[pidx(k, lane)], xk, x0);
        if (lane + 32 < k && lane + 32 < n)
            x1 = fma(-P[pidx(k, lane + 32)], xk, x1);
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
template <int NT>
__device__ double warp_condest(const Slot<NT> &sl, int n, int lane, double anorm)
{
    if (anorm == 0.0)
        return 1.0 / 0.0;
    double x0 = 1.0 / (double)n, x1 = 1.0 / (double)n;
    warp_apply_inverse(sl, n, lane, x0, x1, false);
    double est;
    if (n == 1) {
        est = fabs(__shfl_sync(FULL_MASK, x0, 0));
    } else {
        est = vsum_abs(x0, x1, lane, n);
        int s0 = x0 >= 0.0 ? 1 : -1, s1 = x1 >= 0.0 ? 1 : -1;
        x0 = (double)s0;
        x1 = (double)s1;
        warp_apply_inverse(sl, n, lane, x0, x1, false);
        int j = warp_iamax(x0, x1, lane, n);
        int iter = 2;
        for (;;) {
            x0 = (lane == j) ? 1.0 : 0.0;
            x1 = (lane + 32 == j) ? 1.0 : 0.0;
            warp_apply_inverse(sl, n, lane, x0, x1, false);
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
            warp_apply_inverse(sl, n, lane, x0, x1, false);
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
        warp_apply_inverse(sl, n, lane, x0, x1, false);
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
};

template <int NT>
__device__ void finalize(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane)
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
template <int NT>
__device__ bool regularize(Slot<NT> &sl, const ClosureParams &P, int lane)
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
template <int NT>
__device__ void begin_iteration(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane)
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
            sl.s.need = NEED_H;
        __syncwarp();
        return;
    }
}

template <int NT>
__device__ void load_cell(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, long long c,
                          int lane)
{
    const int nm = P.nm;
    constexpr int NMP = Cfg<NT>::NMP;
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
template <int NT>
__device__ void next_trial(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane);

template <int NT>
__device__ void next_trial(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane)
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
        if (lane == 0)
            sl.s.t = 0.0;
        __syncwarp();
        begin_iteration(sl, P, O, lane);
    }
}

template <int NT>
__device__ void after_hessian(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane,
                              double m0)
{
    const int nm = P.nm;
    // g_i = H_i0 / m_0 - u_i ; f = H_00 / m_0^2 - alpha.u  (src/opt/fobj.cpp:121-129)
    for (int i = lane; i < nm; i += 32)
        sl.g[i] = sl.L[pidx(i, 0)] / m0 - sl.u[i];
    __syncwarp();
    double f = 0.0;
    if (lane == 0) {
        f = sl.L[0] / (m0 * m0);
        for (int i = 0; i < nm; ++i)
            f = __dsub_rn(f, __dmul_rn(sl.alpha[i], sl.u[i]));
    }
    f = __shfl_sync(FULL_MASK, f, 0);
    // 1-norm: max row sum of |H| (src/utils.cpp:35-49)
    double rs = 0.0, gmin = 1.0 / 0.0;
    for (int i = lane; i < nm; i += 32) {
        double s = 0.0;
        for (int j = 0; j < nm; ++j)
            s += fabs(j <= i ? sl.L[pidx(i, j)] : sl.L[pidx(j, i)]);
        rs = fmax(rs, s);
        gmin = fmin(gmin, 2.0 * sl.L[pidx(i, i)] - s); // Gershgorin: H_ii - sum_{j!=i} |H_ij|
    }
    double norm1 = warp_max(rs);
    gmin = -warp_max(-gmin);
    // All eigenvalues of H are >= gmin, so when gmin > 0, ||H^-1||_1 <= sqrt(n)/gmin and the
    // 1-norm condition number is at most norm1 sqrt(n)/gmin. The Hager estimate can only be
    // smaller, so if this bound is below condHMax/2 the reference's test `condest > condHMax`
    // is false whatever the estimate; the estimate is then skipped.
    bool condSure = gmin > 0.0 && norm1 * sqrt((double)nm) / gmin <= 0.5 * P.condHMax;
    __syncwarp();
    int info = warp_cholesky(sl, nm, lane);
    double cond = 0.0;
    if (info == 0) {
        for (int i = lane; i < nm; i += 32)
            sl.rinv[i] = 1.0 / sl.L[pidx(i, i)];
        __syncwarp();
        if (!condSure)
            cond = warp_condest(sl, nm, lane, norm1);
    }
    __syncwarp();

    bool bad = (info != 0) || (cond > P.condHMax);
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
    warp_apply_inverse(sl, nm, lane, x0, x1, true);
    if (lane < nm)
        sl.d[lane] = -x0;
    if (lane + 32 < nm)
        sl.d[lane + 32] = -x1;
    __syncwarp();
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

template <int NT>
__device__ void after_trial(Slot<NT> &sl, const ClosureParams &P, const Outputs &O, int lane,
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

// ---------------------------------------------------------------- kernel

template <int NT, int W>
__global__ void __launch_bounds__(W * 32, 1)
    closure_fp64_kernel(ClosureParams P, const double *__restrict__ chunks, long long ncells,
                        unsigned long long *counter, Outputs O, int *errorFlag)
{
    constexpr int NMP = Cfg<NT>::NMP;
    constexpr int CH = Cfg<NT>::CHUNK;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *stage = reinterpret_cast<double *>(smem_raw);
    Slot<NT> *slots = reinterpret_cast<Slot<NT> *>(stage + STAGES * CH);
    uint64_t *full = reinterpret_cast<uint64_t *>(slots + W);
    __shared__ int s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nm = P.nm, nchunks = P.nchunks;
    const uint32_t chunkBytes = CH * sizeof(double);
    Slot<NT> &sl = slots[warp];
    const double m0 = chunks[0]; // M[0][0], the constant harmonic 1/(2 sqrt(pi))

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s)
            mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
    }
    if (lane == 0) {
        sl.s.need = NEED_NONE;
        sl.s.cell = -1;
        sl.s.exhausted = 0;
    }
    __syncthreads();

    uint32_t seq = 0; // chunks consumed so far by this CTA (uniform)
    for (;;) {
        // refill an empty slot from the device work queue
        if (sl.s.need == NEED_NONE && !sl.s.exhausted) {
            for (;;) {
                unsigned long long c = 0;
                if (lane == 0)
                    c = atomicAdd(counter, 1ull);
                c = __shfl_sync(FULL_MASK, c, 0);
                if ((long long)c >= ncells) {
                    if (lane == 0)
                        sl.s.exhausted = 1;
                    __syncwarp();
                    break;
                }
                load_cell(sl, P, O, (long long)c, lane);
                if (sl.s.need != NEED_NONE)
                    break;
            }
        }
        __syncwarp();
        const int need = sl.s.need;
        if (!__syncthreads_or(need != NEED_NONE))
            break;

        // ------------------------------------------------ one pass over the basis
        double acc[Cfg<NT>::NTILE][2];
#pragma unroll
        for (int t = 0; t < Cfg<NT>::NTILE; ++t)
            acc[t][0] = acc[t][1] = 0.0;
        double fpart = 0.0;

        if (tid == 0) {
            for (int k = 0; k < STAGES && k < nchunks; ++k) {
                uint32_t s = (seq + k) % STAGES;
                mbar_expect_tx(&full[s], chunkBytes);
                bulk_g2s(stage + s * CH, chunks + (size_t)k * CH, chunkBytes, &full[s]);
            }
        }
        for (int k = 0; k < nchunks; ++k) {
            uint32_t s = (seq + k) % STAGES;
            uint32_t parity = ((seq + k) / STAGES) & 1u;
            if (!mbar_wait(&full[s], parity))
                s_abort = 1;
            if (__syncthreads_or(s_abort)) {
                if (tid == 0)
                    atomicExch(errorFlag, 1);
                return;
            }
            const double *ch = stage + s * CH;
            if (need != NEED_NONE) {
                // exponent alpha . m_q for q = k*QC + lane, moment index ascending, unfused
                double z = 0.0;
                for (int i = 0; i < nm; ++i)
                    z = __dadd_rn(z, __dmul_rn(sl.alpha[i], ch[i * QCP + lane]));
                double e = exp(z);
                double wq = ch[NMP * QCP + lane];
                if (need == NEED_TRIAL) {
                    fpart += wq * e;
                } else {
                    double c = wq * e;
#pragma unroll
                    for (int g = 0; g < QC / 4; ++g) {
                        double cq = __shfl_sync(FULL_MASK, c, 4 * g + (lane & 3));
                        double m[NT], a[NT];
#pragma unroll
                        for (int I = 0; I < NT; ++I) {
                            m[I] = ch[(8 * I + (lane >> 2)) * QCP + 4 * g + (lane & 3)];
                            a[I] = cq * m[I];
                        }
#pragma unroll
                        for (int I = 0; I < NT; ++I)
#pragma unroll
                            for (int J = 0; J <= I; ++J)
                                dmma(acc[I * (I + 1) / 2 + J][0], acc[I * (I + 1) / 2 + J][1], a[I],
                                     m[J]);
                    }
                }
            }
            __syncthreads();
            if (tid == 0 && k + STAGES < nchunks) {
                mbar_expect_tx(&full[s], chunkBytes);
                bulk_g2s(stage + s * CH, chunks + (size_t)(k + STAGES) * CH, chunkBytes, &full[s]);
            }
        }
        seq += nchunks;

        // ------------------------------------------------ per-warp Newton logic
        if (need == NEED_H) {
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J) {
                    int row = 8 * I + (lane >> 2);
#pragma unroll
                    for (int e2 = 0; e2 < 2; ++e2) {
                        int col = 8 * J + 2 * (lane & 3) + e2;
                        if (row < nm && col < nm && col <= row)
                            sl.L[pidx(row, col)] = acc[I * (I + 1) / 2 + J][e2];
                    }
                }
            __syncwarp();
            after_hessian(sl, P, O, lane, m0);
        } else if (need == NEED_TRIAL) {
            double fq = warp_sum(fpart);
            after_trial(sl, P, O, lane, fq);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- Gaunt-form closure

// The same per-cell Newton logic with H formed as in the reference's Gaunt modes
// (src/opt/fobj.cpp:58-61, :75-95): extended moments mom_k = sum_q w_q e^{alpha.m_q} m2_qk
// for the nm2 = (2N+1)^2 harmonics of degree <= 2N, then H_ij = sum_k beta_ijk mom_k over
// the CSR table (|beta| > 1e-13 for the sparse mode, all nonzeros for the dense mode),
// summed in the reference's order. Per chunk, each warp computes its cell's exponents
// and writes the coefficients c_q = w_q e_q into a shared [q][cell] tile; then all warps
// accumulate the moments of the CTA's W = 8 cells as one DMMA GEMM
// (moments[k][cell] += M2^T[k][q] C[q][cell]) with the staged M2^T chunk as the shared
// operand: ~7x fewer FLOPs than the direct lower triangle for M_6.
constexpr int GSTAGES = 2;
constexpr int CST = 12; // row stride of the coefficient tile (bank-conflict-free B fragments)

template <int NT, int NT2, int W>
__global__ void __launch_bounds__(W * 32, 1)
    closure_gaunt_kernel(ClosureParams P, const double *__restrict__ chunks, long long ncells,
                         unsigned long long *counter, Outputs O, int *errorFlag,
                         const int *__restrict__ bRow, const int *__restrict__ bCol,
                         const double *__restrict__ bVal)
{
    static_assert(W == 8, "the moment GEMM uses one 8-wide DMMA column tile of cells");
    constexpr int NM2P = 8 * NT2;
    constexpr int CH = (NM2P + 1) * QCP;
    constexpr int RT = (NT2 + W - 1) / W;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *stage = reinterpret_cast<double *>(smem_raw);
    Slot<NT> *slots = reinterpret_cast<Slot<NT> *>(stage + GSTAGES * CH);
    double *mom = reinterpret_cast<double *>(slots + W); // W x NM2P
    double *cbuf = mom + W * NM2P;                        // QC x CST
    uint64_t *full = reinterpret_cast<uint64_t *>(cbuf + QC * CST);
    __shared__ int s_abort;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nm = P.nm, nchunks = P.nchunks;
    const uint32_t chunkBytes = CH * sizeof(double);
    Slot<NT> &sl = slots[warp];
    const double m0 = chunks[0];
    const int npk = nm * (nm + 1) / 2;

    if (tid == 0) {
        for (int s = 0; s < GSTAGES; ++s)
            mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
    }
    if (lane == 0) {
        sl.s.need = NEED_NONE;
        sl.s.cell = -1;
        sl.s.exhausted = 0;
    }
    __syncthreads();

    uint32_t seq = 0;
    for (;;) {
        if (sl.s.need == NEED_NONE && !sl.s.exhausted) {
            for (;;) {
                unsigned long long c = 0;
                if (lane == 0)
                    c = atomicAdd(counter, 1ull);
                c = __shfl_sync(FULL_MASK, c, 0);
                if ((long long)c >= ncells) {
                    if (lane == 0)
                        sl.s.exhausted = 1;
                    __syncwarp();
                    break;
                }
                load_cell(sl, P, O, (long long)c, lane);
                if (sl.s.need != NEED_NONE)
                    break;
            }
        }
        __syncwarp();
        const int need = sl.s.need;
        if (!__syncthreads_or(need != NEED_NONE))
            break;
        const bool anyH = __syncthreads_or(need == NEED_H);

        double acc[RT][2];
#pragma unroll
        for (int r = 0; r < RT; ++r)
            acc[r][0] = acc[r][1] = 0.0;
        double fpart = 0.0;
        if (tid == 0) {
            for (int k = 0; k < GSTAGES && k < nchunks; ++k) {
                uint32_t s = (seq + k) % GSTAGES;
                mbar_expect_tx(&full[s], chunkBytes);
                bulk_g2s(stage + s * CH, chunks + (size_t)k * CH, chunkBytes, &full[s]);
            }
        }
        for (int k = 0; k < nchunks; ++k) {
            uint32_t s = (seq + k) % GSTAGES;
            uint32_t parity = ((seq + k) / GSTAGES) & 1u;
            if (!mbar_wait(&full[s], parity))
                s_abort = 1;
            if (__syncthreads_or(s_abort)) {
                if (tid == 0)
                    atomicExch(errorFlag, 1);
                return;
            }
            const double *ch = stage + s * CH;
            double c = 0.0;
            if (need != NEED_NONE) {
                double z = 0.0;
                for (int i = 0; i < nm; ++i)
                    z = __dadd_rn(z, __dmul_rn(sl.alpha[i], ch[i * QCP + lane]));
                c = ch[NM2P * QCP + lane] * exp(z);
                if (need == NEED_TRIAL)
                    fpart += c;
            }
            cbuf[lane * CST + warp] = (need == NEED_H) ? c : 0.0;
            __syncthreads();
            if (anyH) {
#pragma unroll
                for (int g = 0; g < QC / 4; ++g) {
                    double b = cbuf[(4 * g + (lane & 3)) * CST + (lane >> 2)];
#pragma unroll
                    for (int r = 0; r < RT; ++r) {
                        int rt = warp + r * W;
                        if (rt < NT2) {
                            double a = ch[(8 * rt + (lane >> 2)) * QCP + 4 * g + (lane & 3)];
                            dmma(acc[r][0], acc[r][1], a, b);
                        }
                    }
                }
            }
            __syncthreads();
            if (tid == 0 && k + GSTAGES < nchunks) {
                mbar_expect_tx(&full[s], chunkBytes);
                bulk_g2s(stage + s * CH, chunks + (size_t)(k + GSTAGES) * CH, chunkBytes, &full[s]);
            }
        }
        seq += nchunks;

        if (anyH) {
#pragma unroll
            for (int r = 0; r < RT; ++r) {
                int rt = warp + r * W;
                if (rt < NT2) {
                    int kk = 8 * rt + (lane >> 2), c0 = 2 * (lane & 3);
                    mom[c0 * NM2P + kk] = acc[r][0];
                    mom[(c0 + 1) * NM2P + kk] = acc[r][1];
                }
            }
        }
        __syncthreads();
        if (need == NEED_H) {
            // H_ij (i >= j) = sum over the CSR row of (j, i) of mom[col] * val, in CSR order
            const double *mw = mom + warp * NM2P;
            int ii = 0, jj = lane;
            while (jj > ii) {
                jj -= ii + 1;
                ++ii;
            }
            for (int e = lane; e < npk; e += 32) {
                int idx = jj * nm + ii;
                double h = 0.0;
                for (int t = bRow[idx]; t < bRow[idx + 1]; ++t)
                    h = __dadd_rn(h, __dmul_rn(mw[bCol[t]], bVal[t]));
                sl.L[e] = h;
                jj += 32;
                while (jj > ii) {
                    jj -= ii + 1;
                    ++ii;
                }
            }
            __syncwarp();
            after_hessian(sl, P, O, lane, m0);
        } else if (need == NEED_TRIAL) {
            double fq = warp_sum(fpart);
            after_trial(sl, P, O, lane, fq);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- batched Hessians

// H_b = sum_q w_q exp(alpha_b . m_q) m_q m_q^T for a batch of multiplier vectors
// (the quantity of src/opt/fobj.cpp:34-102 in its direct form; the reference's
// solveH_cuda). One warp per vector, same staged-chunk DMMA pass as the closure.
template <int NT, int W>
__global__ void __launch_bounds__(W * 32, 1)
    hessian_batch_kernel(int nm, int nchunks, const double *__restrict__ chunks,
                         const double *__restrict__ alphas, long long n, double *__restrict__ hs,
                         int *errorFlag)
{
    constexpr int NMP = Cfg<NT>::NMP;
    constexpr int CH = Cfg<NT>::CHUNK;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *stage = reinterpret_cast<double *>(smem_raw);
    double *sAlpha = stage + STAGES * CH; // W x NMP
    uint64_t *full = reinterpret_cast<uint64_t *>(sAlpha + W * NMP);
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long b = (long long)blockIdx.x * W + warp;
    const bool valid = b < n;
    const uint32_t chunkBytes = CH * sizeof(double);
    for (int i = lane; i < NMP; i += 32)
        sAlpha[warp * NMP + i] = (valid && i < nm) ? alphas[b * nm + i] : 0.0;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s)
            mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
        for (int k = 0; k < STAGES && k < nchunks; ++k) {
            mbar_expect_tx(&full[k], chunkBytes);
            bulk_g2s(stage + k * CH, chunks + (size_t)k * CH, chunkBytes, &full[k]);
        }
    }
    __syncthreads();
    double acc[Cfg<NT>::NTILE][2];
#pragma unroll
    for (int t = 0; t < Cfg<NT>::NTILE; ++t)
        acc[t][0] = acc[t][1] = 0.0;
    const double *al = sAlpha + warp * NMP;
    for (int k = 0; k < nchunks; ++k) {
        uint32_t s = k % STAGES, parity = (k / STAGES) & 1u;
        if (!mbar_wait(&full[s], parity))
            s_abort = 1;
        if (__syncthreads_or(s_abort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *ch = stage + s * CH;
        double z = 0.0;
        for (int i = 0; i < nm; ++i)
            z = __dadd_rn(z, __dmul_rn(al[i], ch[i * QCP + lane]));
        double c = ch[NMP * QCP + lane] * exp(z);
#pragma unroll
        for (int g = 0; g < QC / 4; ++g) {
            double cq = __shfl_sync(FULL_MASK, c, 4 * g + (lane & 3));
            double m[NT], a[NT];
#pragma unroll
            for (int I = 0; I < NT; ++I) {
                m[I] = ch[(8 * I + (lane >> 2)) * QCP + 4 * g + (lane & 3)];
                a[I] = cq * m[I];
            }
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J)
                    dmma(acc[I * (I + 1) / 2 + J][0], acc[I * (I + 1) / 2 + J][1], a[I], m[J]);
        }
        __syncthreads();
        if (tid == 0 && k + STAGES < nchunks) {
            mbar_expect_tx(&full[s], chunkBytes);
            bulk_g2s(stage + s * CH, chunks + (size_t)(k + STAGES) * CH, chunkBytes, &full[s]);
        }
    }
    if (!valid)
        return;
    double *H = hs + b * (long long)nm * nm;
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J) {
            int row = 8 * I + (lane >> 2);
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2) {
                int col = 8 * J + 2 * (lane & 3) + e2;
                if (row < nm && col < nm && col <= row) {
                    double v = acc[I * (I + 1) / 2 + J][e2];
                    H[row * nm + col] = v;
                    H[col * nm + row] = v;
                }
            }
        }
}

// ---------------------------------------------------------------- host launcher

struct ClosureLaunch {
    const ClosureParams *P;
    const double *chunks;
    long long ncells;
    unsigned long long *counter;
    double *u, *alpha;
    int *iters, *iterGamma, *regIdx, *status;
    unsigned long long *failCount;
    unsigned long long *stats;
    int *errorFlag;
    int numSMs;
    cudaStream_t stream;
};

template <int NT, int W> static size_t closure_smem_bytes()
{
    return STAGES * Cfg<NT>::CHUNK * sizeof(double) + W * sizeof(Slot<NT>) + STAGES * sizeof(uint64_t);
}

template <int NT, int W> static cudaError_t launch_closure_t(const ClosureLaunch &L)
{
    size_t smem = closure_smem_bytes<NT, W>();
    auto kern = closure_fp64_kernel<NT, W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    Outputs O{L.u, L.alpha, L.iters, L.iterGamma, L.regIdx, L.status, L.failCount, L.stats};
    long long maxCtas = (L.ncells + W - 1) / W;
    int grid = L.numSMs;
    if (maxCtas < grid)
        grid = (int)maxCtas;
    if (grid < 1)
        grid = 1;
    e = cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), L.stream);
    if (e != cudaSuccess)
        return e;
    kern<<<grid, W * 32, smem, L.stream>>>(*L.P, L.chunks, L.ncells, L.counter, O, L.errorFlag);
    return cudaGetLastError();
}

// Padded moment count (rows of the staged basis) used for nm.
int closure_fp64_nmp(int nm)
{
    int nt = (nm + 7) / 8;
    return 8 * nt;
}

struct GauntTables {
    const double *chunks; // (NM2P + 1) x QCP per chunk
    const int *row, *col;
    const double *val;
};

template <int NT, int NT2>
static cudaError_t launch_gaunt_t(const ClosureLaunch &L, const GauntTables &G)
{
    constexpr int W = 8;
    constexpr int NM2P = 8 * NT2;
    size_t smem = GSTAGES * (size_t)(NM2P + 1) * QCP * sizeof(double) + W * sizeof(Slot<NT>) +
                  (size_t)W * NM2P * sizeof(double) + (size_t)QC * CST * sizeof(double) +
                  GSTAGES * sizeof(uint64_t);
    auto kern = closure_gaunt_kernel<NT, NT2, W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    Outputs O{L.u, L.alpha, L.iters, L.iterGamma, L.regIdx, L.status, L.failCount, L.stats};
    long long maxCtas = (L.ncells + W - 1) / W;
    int grid = L.numSMs;
    if (maxCtas < grid)
        grid = (int)maxCtas;
    if (grid < 1)
        grid = 1;
    e = cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), L.stream);
    if (e != cudaSuccess)
        return e;
    kern<<<grid, W * 32, smem, L.stream>>>(*L.P, G.chunks, L.ncells, L.counter, O, L.errorFlag,
                                            G.row, G.col, G.val);
    return cudaGetLastError();
}

// Moment counts with a Gaunt-form kernel (N <= 6).
bool closure_gaunt_supported(int nm) { return nm == 1 || nm == 4 || nm == 9 || nm == 16 || nm == 25 || nm == 36 || nm == 49; }

cudaError_t launch_closure_gaunt(const ClosureLaunch &L, const GauntTables &G)
{
    switch (L.P->nm) {
    case 1: return launch_gaunt_t<1, 1>(L, G);
    case 4: return launch_gaunt_t<1, 2>(L, G);
    case 9: return launch_gaunt_t<2, 4>(L, G);
    case 16: return launch_gaunt_t<2, 7>(L, G);
    case 25: return launch_gaunt_t<4, 11>(L, G);
    case 36: return launch_gaunt_t<5, 16>(L, G);
    case 49: return launch_gaunt_t<7, 22>(L, G);
    default: return cudaErrorInvalidValue;
    }
}

// Rows of the Gaunt chunk (8 * ceil(nm2/8) harmonics + weights).
int closure_gaunt_nm2p(int nm2) { return 8 * ((nm2 + 7) / 8); }

template <int NT, int W>
static cudaError_t launch_hessian_t(int nm, int nchunks, const double *chunks, const double *alphas,
                                   long long n, double *hs, int *errorFlag, cudaStream_t st)
{
    size_t smem = STAGES * Cfg<NT>::CHUNK * sizeof(double) + W * Cfg<NT>::NMP * sizeof(double) +
                  STAGES * sizeof(uint64_t);
    auto kern = hessian_batch_kernel<NT, W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    long long grid = (n + W - 1) / W;
    if (grid < 1)
        return cudaSuccess;
    kern<<<(unsigned)grid, W * 32, smem, st>>>(nm, nchunks, chunks, alphas, n, hs, errorFlag);
    return cudaGetLastError();
}

cudaError_t launch_hessian_batch(int nm, int nchunks, const double *chunks, const double *alphas,
                                 long long n, double *hs, int *errorFlag, cudaStream_t st)
{
    switch ((nm + 7) / 8) {
    case 1: return launch_hessian_t<1, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 2: return launch_hessian_t<2, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 3: return launch_hessian_t<3, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 4: return launch_hessian_t<4, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 5: return launch_hessian_t<5, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 6: return launch_hessian_t<6, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 7: return launch_hessian_t<7, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    case 8: return launch_hessian_t<8, 8>(nm, nchunks, chunks, alphas, n, hs, errorFlag, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_closure_fp64(const ClosureLaunch &L)
{
    int nt = (L.P->nm + 7) / 8;
    switch (nt) {
    case 1: return launch_closure_t<1, 8>(L);
    case 2: return launch_closure_t<2, 8>(L);
    case 3: return launch_closure_t<3, 8>(L);
    case 4: return launch_closure_t<4, 8>(L);
    case 5: return launch_closure_t<5, 8>(L);
    case 6: return launch_closure_t<6, 8>(L);
    case 7: return launch_closure_t<7, 8>(L);
    case 8: return launch_closure_t<8, 6>(L);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace c3d
