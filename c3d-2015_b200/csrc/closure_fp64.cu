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

#include <cstdio>

#include "closure_core.cuh"

namespace c3d {


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
        long long tc0 = clock64();
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
        long long tc1 = clock64();

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
                // c = w_q e^{z}; rounded product, then an unfused running sum (the same in
                // every engine, whatever the compiler would contract)
                double c = __dmul_rn(ch[NMP * QCP + lane], exp(z));
                if (need == NEED_TRIAL) {
                    fpart = __dadd_rn(fpart, c);
                } else {
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
        long long tc2 = clock64();

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
        if (lane == 0 && O.stats) {
            long long tc3 = clock64();
            atomicAdd(&O.stats[STAT_CLK_REFILL], (unsigned long long)(tc1 - tc0));
            atomicAdd(&O.stats[STAT_CLK_PASS], (unsigned long long)(tc2 - tc1));
            atomicAdd(&O.stats[STAT_CLK_SERIAL], (unsigned long long)(tc3 - tc2));
            if (warp == 0)
                atomicAdd(&O.stats[STAT_PASSES], 1ull);
        }
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
        long long tc0 = clock64();
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
        long long tc1 = clock64();
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
                c = __dmul_rn(ch[NM2P * QCP + lane], exp(z));
                if (need == NEED_TRIAL)
                    fpart = __dadd_rn(fpart, c);
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
        long long tc2 = clock64();

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
        if (lane == 0 && O.stats) {
            long long tc3 = clock64();
            atomicAdd(&O.stats[STAT_CLK_REFILL], (unsigned long long)(tc1 - tc0));
            atomicAdd(&O.stats[STAT_CLK_PASS], (unsigned long long)(tc2 - tc1));
            atomicAdd(&O.stats[STAT_CLK_SERIAL], (unsigned long long)(tc3 - tc2));
            if (warp == 0)
                atomicAdd(&O.stats[STAT_PASSES], 1ull);
        }
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

// Gaunt-form batched Hessians (src/opt/fobj.cpp:34-102 with useGaunt; the reference's
// solveH_cuda with useGaunt = 1, src/cuda/cuda_solveH.cu:224-241). Eight vectors per CTA:
// per staged chunk of QC directions each warp forms one vector's w_q e^{alpha.m_q} (exponent
// summed in the reference's order, unfused), then the extended moments
// mom_k = sum_q w_q e^{alpha.m_q} p2_qk accumulate on the FP64 tensor pipe as an
// [8 vectors x nm2p] tile (A = the weights, B = the staged p2 rows; each warp owns every
// eighth 8-column tile). H_ij = sum_k beta_ijk mom_k follows for j >= i and is mirrored, as
// the CPU path does: over all nm2 harmonics in ascending order (dense beta, stored
// transposed, betaT[k nm^2 + i nm + j]) or over the CSR row of (i, j) in its order.
// Chunk layout (rows of QCP doubles): the nm rows of M^T, the nm2p rows of M2^T (zero past
// nm2), the weight row.
template <int TPW>
__global__ void __launch_bounds__(256, 1)
    gaunt_batch_kernel(int nm, int nm2, int nm2p, int nchunks, const double *__restrict__ chunks,
                       const double *__restrict__ alphas, long long n,
                       const double *__restrict__ betaT, const int *__restrict__ rowPtr,
                       const int *__restrict__ colInd, const double *__restrict__ val, int sparse,
                       double *__restrict__ hs, int *errorFlag)
{
    constexpr int GB = 8; // vectors per CTA: the DMMA row tile
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int CH = (nm + nm2p + 1) * QCP;
    double *stage = reinterpret_cast<double *>(smem_raw); // GSTAGES chunks
    double *sAlpha = stage + GSTAGES * CH;                 // GB x nm
    double *sT = sAlpha + GB * nm;                         // GB x QCP weights of the chunk
    double *sMom = sT + GB * QCP;                          // GB x nm2p extended moments
    uint64_t *full = reinterpret_cast<uint64_t *>(sMom + GB * nm2p);
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long b0 = (long long)blockIdx.x * GB;
    const uint32_t chunkBytes = CH * sizeof(double);
    const int ntiles = nm2p / 8;
    for (int e = tid; e < GB * nm; e += blockDim.x) {
        long long b = b0 + e / nm;
        sAlpha[e] = b < n ? alphas[b * nm + e % nm] : 0.0;
    }
    if (tid == 0) {
        for (int s = 0; s < GSTAGES; ++s)
            mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
        for (int k = 0; k < GSTAGES && k < nchunks; ++k) {
            mbar_expect_tx(&full[k], chunkBytes);
            bulk_g2s(stage + k * CH, chunks + (size_t)k * CH, chunkBytes, &full[k]);
        }
    }
    __syncthreads();
    double acc[TPW][2];
#pragma unroll
    for (int t = 0; t < TPW; ++t)
        acc[t][0] = acc[t][1] = 0.0;
    for (int k = 0; k < nchunks; ++k) {
        uint32_t s = k % GSTAGES, parity = (k / GSTAGES) & 1u;
        if (!mbar_wait(&full[s], parity))
            s_abort = 1;
        if (__syncthreads_or(s_abort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *ch = stage + s * CH;
        {
            const double *al = sAlpha + warp * nm;
            double z = 0.0;
            for (int i = 0; i < nm; ++i)
                z = __dadd_rn(z, __dmul_rn(al[i], ch[i * QCP + lane]));
            sT[warp * QCP + lane] = exp(z) * ch[(nm + nm2p) * QCP + lane];
        }
        __syncthreads();
#pragma unroll
        for (int g = 0; g < QC / 4; ++g) {
            double a = sT[(lane >> 2) * QCP + 4 * g + (lane & 3)];
#pragma unroll
            for (int t = 0; t < TPW; ++t) {
                int j = warp + 8 * t;
                if (j < ntiles)
                    dmma(acc[t][0], acc[t][1], a,
                         ch[(nm + 8 * j + (lane >> 2)) * QCP + 4 * g + (lane & 3)]);
            }
        }
        __syncthreads();
        if (tid == 0 && k + GSTAGES < nchunks) {
            mbar_expect_tx(&full[s], chunkBytes);
            bulk_g2s(stage + s * CH, chunks + (size_t)(k + GSTAGES) * CH, chunkBytes, &full[s]);
        }
    }
#pragma unroll
    for (int t = 0; t < TPW; ++t) {
        int j = warp + 8 * t;
        if (j < ntiles) {
            int col = 8 * j + 2 * (lane & 3);
            sMom[(lane >> 2) * nm2p + col] = acc[t][0];
            sMom[(lane >> 2) * nm2p + col + 1] = acc[t][1];
        }
    }
    __syncthreads();
    const int nmm = nm * nm;
    for (int e = tid; e < GB * nmm; e += blockDim.x) {
        int c = e / nmm, ij = e % nmm, i = ij / nm, j = ij % nm;
        long long b = b0 + c;
        if (b >= n || j < i)
            continue;
        const double *mom = sMom + c * nm2p;
        double h = 0.0;
        if (sparse) {
            for (int p = rowPtr[ij]; p < rowPtr[ij + 1]; ++p)
                h = __dadd_rn(h, __dmul_rn(mom[colInd[p]], val[p]));
        } else {
            for (int kk = 0; kk < nm2; ++kk)
                h = __dadd_rn(h, __dmul_rn(mom[kk], betaT[(size_t)kk * nmm + ij]));
        }
        double *H = hs + b * (long long)nmm;
        H[i * nm + j] = h;
        H[j * nm + i] = h;
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
    double *gamma, *normG; // per-cell final gamma and |g| (may be null)
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
    Outputs O{L.u,      L.alpha,     L.iters, L.iterGamma, L.regIdx,
              L.status, L.failCount, L.stats, L.gamma,     L.normG};
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
    Outputs O{L.u,      L.alpha,     L.iters, L.iterGamma, L.regIdx,
              L.status, L.failCount, L.stats, L.gamma,     L.normG};
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

// Shared memory of gaunt_batch_kernel (0 if the sizes do not fit).
size_t gaunt_batch_smem(int nm, int nm2p)
{
    size_t b = ((size_t)GSTAGES * (nm + nm2p + 1) * QCP + 8 * (size_t)(nm + QCP + nm2p)) *
                   sizeof(double) + GSTAGES * sizeof(uint64_t);
    return b <= 227 * 1024 ? b : 0;
}

cudaError_t launch_gaunt_batch(int nm, int nm2, int nm2p, int nchunks, const double *chunks,
                               const double *alphas, long long n, const double *betaT,
                               const int *rowPtr, const int *colInd, const double *val,
                               int sparse, double *hs, int *errorFlag, cudaStream_t st)
{
    size_t smem = gaunt_batch_smem(nm, nm2p);
    int tpw = (nm2p / 8 + 7) / 8;
    if (smem == 0 || nm < 1 || nm > 64 || nm2p % 8 != 0 || tpw < 1 || tpw > 4)
        return cudaErrorInvalidValue;
    if (n < 1)
        return cudaSuccess;
    void (*kern)(int, int, int, int, const double *, const double *, long long, const double *,
                 const int *, const int *, const double *, int, double *, int *) =
        tpw == 1 ? gaunt_batch_kernel<1> : tpw == 2 ? gaunt_batch_kernel<2>
                                         : tpw == 3 ? gaunt_batch_kernel<3> : gaunt_batch_kernel<4>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    long long grid = (n + 7) / 8;
    kern<<<(unsigned)grid, 256, smem, st>>>(nm, nm2, nm2p, nchunks, chunks, alphas, n, betaT, rowPtr,
                                            colInd, val, sparse, hs, errorFlag);
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
