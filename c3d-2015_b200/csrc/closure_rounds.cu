// Work-list form of the FP64 M_N closure: the reference's batched structure
// (Optimization::opt with its stacks, src/opt/optBatch.cpp:350-472) on the device.
//
// A closure runs in rounds over a device work list of cells that need a quadrature
// pass (a Hessian evaluation or a line-search trial):
//   init kernel    per cell: scale u and alpha (preProcess, src/opt/optBatch.cpp:312-331),
//                  start the first Newton iteration, append the cell to the work list;
//   pass kernel    per listed cell: exponents alpha.m_q and either the extended moments
//                  of the Gaunt form (one DMMA GEMM for the 8 cells of a CTA, shared
//                  staged M2^T chunks) or the direct Hessian tiles, or the trial's f;
//   Newton kernel  one warp per listed cell: assemble H, Cholesky, condition estimate,
//                  direction, stop tests, Armijo (solveTheRest, src/opt/optBatch.cpp:143-283)
//                  with the state machine shared with the persistent kernels; cells that
//                  need another pass are appended to the next round's list.
// Separating the passes (tensor-pipe work, small shared memory) from the per-cell logic
// (latency-bound, one warp per cell) lets each run at its own occupancy; a cell that
// needs many iterations only ever occupies the short lists of later rounds.
#include "closure_core.cuh"

#include <mutex>
#include <vector>
#include "rounds_launch.h"
#include "umma.cuh"

#include <cuda_bf16.h>
#include <cstdio>
#include <type_traits>

namespace c3d {

// Per-cell Newton state between rounds: the slot without the factor, the reciprocal
// pivots and the gradient (recomputed from H on every Hessian visit, unused by trials).
template <int NT> struct CellState {
    static constexpr int NMP = Cfg<NT>::NMP;
    double u[NMP], alpha[NMP], alpha0[NMP], uOrig[NMP], d[NMP], alphaOld[NMP];
    SlotScalars s;
};

namespace {

// lineSearch = false skips d and alphaOld, which a Hessian visit recomputes before use.
template <int NT, class S>
__device__ void state_to_slot(const CellState<NT> &st, S &sl, int lane, bool lineSearch = true)
{
    constexpr int NMP = Cfg<NT>::NMP;
    for (int i = lane; i < NMP; i += 32) {
        sl.u[i] = st.u[i];
        sl.alpha[i] = st.alpha[i];
        sl.alpha0[i] = st.alpha0[i];
        sl.uOrig[i] = st.uOrig[i];
        if (lineSearch) {
            sl.d[i] = st.d[i];
            sl.alphaOld[i] = st.alphaOld[i];
        }
    }
    if (lane == 0)
        sl.s = st.s;
    __syncwarp();
}

template <int NT, class S>
__device__ void slot_to_state(const S &sl, CellState<NT> &st, int lane)
{
    constexpr int NMP = Cfg<NT>::NMP;
    __syncwarp();
    for (int i = lane; i < NMP; i += 32) {
        st.u[i] = sl.u[i];
        st.alpha[i] = sl.alpha[i];
        st.alpha0[i] = sl.alpha0[i];
        st.uOrig[i] = sl.uOrig[i];
        st.d[i] = sl.d[i];
        st.alphaOld[i] = sl.alphaOld[i];
    }
    if (lane == 0)
        st.s = sl.s;
}

// The work lists of one round: 0 trials and FP64 Hessian passes, 1 BF16 Hessian passes,
// 2 3xTF32 Hessian passes (lists 1 and 2: mixed-precision closure only), 3 first visits
// through the probe pass (convergence certificate).
constexpr int NLISTS = 4;
struct Lists {
    int *list[NLISTS];
    unsigned int *count[NLISTS];
};

// The list of a cell's next pass. Mixed precision: the Hessian's moments in BF16 when the
// last condition estimate is <= condBf16, in 3xTF32 up to condMixMax or when there is no
// estimate yet, else (and after mixIterMax iterations at one regularisation level, or once a
// reduced-precision factorisation failed) in FP64.
template <class S> __device__ int route_list(const S &sl, const ClosureParams &P)
{
    if (sl.s.need == NEED_PROBE)
        return 3;
    if (sl.s.need != NEED_H || !P.mixed || sl.s.fp64 || sl.s.iter > P.mixIterMax)
        return 0;
    const double c = sl.s.cnd;
    if (c < 0.0)
        return 2;
    if (c <= P.condBf16)
        return 1;
    if (c <= P.condMixMax)
        return 2;
    return 0;
}

// Appends cell c to its list when it still needs a pass.
template <class S>
__device__ void append_if_needed(const S &sl, const ClosureParams &P, long long c, int lane,
                                 const Lists &out)
{
    if (lane == 0 && sl.s.need != NEED_NONE) {
        // selects, not an indexed parameter array (which would be copied to local memory)
        const int l = route_list(sl, P);
        unsigned int *cnt = l == 0   ? out.count[0]
                            : l == 1 ? out.count[1]
                            : l == 2 ? out.count[2]
                                     : out.count[3];
        int *lst = l == 0 ? out.list[0] : l == 1 ? out.list[1] : l == 2 ? out.list[2] : out.list[3];
        unsigned int pos = atomicAdd(cnt, 1u);
        lst[pos] = (int)c;
    }
}

} // namespace

constexpr int RW = 8;  // warps (cells) per CTA of the init and pass kernels
constexpr int RWN = 4; // warps (cells) per CTA of the Newton kernel

// Entries a round kernel works on: n, or with nDev (the list's device counter, as the
// graph-resident round loop launches them) the smaller of n and *nDev.
__device__ __forceinline__ int round_entries(int n, const unsigned int *nDev)
{
    return nDev ? (int)min((unsigned int)n, *nDev) : n;
}

template <int NT> using TSlot = Slot<NT, true>;

// Per-warp state of a first visit after the probe pass: the vectors and scalars of Slot
// without the factor (the probe's Newton kernel forms no Hessian).
template <int NT> struct alignas(16) ProbeSlot {
    static constexpr int NMP = Cfg<NT>::NMP;
    double u[NMP], alpha[NMP], alpha0[NMP], uOrig[NMP], g[NMP], d[NMP], alphaOld[NMP];
    double pm[NMP + 8]; // the cell's probe entry, loaded before the cell's state
    SlotScalars s;
};
template <int NT, int MODE>
using NewtonSlot = typename std::conditional<MODE == 2, ProbeSlot<NT>, TSlot<NT>>::type;

template <int NT>
__global__ void __launch_bounds__(RW * 32)
    rounds_init_kernel(ClosureParams P, long long ncells, const int *__restrict__ cellMap,
                       Outputs O, CellState<NT> *state, Lists out)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Slot<NT> *slots = reinterpret_cast<Slot<NT> *>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long c = (long long)blockIdx.x * RW + warp;
    if (c >= ncells)
        return;
    Slot<NT> &sl = slots[warp];
    // the state and work lists use the closure's own numbering c; outputs the grid cell's
    load_cell(sl, P, O, cellMap ? (long long)cellMap[c] : c, lane);
    if (sl.s.need != NEED_NONE)
        slot_to_state(sl, state[c], lane);
    append_if_needed(sl, P, c, lane, out);
}

// Pass of the Gaunt form over RWP = 16 listed cells per CTA (warp w: cells 2w, 2w + 1):
// per staged chunk of QC directions, each lane forms the exponents alpha.m_q of both cells
// for its direction (the reference's order: moment index ascending, unfused,
// src/opt/fobj.cpp:64-79) and c_q = w_q e^{alpha.m_q}; then either the extended moments
// mom_k = sum_q M2[k][q] c_q of the cells that need H, as a DMMA GEMM [nm2 x QC] x [QC x 16]
// (each A fragment of M2 serves both 8-cell tiles), or the trial objective's quadrature sum.
// Chunk layout (c3d_set_gaunt): nm2 rows of M2 then the weight row, row stride QCP.
constexpr int RWP = 16;
constexpr int CST2 = 20; // row stride (cells) of the coefficient tile: conflict-free B fragments

template <int NT, int NT2>
__global__ void __launch_bounds__(RW * 32, 2)
    rounds_pass_gaunt_kernel(ClosureParams P, const double *__restrict__ chunks, int nm2,
                             const int *__restrict__ list, int n, const unsigned int *nDev,
                             CellState<NT> *state, double *__restrict__ momBuf, int *errorFlag)
{
    n = round_entries(n, nDev);
    if (blockIdx.x * RWP >= n)
        return;
    constexpr int NM2P = 8 * NT2;
    constexpr int RT = (NT2 + RW - 1) / RW;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nm = P.nm, nchunks = P.nchunks;
    const int CH = (nm2 + 1) * QCP; // doubles per chunk (multiple of 4: 16-byte copies)
    double *stage = reinterpret_cast<double *>(smem_raw);
    double *cbuf = stage + GSTAGES * CH; // QC x CST2
    // multipliers of warp w's two cells interleaved, (cell 2w, cell 2w + 1) per moment: one
    // 16-byte broadcast load feeds both cells' exponents
    double2 *alph = reinterpret_cast<double2 *>(cbuf + QC * CST2); // RW x nm
    uint64_t *full = reinterpret_cast<uint64_t *>(alph + RW * nm);
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t chunkBytes = CH * sizeof(double);
    int need[2];
    long long cell[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int pos = blockIdx.x * RWP + 2 * warp + e;
        need[e] = NEED_NONE;
        cell[e] = -1;
        if (pos < n) {
            cell[e] = list[pos];
            need[e] = state[cell[e]].s.need;
        }
        for (int i = lane; i < nm; i += 32) {
            const double a = cell[e] >= 0 ? state[cell[e]].alpha[i] : 0.0;
            if (e == 0)
                alph[warp * nm + i].x = a;
            else
                alph[warp * nm + i].y = a;
        }
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
    const bool anyH = __syncthreads_or(need[0] == NEED_H || need[1] == NEED_H);
    const double2 *aw = alph + warp * nm;
    double acc[RT][2][2];
#pragma unroll
    for (int r = 0; r < RT; ++r)
        acc[r][0][0] = acc[r][0][1] = acc[r][1][0] = acc[r][1][1] = 0.0;
    double fpart0 = 0.0, fpart1 = 0.0;
    const bool any = need[0] != NEED_NONE || need[1] != NEED_NONE;
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
        double c0 = 0.0, c1 = 0.0;
        if (any) {
            double z0 = 0.0, z1 = 0.0;
            for (int i = 0; i < nm; ++i) {
                const double m = ch[i * QCP + lane];
                const double2 a = aw[i];
                z0 = __dadd_rn(z0, __dmul_rn(a.x, m));
                z1 = __dadd_rn(z1, __dmul_rn(a.y, m));
            }
            const double wq = ch[nm2 * QCP + lane];
            if (need[0] != NEED_NONE) {
                c0 = __dmul_rn(wq, exp(z0));
                if (need[0] == NEED_TRIAL)
                    fpart0 = __dadd_rn(fpart0, c0);
            }
            if (need[1] != NEED_NONE) {
                c1 = __dmul_rn(wq, exp(z1));
                if (need[1] == NEED_TRIAL)
                    fpart1 = __dadd_rn(fpart1, c1);
            }
        }
        cbuf[lane * CST2 + 2 * warp] = (need[0] == NEED_H) ? c0 : 0.0;
        cbuf[lane * CST2 + 2 * warp + 1] = (need[1] == NEED_H) ? c1 : 0.0;
        __syncthreads();
        if (anyH) {
#pragma unroll
            for (int g = 0; g < QC / 4; ++g) {
                const double b0 = cbuf[(4 * g + (lane & 3)) * CST2 + (lane >> 2)];
                const double b1 = cbuf[(4 * g + (lane & 3)) * CST2 + 8 + (lane >> 2)];
#pragma unroll
                for (int r = 0; r < RT; ++r) {
                    const int rt = warp + r * RW;
                    const int row = 8 * rt + (lane >> 2);
                    if (rt < NT2) {
                        const double a = row < nm2 ? ch[row * QCP + 4 * g + (lane & 3)] : 0.0;
                        dmma(acc[r][0][0], acc[r][0][1], a, b0);
                        dmma(acc[r][1][0], acc[r][1][1], a, b1);
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
    if (anyH) {
        const int base = blockIdx.x * RWP;
#pragma unroll
        for (int r = 0; r < RT; ++r) {
            const int rt = warp + r * RW;
            if (rt < NT2) {
                const int kk = 8 * rt + (lane >> 2);
#pragma unroll
                for (int t = 0; t < 2; ++t)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int p = base + 8 * t + 2 * (lane & 3) + e;
                        if (p < n)
                            momBuf[(size_t)p * NM2P + kk] = acc[r][t][e];
                    }
            }
        }
    }
    const double fq0 = warp_sum(fpart0), fq1 = warp_sum(fpart1);
    if (lane == 0) {
        if (need[0] == NEED_TRIAL)
            state[cell[0]].s.fquad = fq0;
        if (need[1] == NEED_TRIAL)
            state[cell[1]].s.fquad = fq1;
    }
}

// Pass of the direct form: per listed cell, the lower-triangle DMMA tiles of H (packed
// into hBuf[pos]) or the trial's quadrature sum.
template <int NT>
__global__ void __launch_bounds__(RW * 32, 1)
    rounds_pass_direct_kernel(ClosureParams P, const double *__restrict__ chunks,
                              const int *__restrict__ list, int n, const unsigned int *nDev,
                              CellState<NT> *state, double *__restrict__ hBuf, int *errorFlag)
{
    n = round_entries(n, nDev);
    if (blockIdx.x * RW >= n)
        return;
    constexpr int NMP = Cfg<NT>::NMP;
    constexpr int CH = Cfg<NT>::CHUNK;
    constexpr int ST = 3;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *stage = reinterpret_cast<double *>(smem_raw);
    double *alph = stage + ST * CH;
    uint64_t *full = reinterpret_cast<uint64_t *>(alph + RW * NMP);
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nm = P.nm, nchunks = P.nchunks;
    const uint32_t chunkBytes = CH * sizeof(double);
    const int pos = blockIdx.x * RW + warp;
    int need = NEED_NONE;
    long long cell = -1;
    if (pos < n) {
        cell = list[pos];
        need = state[cell].s.need;
    }
    for (int i = lane; i < NMP; i += 32)
        alph[warp * NMP + i] = (cell >= 0 && i < nm) ? state[cell].alpha[i] : 0.0;
    if (tid == 0) {
        for (int s = 0; s < ST; ++s)
            mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
        for (int k = 0; k < ST && k < nchunks; ++k) {
            mbar_expect_tx(&full[k], chunkBytes);
            bulk_g2s(stage + k * CH, chunks + (size_t)k * CH, chunkBytes, &full[k]);
        }
    }
    __syncthreads();
    const double *al = alph + warp * NMP;
    double acc[Cfg<NT>::NTILE][2];
#pragma unroll
    for (int t = 0; t < Cfg<NT>::NTILE; ++t)
        acc[t][0] = acc[t][1] = 0.0;
    double fpart = 0.0;
    for (int k = 0; k < nchunks; ++k) {
        uint32_t s = k % ST, parity = (k / ST) & 1u;
        if (!mbar_wait(&full[s], parity))
            s_abort = 1;
        if (__syncthreads_or(s_abort)) {
            if (tid == 0)
                atomicExch(errorFlag, 1);
            return;
        }
        const double *ch = stage + s * CH;
        if (need != NEED_NONE) {
            double z = 0.0;
            for (int i = 0; i < nm; ++i)
                z = __dadd_rn(z, __dmul_rn(al[i], ch[i * QCP + lane]));
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
        if (tid == 0 && k + ST < nchunks) {
            mbar_expect_tx(&full[s], chunkBytes);
            bulk_g2s(stage + s * CH, chunks + (size_t)(k + ST) * CH, chunkBytes, &full[s]);
        }
    }
    if (need == NEED_H) {
        // tiles of the padded H, identity in the padding rows
        double *H = hBuf + (size_t)pos * TSlot<NT>::LSIZE;
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J) {
                const int t = I * (I + 1) / 2 + J;
                int row = 8 * I + (lane >> 2), col = 8 * J + 2 * (lane & 3);
                double v0 = acc[t][0], v1 = acc[t][1];
                if (row >= nm || col >= nm)
                    v0 = (row == col) ? 1.0 : 0.0;
                if (row >= nm || col + 1 >= nm)
                    v1 = (row == col + 1) ? 1.0 : 0.0;
                *reinterpret_cast<double2 *>(&H[64 * t + tpair(lane)]) = make_double2(v0, v1);
            }
    } else if (need == NEED_TRIAL) {
        double fq = warp_sum(fpart);
        if (lane == 0)
            state[cell].s.fquad = fq;
    }
}

// ---------------------------------------------------------------- mixed-precision pass
// Pass of the mixed-precision closure over MXC = 16 listed cells per CTA that need a Hessian
// (warp w: cells 2w, 2w + 1; lane: direction of the staged 32-direction chunk):
//   FP64   exponents alpha.m_q (moment index ascending, unfused), c_q = w_q e^{alpha.m_q},
//          f's sum over q, and the first-order moments <m_i e^{alpha.m}> (i < nm) as a DMMA
//          GEMM [nm x QC] x [QC x 16] -- the gradient and objective of the FP64 stopping test
//          and line search;
//   tcgen05 the extended moments mom_k = sum_q M2[k][q] c_q of the Gaunt Hessian as
//          D[128 x 16] += A[128 x K] B[16 x K]^T per M = 128 row tile (A: the staged M2 rows
//          in BF16, or hi and lo TF32 parts; B: the cells' c_q scaled by 2^-shift, the
//          cell's largest c of its previous pass, in the same format), FP32 accumulators in
//          tensor memory. 3xTF32: A_hi B_hi + A_hi B_lo + A_lo B_hi.
// One thread issues the MMAs of a chunk once the CTA has written its B tile; their commit
// releases the chunk's stage and B buffer. Staged chunk: the nm rows of M2 of degree <= N
// and the weight row (FP64, row stride QCP), then the A operand (c3d_set_gaunt).
// Output entry (stride NM2P + NMP + 8 doubles): the nm2 moments, the nm FP64 moments, f's sum.
template <int KIND> struct MixKind;
template <> struct MixKind<0> { // BF16
    static constexpr int ES = 2, NP = 1, KI = 16;
    static constexpr uint32_t FMT = 1;
};
template <> struct MixKind<1> { // 3xTF32
    static constexpr int ES = 4, NP = 2, KI = 8;
    static constexpr uint32_t FMT = 2;
};
template <> struct MixKind<2> { // probe: the FP64 part alone
    static constexpr int ES = 8, NP = 0, KI = 8;
    static constexpr uint32_t FMT = 0;
};
constexpr int MXC = 16;

template <int NT2> struct MixRows {
    static constexpr int NM2P = 8 * NT2;
    static constexpr int NA = NM2P < 128 ? 128 : NM2P; // staged A rows (zero beyond nm2)
    static constexpr int MT = NM2P <= 128 ? 1 : 2;     // M = 128 row tiles
    static constexpr int ROW1 = NM2P - 128;            // first row of tile 1 (overlaps tile 0)
    static_assert(NM2P <= 256, "two row tiles");
};

__host__ __device__ constexpr int mix_entry_doubles(int nmp, int nm2p) { return nm2p + nmp + 8; }
// Probe entry (KIND 2): the NMP first-order moments, f's sum, e_min, e_max.
__host__ __device__ constexpr int probe_entry_doubles(int nmp) { return nmp + 8; }

// KIND 2 is the probe pass of a cell's first visit (the convergence certificate): the FP64
// part alone, with the extreme values of e^{alpha.m_q} over the chunk's directions.
// ZD (the mixed closure's passes): the exponents of the chunk as a DMMA GEMM
// Z[32 x 16] = M_chunk^T [32 x nm] alpha [nm x 16] (warp w: directions 8 (w % 4) .., cells
// 8 (w / 4) ..) staged through shared memory, instead of the reference's unfused order.
constexpr int ZS = 18; // row stride (cells) of the exponent tile: 16-byte pairs, 8-lane phases
                       // conflict-free

// The first round of a closure with the convergence certificate: no list and no set-up
// kernel; list position p is closure cell off + p, its grid cell cellMap[off + p] (or the
// same index), and the probe pass reads the grid's moments and multipliers directly (the
// scaling of load_cell, src/opt/optBatch.cpp:312-331), the probe's Newton kernel sets the cell
// up with load_cell.
struct FirstRound {
    long long off;
    const int *cellMap;
    const double *u, *alpha;
    // ansatz hand-off to the kinetic flux (grid closures with the certificate): the probe pass
    // writes psi[q nall + c] = exp(alpha_c . m_q) of every cell it solves, and the probe's
    // Newton kernel lists in refresh the cells whose multipliers may still change (their psi is
    // rewritten after the closure). Null psi: no hand-off.
    double *psi;
    long long nall;
    int *refresh;
    unsigned int *refreshCount;
    // nonzero: psi already holds the ansatz of every cell but the face ghosts for the closure's
    // starting multipliers (the previous closure's final ones), so the probe writes only the
    // face ghosts' (gnx, gny, gnz: the interior sizes that tell them)
    const int *psiValid;
    int gnx, gny, gnz;
};
constexpr int PSTR = 17; // row stride (cells) of the probe's psi tile
constexpr int PRS = 3;   // stages of the mixed probe's psi read ring (chunks k .. k + 2)

// 8-byte asynchronous global -> shared copy (zero fill when !valid; src is not read then)
__device__ __forceinline__ void cp_async8(double *dst, const double *src, bool valid)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NT, int NT2, int KIND, bool ZD>
__global__ void __launch_bounds__(RW * 32, KIND == 1 ? 1 : KIND == 2 ? 3 : 2)
    rounds_pass_mixed_kernel(ClosureParams P, const double *__restrict__ f64c,
                             const unsigned char *__restrict__ ac, const int *__restrict__ list,
                             int n, const unsigned int *nDev, CellState<NT> *state,
                             double *__restrict__ out, int *errorFlag, FirstRound first)
{
    n = round_entries(n, nDev);
    if (blockIdx.x * MXC >= n)
        return;
    using K = MixKind<KIND>;
    using R = MixRows<NT2>;
    constexpr int NMP = 8 * NT;
    constexpr int KG = QC * K::ES / 16, SBO = KG * 128;
    constexpr uint32_t APB = R::NA * QC * K::ES, BPB = MXC * QC * K::ES;
    constexpr bool TC = KIND < 2; // tensor-core moments
    constexpr int ESTR = TC ? mix_entry_doubles(NMP, R::NM2P) : probe_entry_doubles(NMP);
    constexpr uint32_t IDESC = umma_idesc(K::FMT, 128, MXC);
    static_assert(NT <= RW, "one FP64 row tile per warp");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nm = P.nm, nchunks = P.nchunks;
    const uint32_t f64Bytes = (uint32_t)(nm + 1) * QCP * 8;
    const uint32_t f64Pad = (f64Bytes + 127u) & ~127u;
    const uint32_t stg = f64Pad + K::NP * APB;
    unsigned char *bbuf = smem_raw + GSTAGES * stg; // GSTAGES x NP x BPB
    double *cbuf = reinterpret_cast<double *>(bbuf + GSTAGES * K::NP * BPB); // QC x CST2
    double2 *alph = reinterpret_cast<double2 *>(cbuf + QC * CST2);          // RW x nm
    double *zbuf = reinterpret_cast<double *>(alph + RW * nm);              // ZD: QC x ZS
    double *psiT = zbuf + (ZD ? QC * ZS : 0);                               // probe: QC x PSTR
    double *psiR = psiT + (KIND == 2 ? QC * PSTR : 0); // mixed probe: PRS x QC x PSTR
    long long *psiCell =
        reinterpret_cast<long long *>(psiR + (KIND == 2 && ZD ? PRS * QC * PSTR : 0));
    uint64_t *full = reinterpret_cast<uint64_t *>(psiCell + (KIND == 2 ? MXC : 0));
    uint64_t *mmab = full + GSTAGES;
    uint64_t *fin = mmab + GSTAGES;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    __shared__ int s_shift[MXC];
    __shared__ long long s_gc[MXC];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int base = blockIdx.x * MXC;
    // first round of a grid closure: hand the ansatz of every direction to the kinetic flux,
    // psi = u_0 e^{alpha_scaled . m_q} (the scaling shifts alpha_0 by log(u_0) 2 sqrt(pi), and
    // m_0 = 1 / (2 sqrt(pi)))
    const bool emit = KIND == 2 && !list && first.psi != nullptr;
    const bool valid = emit && first.psiValid && *first.psiValid != 0;
    long long cell[2];
    double scale[2], u0e[2] = {0.0, 0.0};
    int needMine = 0; // lane 0: one of the warp's cells has its psi written by this pass
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int pos = base + 2 * warp + e;
        cell[e] = pos < n ? (list ? list[pos] : first.off + pos) : -1;
        long long gc = -1;
        double ascale = 0.0;
        if (!list && cell[e] >= 0) {
            gc = first.cellMap ? first.cellMap[cell[e]] : cell[e];
            u0e[e] = first.u[gc * nm];
            ascale = log(u0e[e]) * 2.0 * sqrt(M_PI);
        }
        if constexpr (KIND == 2)
            if (lane == 0) {
                bool need = emit;
                if (valid && gc >= 0) {
                    // only a face ghost's psi may be missing (its image's was read instead)
                    const int gz = first.gnz + 4, gy = first.gny + 4;
                    const int k = (int)(gc % gz), j = (int)((gc / gz) % gy), i = (int)(gc / gz / gy);
                    const int in = (i >= 2 && i < first.gnx + 2) + (j >= 2 && j < first.gny + 2) +
                                   (k >= 2 && k < first.gnz + 2);
                    need = in == 2;
                }
                psiCell[2 * warp + e] = need ? gc : -1;
                s_gc[2 * warp + e] = gc;
                needMine |= need && gc >= 0;
            }
        for (int i = lane; i < nm; i += 32) {
            double a = 0.0;
            if (cell[e] >= 0) {
                if (list) {
                    a = state[cell[e]].alpha[i];
                } else {
                    a = first.alpha[gc * nm + i];
                    if (i == 0)
                        a = a - ascale;
                }
            }
            if (e == 0)
                alph[warp * nm + i].x = a;
            else
                alph[warp * nm + i].y = a;
        }
        const int sh = (cell[e] >= 0 && list) ? state[cell[e]].s.cshift : 0;
        if (lane == 0)
            s_shift[2 * warp + e] = sh;
        scale[e] = ldexp(1.0, -sh);
    }
    if (tid == 0) {
        for (int s = 0; s < GSTAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&mmab[s], 1);
        }
        mbar_init(fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_abort = 0;
        for (int k = 0; k < GSTAGES && k < nchunks; ++k) {
            unsigned char *st = smem_raw + k * stg;
            mbar_expect_tx(&full[k], f64Bytes + K::NP * APB);
            bulk_g2s(st, f64c + (size_t)k * (nm + 1) * QCP, f64Bytes, &full[k]);
            if constexpr (TC)
                bulk_g2s(st + f64Pad, ac + (size_t)k * K::NP * APB, K::NP * APB, &full[k]);
        }
    }
    if constexpr (TC)
        if (warp == 0)
            tmem_alloc(&s_tmem, 32);
    tc_fence_before();
    const int anyNeed = __syncthreads_or(needMine);
    tc_fence_after();
    const uint32_t tmem = TC ? s_tmem : 0u;
    // mixed probe with psi valid and no cell of the CTA needing its psi written: psi already
    // holds u_0 e^{alpha_scaled . m_q} of every cell, so the pass reads e^{alpha_scaled . m_q}
    // back (psi / u_0) instead of forming the exponent tile and the exponentials; the reads
    // run two chunks ahead through a ring of asynchronous copies
    const bool rd = ZD && valid && !anyNeed;
    auto psi_fetch = [&](int kc) {
        double *dst = psiR + (kc % PRS) * QC * PSTR;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int row = 4 * warp + 2 * i + (lane >> 4), j = lane & 15;
            const int q = kc * QC + row;
            const long long gc = s_gc[j];
            const bool ok = kc < nchunks && gc >= 0 && q < P.nq;
            cp_async8(dst + row * PSTR + j, ok ? first.psi + (long long)q * first.nall + gc : first.psi,
                      ok);
        }
        cp_async_commit();
    };
    if constexpr (KIND == 2 && ZD) {
        if (rd) {
            // u0e holds 1 / u_0 from here on: the read path writes no psi
            u0e[0] = 1.0 / u0e[0];
            u0e[1] = 1.0 / u0e[1];
            psi_fetch(0);
            psi_fetch(1);
        }
    }
    const double2 *aw = alph + warp * nm;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    double fpart0 = 0.0, fpart1 = 0.0, cmax0 = 0.0, cmax1 = 0.0;
    double emin0 = 1.0 / 0.0, emin1 = 1.0 / 0.0, emax0 = 0.0, emax1 = 0.0;
    for (int k = 0; k < nchunks; ++k) {
        const uint32_t s = k % GSTAGES, parity = (k / GSTAGES) & 1u;
        if (!mbar_wait(&full[s], parity))
            s_abort = 1;
        if constexpr (KIND == 2 && ZD)
            if (rd)
                cp_async_wait<1>(); // this thread's copies of chunk k have landed
        if (__syncthreads_or(s_abort))
            break;
        const unsigned char *stb = smem_raw + s * stg;
        const double *ch = reinterpret_cast<const double *>(stb);
        double z0 = 0.0, z1 = 0.0, ez0 = 0.0, ez1 = 0.0;
        if (KIND == 2 && ZD && rd) {
            // stage (k + 2) % PRS was last read in chunk k - 1, before the barrier above
            psi_fetch(k + 2);
            const double *pr = psiR + (k % PRS) * QC * PSTR + lane * PSTR + 2 * warp;
            const bool qv = k * QC + lane < P.nq; // padded directions: exponent 0
            ez0 = cell[0] >= 0 && qv ? pr[0] * u0e[0] : 1.0;
            ez1 = cell[1] >= 0 && qv ? pr[1] * u0e[1] : 1.0;
        } else if constexpr (ZD) {
            // A[dir r][k] = M2[k][8 dt + r], B[k][cell n] = alpha_n[k] (zero for k >= nm)
            const int dt = warp & 3, ct = warp >> 2, r = lane >> 2, kq = lane & 3;
            const int nb = 8 * ct + r;
            const double2 *ab = alph + (nb >> 1) * nm;
            double d0 = 0.0, d1 = 0.0;
            for (int ks = 0; ks < (nm + 3) / 4; ++ks) {
                const int k = 4 * ks + kq;
                double a = 0.0, b = 0.0;
                if (k < nm) {
                    a = ch[k * QCP + 8 * dt + r];
                    const double2 v = ab[k];
                    b = (nb & 1) ? v.y : v.x;
                }
                dmma(d0, d1, a, b);
            }
            *reinterpret_cast<double2 *>(&zbuf[(8 * dt + r) * ZS + 8 * ct + 2 * kq]) =
                make_double2(d0, d1);
            __syncthreads();
            const double2 zz = *reinterpret_cast<const double2 *>(&zbuf[lane * ZS + 2 * warp]);
            z0 = zz.x;
            z1 = zz.y;
        } else {
            for (int i = 0; i < nm; ++i) {
                const double m = ch[i * QCP + lane];
                const double2 a = aw[i];
                z0 = __dadd_rn(z0, __dmul_rn(a.x, m));
                z1 = __dadd_rn(z1, __dmul_rn(a.y, m));
            }
        }
        const double wq = ch[nm * QCP + lane];
        if (!(KIND == 2 && ZD && rd)) {
            ez0 = exp(z0);
            ez1 = exp(z1);
        }
        if constexpr (KIND == 2) {
            if (emit && !rd) {
                psiT[lane * PSTR + 2 * warp] = u0e[0] * ez0;
                psiT[lane * PSTR + 2 * warp + 1] = u0e[1] * ez1;
            }
        }
        const double c0 = cell[0] >= 0 ? __dmul_rn(wq, ez0) : 0.0;
        const double c1 = cell[1] >= 0 ? __dmul_rn(wq, ez1) : 0.0;
        fpart0 = __dadd_rn(fpart0, c0);
        fpart1 = __dadd_rn(fpart1, c1);
        if constexpr (TC) {
            cmax0 = fmax(cmax0, c0);
            cmax1 = fmax(cmax1, c1);
        } else {
            emin0 = fmin(emin0, ez0);
            emin1 = fmin(emin1, ez1);
            emax0 = fmax(emax0, ez0);
            emax1 = fmax(emax1, ez1);
        }
        cbuf[lane * CST2 + 2 * warp] = c0;
        cbuf[lane * CST2 + 2 * warp + 1] = c1;
        // B tile: cell row nn, direction column lane
        unsigned char *bt = bbuf + s * K::NP * BPB;
#pragma unroll
        for (int e = 0; e < (TC ? 2 : 0); ++e) {
            const int nn = 2 * warp + e;
            const double v = (e == 0 ? c0 : c1) * scale[e];
            const uint32_t off = (nn >> 3) * SBO + ((lane * K::ES) >> 4) * 128 + (nn & 7) * 16 +
                                 ((lane * K::ES) & 15);
            if constexpr (KIND == 0) {
                *reinterpret_cast<__nv_bfloat16 *>(bt + off) = __float2bfloat16_rn((float)v);
            } else {
                const uint32_t hi = to_tf32((float)v);
                const float lo = (float)(v - (double)__uint_as_float(hi));
                *reinterpret_cast<uint32_t *>(bt + off) = hi;
                *reinterpret_cast<uint32_t *>(bt + BPB + off) = to_tf32(lo);
            }
        }
        if constexpr (TC)
            fence_async_smem();
        __syncthreads();
        if (TC && tid == 0) {
            tc_fence_after();
            const uint32_t aAddr = umma_smem_u32(stb + f64Pad), bAddr = umma_smem_u32(bt);
#pragma unroll
            for (int j = 0; j < QC / K::KI; ++j)
#pragma unroll
                for (int t = 0; t < R::MT; ++t) {
                    const uint32_t d = tmem + 16 * t;
                    const uint32_t a0 = aAddr + (t == 0 ? 0 : (R::ROW1 / 8) * SBO) + 256 * j;
                    const uint32_t b0 = bAddr + 256 * j;
                    umma_issue<KIND == 1>(d, umma_desc(a0, SBO), umma_desc(b0, SBO), IDESC,
                                          (k > 0 || j > 0) ? 1u : 0u);
                    if constexpr (KIND == 1) {
                        umma_issue<true>(d, umma_desc(a0, SBO), umma_desc(b0 + BPB, SBO), IDESC, 1u);
                        umma_issue<true>(d, umma_desc(a0 + APB, SBO), umma_desc(b0, SBO), IDESC, 1u);
                    }
                }
            umma_commit(&mmab[s]);
        }
        if constexpr (KIND == 2) {
            // the chunk's psi rows: warp w stores directions 4w .. 4w + 3, 16 cells each
            if (emit && !rd) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int row = 4 * warp + 2 * i + (lane >> 4), j = lane & 15;
                    const long long gc = psiCell[j];
                    const int q = k * QC + row;
                    if (gc >= 0 && q < P.nq)
                        first.psi[(long long)q * first.nall + gc] = psiT[row * PSTR + j];
                }
            }
        }
        // FP64 first-order moments: warp w, rows 8w .. 8w + 7
        if (warp < NT) {
            const int row = 8 * warp + (lane >> 2);
#pragma unroll
            for (int g = 0; g < QC / 4; ++g) {
                const double b0 = cbuf[(4 * g + (lane & 3)) * CST2 + (lane >> 2)];
                const double b1 = cbuf[(4 * g + (lane & 3)) * CST2 + 8 + (lane >> 2)];
                const double a = row < nm ? ch[row * QCP + 4 * g + (lane & 3)] : 0.0;
                dmma(acc[0][0], acc[0][1], a, b0);
                dmma(acc[1][0], acc[1][1], a, b1);
            }
        }
        __syncthreads();
        if (tid == 0 && k + GSTAGES < nchunks) {
            // the MMAs of chunk k have read stage s and B buffer s
            if (TC && !mbar_wait(&mmab[s], parity)) {
                s_abort = 1;
            } else {
                unsigned char *st = smem_raw + s * stg;
                const int kn = k + GSTAGES;
                mbar_expect_tx(&full[s], f64Bytes + K::NP * APB);
                bulk_g2s(st, f64c + (size_t)kn * (nm + 1) * QCP, f64Bytes, &full[s]);
                if constexpr (TC)
                    bulk_g2s(st + f64Pad, ac + (size_t)kn * K::NP * APB, K::NP * APB, &full[s]);
            }
        }
    }
    if constexpr (KIND == 2 && ZD)
        if (rd)
            cp_async_wait<0>(); // no copy outstanding past the loop (an abort leaves it early)
    // every MMA complete before the accumulators are read and the columns freed
    if (TC && tid == 0) {
        umma_commit(fin);
        if (!mbar_wait(fin, 0))
            s_abort = 1;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const bool ok = s_abort == 0;
    if (!ok && tid == 0)
        atomicExch(errorFlag, 1);
    if (ok) {
        const int qw = warp & 3, t = warp >> 2;
        if (TC && t < R::MT) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(32 * qw) << 16) + 16 * t, r);
            const int row = (t == 0 ? 0 : R::ROW1) + 32 * qw + lane;
            if (row < R::NM2P && (t == 0 || row >= 128)) {
#pragma unroll
                for (int j = 0; j < MXC; ++j)
                    if (base + j < n)
                        out[(size_t)(base + j) * ESTR + row] =
                            ldexp((double)__uint_as_float(r[j]), s_shift[j]);
            }
        }
        if (warp < NT) {
            const int kk = 8 * warp + (lane >> 2);
#pragma unroll
            for (int tt = 0; tt < 2; ++tt)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int p = base + 8 * tt + 2 * (lane & 3) + e;
                    if (p < n)
                        out[(size_t)p * ESTR + (TC ? R::NM2P : 0) + kk] = acc[tt][e];
                }
        }
        const double fq0 = warp_sum(fpart0), fq1 = warp_sum(fpart1);
        double x0, x1, y0 = 0.0, y1 = 0.0;
        if constexpr (TC) {
            x0 = warp_max(cmax0);
            x1 = warp_max(cmax1);
        } else {
            x0 = -warp_max(-emin0);
            x1 = -warp_max(-emin1);
            y0 = warp_max(emax0);
            y1 = warp_max(emax1);
        }
        if (lane == 0) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int p = base + 2 * warp + e;
                if (p < n) {
                    double *o = out + (size_t)p * ESTR + (TC ? R::NM2P : 0) + NMP;
                    o[0] = e == 0 ? fq0 : fq1;
                    if constexpr (TC) {
                        const double cm = e == 0 ? x0 : x1;
                        int sh = (cm > 0.0 && cm < 1.0 / 0.0) ? ilogb(cm) : 0;
                        state[cell[e]].s.cshift = sh < -120 ? -120 : sh > 120 ? 120 : sh;
                    } else {
                        o[1] = e == 0 ? x0 : x1;
                        o[2] = e == 0 ? y0 : y1;
                    }
                }
            }
        }
    }
    if constexpr (TC) {
        tc_fence_before();
        __syncthreads();
        if (warp == 0) {
            tc_fence_after();
            tmem_dealloc(tmem, 32);
        }
    }
}

// Newton logic for the listed cells: one warp per cell, RWN cells per CTA, state staged
// in shared memory with H in the tiled layout (TSlot).
// MODE 0: FP64 Hessians and trials. MODE 1: the list of a mixed-precision pass (entries of
// mix_entry_doubles): H from the reduced-precision moments, g and f from the pass's FP64
// moments; a visit whose moments are not all finite is redone in FP64. MODE 2: first visits
// after the probe pass (entries of probe_entry_doubles; g0: the Gaunt terms of H's column 0,
// g0n per row, null in the mixed closure), no Hessian. level: the list (0 FP64 and trials,
// 1 BF16, 2 3xTF32, 3 probe).
// GAUNT: the CTA assembles H_ij = sum_k beta_ijk mom_k (i >= j, the CSR terms of beta in
// the order of src/opt/fobj.cpp:81-99, laid out per tile slot by c3d_set_gaunt) for its
// cells that need a Hessian in one sweep over the tile slots, so that each term is read once
// for RWN cells. A cell's moments sit in its slot's g..rinv vectors, which a Hessian visit
// recomputes afterwards. Otherwise the pass wrote H in tiles to hBuf.
template <int NT, int NT2, bool GAUNT, int MODE>
__global__ void __launch_bounds__(RWN * 32)
    rounds_newton_kernel(ClosureParams P, double m0, const int *__restrict__ list, int n,
                         const unsigned int *nDev, CellState<NT> *state,
                         const double *__restrict__ buf,
                         const GauntTerm *__restrict__ stream, int streamLen,
                         Outputs Og, Lists out, int level, const GauntTerm *__restrict__ g0,
                         int g0n, FirstRound first)
{
    n = round_entries(n, nDev);
    if (blockIdx.x * RWN >= n)
        return;
    constexpr bool MIX = MODE == 1;
    constexpr int NM2P = 8 * NT2;
    constexpr int NMP = Cfg<NT>::NMP;
    constexpr int BSTR = MODE == 1 ? mix_entry_doubles(NMP, NM2P)
                                   : MODE == 2 ? probe_entry_doubles(NMP) : NM2P;
    constexpr int LS = TSlot<NT>::LSIZE;
    static_assert(!GAUNT || NM2P <= 4 * NMP, "moments must fit in g, d, alphaOld, rinv");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    using SlotT = NewtonSlot<NT, MODE>;
    SlotT *slots = reinterpret_cast<SlotT *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // the CTA's closure counters, added to the context's once at the end (one global atomic
    // per counter and CTA instead of several per finished cell)
    __shared__ unsigned long long sStat[STAT_COUNT];
    for (int q = tid; q < STAT_COUNT; q += RWN * 32)
        sStat[q] = 0;
    __syncthreads();
    Outputs O = Og;
    if (Og.stats)
        O.stats = sStat;
    const int pos = blockIdx.x * RWN + warp;
    const bool active = pos < n;
    const long long cell = active ? (list ? list[pos] : first.off + pos) : -1;
    const bool needH = MODE != 2 && active && state[cell].s.need == NEED_H;
    SlotT &sl = slots[warp];
    // probe visits: the probe entry's loads go out before the cell's state is read, so the
    // two global round trips overlap
    constexpr int PMR = (BSTR + 31) / 32;
    double pmr[PMR];
    if constexpr (MODE == 2)
        if (active)
#pragma unroll
            for (int r = 0; r < PMR; ++r)
                pmr[r] = lane + 32 * r < BSTR ? buf[(size_t)pos * BSTR + lane + 32 * r] : 0.0;
    C3D_NCLK_DECL
    long long gcell = -1; // probe visits: the grid cell, for the ansatz hand-off's refresh list
    if (MODE == 2 && active && first.refresh)
        gcell = !list ? (first.cellMap ? (long long)first.cellMap[cell] : cell) : state[cell].s.cell;
    if (active) {
        if (MODE == 2 && !list)
            load_cell(sl, P, O, first.cellMap ? (long long)first.cellMap[cell] : cell, lane);
        else
            state_to_slot(state[cell], sl, lane, MODE != 2 && !(GAUNT && needH));
    } else if (lane == 0) {
        sl.s.need = NEED_NONE;
    }
    bool nonFinite = false;
    if constexpr (MODE == 2) {
    } else if (GAUNT) {
        double *mom = sl.scratch(); // g, d, alphaOld, rinv: NM2P <= 4 NMP doubles
        if (needH) {
            bool nf = false;
            for (int k = lane; k < NM2P; k += 32) {
                const double v = buf[(size_t)pos * BSTR + k];
                nf |= MIX && !isfinite(v);
                mom[k] = v;
            }
            nonFinite = __any_sync(FULL_MASK, nf);
        }
        if (__syncthreads_or(needH)) {
            bool hw[RWN];
#pragma unroll
            for (int w = 0; w < RWN; ++w)
                hw[w] = slots[w].s.need == NEED_H;
            static_assert(RWN * 32 == NEWTON_THREADS, "stream layout");
            double h[RWN];
#pragma unroll
            for (int w = 0; w < RWN; ++w)
                h[w] = 0.0;
#pragma unroll 4
            for (int k = 0; k < streamLen; ++k) {
                const GauntTerm gt = stream[k * NEWTON_THREADS + tid];
                if (gt.col >= 0) {
#pragma unroll
                    for (int w = 0; w < RWN; ++w)
                        h[w] = __dadd_rn(h[w], __dmul_rn(slots[w].scratch()[gt.col], gt.v));
                } else {
#pragma unroll
                    for (int w = 0; w < RWN; ++w)
                        h[w] = 1.0;
                }
                if (gt.slot >= 0) {
#pragma unroll
                    for (int w = 0; w < RWN; ++w) {
                        if (hw[w])
                            slots[w].L[gt.slot] = h[w];
                        h[w] = 0.0;
                    }
                }
            }
        }
        __syncthreads();
    } else if (needH) {
        const double2 *H = reinterpret_cast<const double2 *>(buf + (size_t)pos * LS);
        double2 *L = reinterpret_cast<double2 *>(sl.L);
        for (int e = lane; e < LS / 2; e += 32)
            L[e] = H[e];
        __syncwarp();
    }
    if (active) {
    C3D_NCLK(O.stats, 0, lane);
    if constexpr (MODE == 2) {
        if (sl.s.need == NEED_PROBE) {
#pragma unroll
            for (int r = 0; r < PMR; ++r)
                if (lane + 32 * r < BSTR)
                    sl.pm[lane + 32 * r] = pmr[r];
            __syncwarp();
            after_probe(sl, P, O, lane, m0, sl.pm, g0, g0n);
        }
    } else if (sl.s.need == NEED_H) {
        if (lane == 0) {
            sl.s.hprec = MIX ? level : 0;
            if (P.mixed && O.stats)
                atomicAdd(&O.stats[level == 1   ? STAT_H_BF16
                                   : level == 2 ? STAT_H_TF32X3
                                                : STAT_H_FP64],
                          1ull);
        }
        if constexpr (MIX) {
            if (nonFinite) {
                escalate_fp64(sl, O, lane);
            } else {
                const double *e = buf + (size_t)pos * BSTR + NM2P;
                after_hessian(sl, P, O, lane, m0, e, e[NMP]);
            }
        } else {
            after_hessian(sl, P, O, lane, m0);
        }
        C3D_NCLK(O.stats, 5, lane);
    } else if (sl.s.need == NEED_TRIAL) {
        after_trial(sl, P, O, lane, sl.s.fquad);
        C3D_NCLK(O.stats, 7, lane);
    }
    if constexpr (MODE == 2) {
        // a cell that goes on past its probe visit (or failed there) may end with other
        // multipliers than the probe's: its psi is rewritten after the closure
        if (gcell >= 0 && lane == 0 && (sl.s.need != NEED_NONE || sl.s.status != CELL_OK))
            first.refresh[atomicAdd(first.refreshCount, 1u)] = (int)gcell;
    }
    // a finished cell's state is not read again
    if (sl.s.need != NEED_NONE)
        slot_to_state(sl, state[cell], lane);
    append_if_needed(sl, P, cell, lane, out);
    C3D_NCLK(O.stats, 6, lane);
    }
    __syncthreads();
    if (Og.stats)
        for (int q = tid; q < STAT_COUNT; q += RWN * 32) {
            const unsigned long long v = sStat[q];
            if (v == 0)
                continue;
            if (q == STAT_MAX_ITER || q == STAT_MAX_ITER_GAMMA)
                atomicMax(&Og.stats[q], v);
            else
                atomicAdd(&Og.stats[q], v);
        }
}

// ---------------------------------------------------------------- host side

template <int NT> static size_t state_bytes_t() { return sizeof(CellState<NT>); }

size_t rounds_state_bytes(int nm)
{
    switch ((nm + 7) / 8) {
    case 1: return state_bytes_t<1>();
    case 2: return state_bytes_t<2>();
    case 3: return state_bytes_t<3>();
    case 4: return state_bytes_t<4>();
    case 5: return state_bytes_t<5>();
    case 6: return state_bytes_t<6>();
    case 7: return state_bytes_t<7>();
    default: return state_bytes_t<8>();
    }
}

// Doubles per list entry of the pass output buffer.
size_t rounds_buf_doubles(int nm, int nm2, bool gaunt, bool mixed)
{
    const int nt = (nm + 7) / 8;
    if (gaunt) {
        const int nm2p = 8 * ((nm2 + 7) / 8);
        const size_t e = (size_t)(mixed ? mix_entry_doubles(8 * nt, nm2p) : nm2p);
        const size_t pr = (size_t)probe_entry_doubles(8 * nt);
        return e > pr ? e : pr;
    }
    return (size_t)64 * nt * (nt + 1) / 2; // the tiled lower triangle
}

// Bytes of one staged chunk of the mixed pass's A operand (format 0 BF16, 1 TF32 hi + lo).
size_t mixed_a_chunk_bytes(int nm2, int fmt)
{
    const int nm2p = 8 * ((nm2 + 7) / 8);
    const int na = nm2p < 128 ? 128 : nm2p;
    return (size_t)na * QC * (fmt == 0 ? 2 : 8);
}

template <int NT, int KIND, bool ZD> static size_t mixed_pass_smem(const ClosureParams &P, int nm2)
{
    using K = MixKind<KIND>;
    const size_t f64Pad = ((size_t)(P.nm + 1) * QCP * 8 + 127) & ~(size_t)127;
    const size_t stg = f64Pad + (KIND < 2 ? mixed_a_chunk_bytes(nm2, KIND) : 0);
    return GSTAGES * stg + GSTAGES * (size_t)K::NP * MXC * QC * K::ES + (size_t)QC * CST2 * 8 +
           (size_t)RW * P.nm * 16 + (ZD ? (size_t)QC * ZS * 8 : 0) +
           (KIND == 2 ? (size_t)QC * PSTR * 8 + MXC * 8 : 0) +
           (KIND == 2 && ZD ? (size_t)PRS * QC * PSTR * 8 : 0) + (2 * GSTAGES + 1) * 8;
}

// ---------------------------------------------------------------- graph-resident round loop
//
// A closure is one CUDA graph: round 0 (set-up, or the certificate's probe round) then a
// conditional WHILE node whose body runs two rounds (lists A -> B, then B -> A) and sets the
// loop condition on the device, so no round waits for the host. Within a round, each list's
// pass and Newton kernels sit in a SWITCH node whose branch -- one of four launch sizes
// (up to 512, 8192, 65536 and `cap` entries) or none for an empty list -- a control kernel
// picks from the list's device counter; entries past `cap` are carried to the next round's
// list. The kernels read their entry count from the counter (round_entries).

constexpr int NTIER = 4;
__host__ __device__ inline long long tier_entries(int t, long long cap)
{
    const long long t0 = t == 0 ? 512 : t == 1 ? 8192 : 65536;
    return t < 3 && t0 < cap ? t0 : cap;
}

struct TierHandles {
    cudaGraphConditionalHandle h[NLISTS];
};

// Picks each used list's launch size (SWITCH branch; NTIER = none) from its counter (bit l of
// mask marks list l as used) and clears the counters of the lists the round fills.
__global__ void rounds_tier_kernel(const Lists in, Lists out, TierHandles th, unsigned int mask,
                                   long long cap, unsigned long long *launches)
{
    if (threadIdx.x != 0)
        return;
    for (int l = 0; l < NLISTS; ++l)
        *out.count[l] = 0;
    unsigned long long l2 = 1;
    for (int l = 0; l < NLISTS; ++l) {
        if (!((mask >> l) & 1u))
            continue;
        const long long c = (long long)*in.count[l];
        int t = NTIER;
        for (int k = NTIER - 1; k >= 0; --k)
            if (c > 0 && c <= tier_entries(k, cap))
                t = k;
        if (c > cap)
            t = NTIER - 1;
        cudaGraphSetConditional(th.h[l], (unsigned int)t);
        l2 += t < NTIER ? 2 : 0;
    }
    if (launches)
        atomicAdd(launches, l2);
}

// Entries past cap stay for the next round: appended to that round's list.
__global__ void rounds_carry_kernel(const Lists in, Lists out, unsigned int mask, long long cap)
{
    __shared__ unsigned int base[NLISTS];
    for (int l = 0; l < NLISTS; ++l) {
        if (!((mask >> l) & 1u))
            continue;
        const long long c = (long long)*in.count[l];
        if (c <= cap)
            continue; // uniform over the block
        if (threadIdx.x == 0)
            base[l] = atomicAdd(out.count[l], (unsigned int)(c - cap));
        __syncthreads();
        for (long long i = cap + threadIdx.x; i < c; i += blockDim.x)
            out.list[l][base[l] + (i - cap)] = in.list[l][i];
        __syncthreads();
    }
}

// Loop condition after the body's two rounds: more work and the round limit not reached;
// past the limit the closure stops with errorFlag 2 (c3d_sync: C3D_ERR_TIMEOUT).
__global__ void rounds_cond_kernel(const Lists in, unsigned int mask, unsigned int *rounds,
                                   long long maxRounds, int *errorFlag,
                                   cudaGraphConditionalHandle loop, unsigned long long *launches)
{
    if (threadIdx.x != 0)
        return;
    unsigned long long total = 0;
    for (int l = 0; l < NLISTS; ++l)
        if ((mask >> l) & 1u)
            total += *in.count[l];
    const unsigned int r = *rounds + 2;
    *rounds = r;
    bool more = total > 0;
    if (more && (long long)r >= maxRounds) {
        atomicExch(errorFlag, 2);
        more = false;
    }
    cudaGraphSetConditional(loop, more ? 1u : 0u);
    if (launches)
        atomicAdd(launches, 1ull);
}

// Appends a conditional node after the current dependencies of the graph being captured on st.
cudaError_t capture_conditional(cudaStream_t st, cudaGraphConditionalHandle h,
                                       cudaGraphConditionalNodeType type, unsigned int size,
                                       cudaGraph_t **bodies)
{
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &ndeps);
    if (e != cudaSuccess)
        return e;
    if (status != cudaStreamCaptureStatusActive)
        return cudaErrorStreamCaptureInvalidated;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = size;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, ndeps, &p);
    if (e != cudaSuccess)
        return e;
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    *bodies = p.conditional.phGraph_out;
    return e;
}

// Graph capture and instantiation run one thread at a time in the process (contexts driven
// from several host threads, as the serving loop does, build their graphs in turn; launches of
// built graphs do not wait).
std::mutex &graph_build_mutex()
{
    static std::mutex m;
    return m;
}

// The instantiated closure graphs of the last few configurations (a configuration is every
// launch parameter; switching, e.g., between precisions reuses its graph), with the streams
// their capture uses.
struct RoundsGraph {
    static constexpr int SLOTS = 6;
    struct Slot {
        std::vector<unsigned char> key;
        cudaGraphExec_t exec = nullptr;
        unsigned long long used = 0;
    } slot[SLOTS];
    unsigned long long tick = 0;
    cudaStream_t cs[3] = {nullptr, nullptr, nullptr};
    ~RoundsGraph()
    {
        for (Slot &s : slot)
            if (s.exec)
                cudaGraphExecDestroy(s.exec);
        for (cudaStream_t s : cs)
            if (s)
                cudaStreamDestroy(s);
    }
};

template <class T> static void key_add(std::vector<unsigned char> &k, const T &v)
{
    const unsigned char *b = reinterpret_cast<const unsigned char *>(&v);
    k.insert(k.end(), b, b + sizeof(T));
}

std::vector<unsigned char> rounds_graph_key(const RoundsLaunch &R, bool gaunt)
{
    std::vector<unsigned char> k;
    key_add(k, *R.P);
    const void *ptrs[] = {R.chunks, R.gstream, R.cellMap, R.u, R.alpha, R.iters, R.iterGamma,
                          R.regIdx, R.status, R.failCount, R.stats, R.gamma, R.normG, R.cond,
                          R.state, R.listA, R.listB, R.counts, R.buf, R.mixF64, R.mixA[0],
                          R.mixA[1], R.g0, R.errorFlag, R.psi, R.refresh, R.refreshCount,
                          R.launchDev};
    for (const void *p : ptrs)
        key_add(k, p);
    key_add(k, R.nm2);
    key_add(k, R.streamLen);
    key_add(k, R.m0);
    key_add(k, R.ncells);
    key_add(k, R.batch);
    key_add(k, R.g0n);
    key_add(k, R.psiNall);
    key_add(k, R.maxRounds);
    key_add(k, gaunt);
    return k;
}

template <int NT, int NT2, bool GAUNT> static cudaError_t rounds_t(const RoundsLaunch &R)
{
    const ClosureParams &P = *R.P;
    CellState<NT> *state = reinterpret_cast<CellState<NT> *>(R.state);
    cudaStream_t st = R.stream;
    const bool mixed = GAUNT && P.mixed;
    cudaError_t e;
    size_t slotSmem = RW * sizeof(Slot<NT>);
    e = cudaFuncSetAttribute(rounds_init_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)slotSmem);
    if (e != cudaSuccess)
        return e;
    size_t newtonSmem = RWN * sizeof(TSlot<NT>);
    e = cudaFuncSetAttribute(rounds_newton_kernel<NT, NT2, GAUNT, 0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)newtonSmem);
    if (e != cudaSuccess)
        return e;
    const bool probe = GAUNT && P.probe;
    const size_t probeSmem = RWN * sizeof(ProbeSlot<NT>);
    size_t passSmem, mixSmem[3] = {0, 0, 0};
    if (GAUNT) {
        passSmem = GSTAGES * (size_t)(R.nm2 + 1) * QCP * 8 + (size_t)QC * CST2 * 8 +
                   (size_t)(RWP * P.nm + 1) * 8 + GSTAGES * 8;
        e = cudaFuncSetAttribute(rounds_pass_gaunt_kernel<NT, NT2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)passSmem);
        if (e == cudaSuccess && probe) {
            e = cudaFuncSetAttribute(rounds_newton_kernel<NT, NT2, GAUNT, 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)probeSmem);
            mixSmem[2] = mixed ? mixed_pass_smem<NT, 2, true>(P, R.nm2)
                               : mixed_pass_smem<NT, 2, false>(P, R.nm2);
            if (e == cudaSuccess)
                e = mixed ? cudaFuncSetAttribute(rounds_pass_mixed_kernel<NT, NT2, 2, true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)mixSmem[2])
                          : cudaFuncSetAttribute(rounds_pass_mixed_kernel<NT, NT2, 2, false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)mixSmem[2]);
        }
        if (e == cudaSuccess && mixed) {
            e = cudaFuncSetAttribute(rounds_newton_kernel<NT, NT2, GAUNT, 1>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)newtonSmem);
            mixSmem[0] = mixed_pass_smem<NT, 0, true>(P, R.nm2);
            mixSmem[1] = mixed_pass_smem<NT, 1, true>(P, R.nm2);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(rounds_pass_mixed_kernel<NT, NT2, 0, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mixSmem[0]);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(rounds_pass_mixed_kernel<NT, NT2, 1, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mixSmem[1]);
        }
    } else {
        passSmem = 3 * (size_t)Cfg<NT>::CHUNK * 8 + (size_t)RW * Cfg<NT>::NMP * 8 + 3 * 8;
        e = cudaFuncSetAttribute(rounds_pass_direct_kernel<NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)passSmem);
    }
    if (e != cudaSuccess)
        return e;
    const double m0 = R.m0;
    const Outputs O{R.u,      R.alpha,     R.iters, R.iterGamma, R.regIdx,
                    R.status, R.failCount, R.stats, R.gamma,     R.normG, R.cond};

    Lists A, B;
    for (int l = 0; l < NLISTS; ++l) {
        A.list[l] = R.listA + (size_t)l * R.ncells;
        B.list[l] = R.listB + (size_t)l * R.ncells;
        A.count[l] = R.counts + l;
        B.count[l] = R.counts + NLISTS + l;
    }
    // the lists the graph's rounds can fill: FP64 Hessian passes and, when the mixed closure
    // routes any visit to reduced precision, its BF16 and 3xTF32 ones (probe passes happen in
    // round 0 only: no later visit is a first visit)
    const unsigned int usedLists = 1u | (mixed && P.mixIterMax > 0 ? 6u : 0u);

    // pass + Newton kernels of list l: entries la[0 .. nb) (with nDev, at most *nDev of them),
    // the cells still in need appended to out
    auto launch_list = [&](int l, const int *la, int nb, const unsigned int *nDev, const Lists &out,
                           cudaStream_t s) {
        if (l == 3) {
            // probe passes of first visits (Gaunt form only)
            if constexpr (GAUNT) {
                const unsigned grid = (unsigned)((nb + MXC - 1) / MXC);
                if (mixed)
                    rounds_pass_mixed_kernel<NT, NT2, 2, true><<<grid, RW * 32, mixSmem[2], s>>>(
                        P, R.mixF64, nullptr, la, nb, nDev, state, R.buf, R.errorFlag,
                        FirstRound{});
                else
                    rounds_pass_mixed_kernel<NT, NT2, 2, false><<<grid, RW * 32, mixSmem[2], s>>>(
                        P, R.mixF64, nullptr, la, nb, nDev, state, R.buf, R.errorFlag,
                        FirstRound{});
                rounds_newton_kernel<NT, NT2, GAUNT, 2>
                    <<<(unsigned)((nb + RWN - 1) / RWN), RWN * 32, probeSmem, s>>>(
                        P, m0, la, nb, nDev, state, R.buf, R.gstream, R.streamLen, O, out, l,
                        mixed ? nullptr : R.g0, R.g0n, FirstRound{});
            }
        } else if (l > 0) {
            // mixed-precision Hessian passes (Gaunt form only)
            if constexpr (GAUNT) {
                const unsigned grid = (unsigned)((nb + MXC - 1) / MXC);
                if (l == 1)
                    rounds_pass_mixed_kernel<NT, NT2, 0, true><<<grid, RW * 32, mixSmem[0], s>>>(
                        P, R.mixF64, R.mixA[0], la, nb, nDev, state, R.buf, R.errorFlag,
                        FirstRound{});
                else
                    rounds_pass_mixed_kernel<NT, NT2, 1, true><<<grid, RW * 32, mixSmem[1], s>>>(
                        P, R.mixF64, R.mixA[1], la, nb, nDev, state, R.buf, R.errorFlag,
                        FirstRound{});
                rounds_newton_kernel<NT, NT2, GAUNT, 1>
                    <<<(unsigned)((nb + RWN - 1) / RWN), RWN * 32, newtonSmem, s>>>(
                        P, m0, la, nb, nDev, state, R.buf, R.gstream, R.streamLen, O, out, l,
                        nullptr, 0, FirstRound{});
            }
        } else {
            if (GAUNT)
                rounds_pass_gaunt_kernel<NT, NT2>
                    <<<(unsigned)((nb + RWP - 1) / RWP), RW * 32, passSmem, s>>>(
                        P, R.chunks, R.nm2, la, nb, nDev, state, R.buf, R.errorFlag);
            else
                rounds_pass_direct_kernel<NT>
                    <<<(unsigned)((nb + RW - 1) / RW), RW * 32, passSmem, s>>>(
                        P, R.chunks, la, nb, nDev, state, R.buf, R.errorFlag);
            rounds_newton_kernel<NT, NT2, GAUNT, 0>
                <<<(unsigned)((nb + RWN - 1) / RWN), RWN * 32, newtonSmem, s>>>(
                    P, m0, la, nb, nDev, state, R.buf, R.gstream, R.streamLen, O, out, 0, nullptr,
                    0, FirstRound{});
        }
        return cudaGetLastError();
    };

    // round 0: set-up of every cell (with the certificate: set-up and probe pass in one round)
    auto round0 = [&](cudaStream_t s) -> cudaError_t {
        cudaError_t e0 = cudaMemsetAsync(A.count[0], 0, NLISTS * sizeof(unsigned int), s);
        if (e0 != cudaSuccess)
            return e0;
        if (probe) {
            if constexpr (GAUNT) {
                for (long long off = 0; off < R.ncells; off += R.batch) {
                    const int nb = (int)((R.ncells - off) < R.batch ? (R.ncells - off) : R.batch);
                    const FirstRound fr{off,       R.cellMap,      R.u,      R.alpha,
                                        R.psi,     R.psiNall,      R.refresh, R.refreshCount,
                                        R.psiValid, R.gnx,         R.gny,    R.gnz};
                    const unsigned grid = (unsigned)((nb + MXC - 1) / MXC);
                    if (mixed)
                        rounds_pass_mixed_kernel<NT, NT2, 2, true><<<grid, RW * 32, mixSmem[2], s>>>(
                            P, R.mixF64, nullptr, nullptr, nb, nullptr, state, R.buf, R.errorFlag,
                            fr);
                    else
                        rounds_pass_mixed_kernel<NT, NT2, 2, false><<<grid, RW * 32, mixSmem[2], s>>>(
                            P, R.mixF64, nullptr, nullptr, nb, nullptr, state, R.buf, R.errorFlag,
                            fr);
                    rounds_newton_kernel<NT, NT2, GAUNT, 2>
                        <<<(unsigned)((nb + RWN - 1) / RWN), RWN * 32, probeSmem, s>>>(
                            P, m0, nullptr, nb, nullptr, state, R.buf, R.gstream, R.streamLen, O,
                            A, 3, mixed ? nullptr : R.g0, R.g0n, fr);
                    *R.launches += 2;
                }
            }
        } else {
            rounds_init_kernel<NT><<<(unsigned)((R.ncells + RW - 1) / RW), RW * 32, slotSmem, s>>>(
                P, R.ncells, R.cellMap, O, state, A);
            *R.launches += 1;
        }
        return cudaGetLastError();
    };

    // Appends the closure to the graph being captured on cs[0] (top: that capture's top-level
    // graph, which owns the conditional handles); cs[1], cs[2] capture the loop and switch
    // bodies.
    auto capture_into = [&](cudaGraph_t top, cudaStream_t const *cs) -> cudaError_t {
        const long long cap = R.batch;
        cudaGraphConditionalHandle hLoop;
        TierHandles th[2];
        cudaError_t ec = cudaGraphConditionalHandleCreate(&hLoop, top, 1, cudaGraphCondAssignDefault);
        // one handle per SWITCH node the graph has (a handle without its node makes the
        // graph invalid)
        for (int hr = 0; hr < 2 && ec == cudaSuccess; ++hr)
            for (int l = 0; l < NLISTS && ec == cudaSuccess; ++l)
                if ((usedLists >> l) & 1u)
                    ec = cudaGraphConditionalHandleCreate(&th[hr].h[l], top, NTIER,
                                                          cudaGraphCondAssignDefault);
        if (ec == cudaSuccess)
            ec = cudaMemsetAsync(R.counts + 2 * NLISTS, 0, sizeof(unsigned int), cs[0]);
        const long long launches0 = *R.launches;
        if (ec == cudaSuccess)
            ec = round0(cs[0]);
        *R.launches = launches0;
        cudaGraph_t *loopBody = nullptr;
        if (ec == cudaSuccess)
            ec = capture_conditional(cs[0], hLoop, cudaGraphCondTypeWhile, 1, &loopBody);
        if (ec == cudaSuccess)
            ec = cudaStreamBeginCaptureToGraph(cs[1], loopBody[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed);
        if (ec != cudaSuccess)
            return ec;
        for (int hr = 0; hr < 2 && ec == cudaSuccess; ++hr) {
            const Lists &X = hr == 0 ? A : B, &Y = hr == 0 ? B : A;
            rounds_tier_kernel<<<1, 32, 0, cs[1]>>>(X, Y, th[hr], usedLists, cap, R.launchDev);
            ec = cudaGetLastError();
            for (int l = 0; l < NLISTS && ec == cudaSuccess; ++l) {
                if (!((usedLists >> l) & 1u))
                    continue;
                cudaGraph_t *tiers = nullptr;
                ec = capture_conditional(cs[1], th[hr].h[l], cudaGraphCondTypeSwitch, NTIER, &tiers);
                for (int t = 0; t < NTIER && ec == cudaSuccess; ++t) {
                    ec = cudaStreamBeginCaptureToGraph(cs[2], tiers[t], nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeRelaxed);
                    if (ec == cudaSuccess) {
                        cudaError_t el = launch_list(l, X.list[l], (int)tier_entries(t, cap),
                                                     X.count[l], Y, cs[2]);
                        cudaGraph_t body = nullptr;
                        ec = cudaStreamEndCapture(cs[2], &body);
                        if (ec == cudaSuccess)
                            ec = el;
                    }
                }
            }
            if (ec == cudaSuccess && cap < R.ncells) { // no list can outgrow cap otherwise
                rounds_carry_kernel<<<1, 1024, 0, cs[1]>>>(X, Y, usedLists, cap);
                ec = cudaGetLastError();
            }
        }
        if (ec == cudaSuccess) {
            rounds_cond_kernel<<<1, 32, 0, cs[1]>>>(A, usedLists, R.counts + 2 * NLISTS,
                                                    R.maxRounds, R.errorFlag, hLoop, R.launchDev);
            ec = cudaGetLastError();
        }
        cudaGraph_t body = nullptr;
        cudaError_t eb = cudaStreamEndCapture(cs[1], &body);
        return ec == cudaSuccess ? eb : ec;
    };

    const long long round0Launches = probe ? 2 * ((R.ncells + R.batch - 1) / R.batch) : 1;
    if (R.captureTop) {
        // inside the capture of a whole RK stage
        e = capture_into(R.captureTop, R.captureStreams);
        if (e == cudaSuccess)
            *R.launches += round0Launches + 1;
        return e;
    }
    if (R.graphs) {
        RoundsGraph *RG = reinterpret_cast<RoundsGraph *>(R.graphs);
        std::vector<unsigned char> key = rounds_graph_key(R, GAUNT);
        RoundsGraph::Slot *G = nullptr;
        for (RoundsGraph::Slot &s : RG->slot)
            if (s.exec && s.key == key)
                G = &s;
        if (!G) {
            std::lock_guard<std::mutex> lk(graph_build_mutex());
            // the least recently used slot; a graph in it may still run on the stream and is
            // destroyed once the stream is idle
            G = &RG->slot[0];
            for (RoundsGraph::Slot &s : RG->slot)
                if (s.used < G->used)
                    G = &s;
            if (G->exec) {
                if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
                    return e;
                cudaGraphExecDestroy(G->exec);
                G->exec = nullptr;
            }
            for (int i = 0; i < 3; ++i)
                if (!RG->cs[i] && (e = cudaStreamCreateWithFlags(&RG->cs[i], cudaStreamNonBlocking)) !=
                                      cudaSuccess)
                    return e;
            cudaGraph_t top = nullptr;
            if ((e = cudaGraphCreate(&top, 0)) != cudaSuccess)
                return e;
            e = cudaStreamBeginCaptureToGraph(RG->cs[0], top, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed);
            if (e == cudaSuccess) {
                const cudaError_t ec = capture_into(top, RG->cs);
                cudaGraph_t topOut = nullptr;
                e = cudaStreamEndCapture(RG->cs[0], &topOut);
                if (e == cudaSuccess)
                    e = ec;
            }
            if (e == cudaSuccess)
                e = cudaGraphInstantiate(&G->exec, top, 0);
            cudaGraphDestroy(top);
            if (e != cudaSuccess) {
                // a failed capture may leave its streams unusable: start over with new ones
                G->exec = nullptr;
                for (cudaStream_t &cs : RG->cs) {
                    if (cs)
                        cudaStreamDestroy(cs);
                    cs = nullptr;
                }
                cudaGetLastError();
                return e;
            }
            G->key = key;
        }
        G->used = ++RG->tick;
        *R.launches += round0Launches + 1;
        return cudaGraphLaunch(G->exec, st);
    }

    // host-driven rounds: the host reads the list counts after each round
    if ((e = round0(st)) != cudaSuccess)
        return e;
    *R.launches += 1;
    long long rounds = 0;
    for (;;) {
        e = cudaMemcpyAsync(R.hostCount, A.count[0], NLISTS * sizeof(unsigned int),
                            cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return e;
        if (R.hostSyncs)
            ++*R.hostSyncs;
        long long cnt[NLISTS], total = 0;
        for (int l = 0; l < NLISTS; ++l)
            total += (cnt[l] = R.hostCount[l]);
        if (total == 0)
            break;
        if (++rounds > R.maxRounds)
            return cudaErrorLaunchTimeout;
        e = cudaMemsetAsync(B.count[0], 0, NLISTS * sizeof(unsigned int), st);
        if (e != cudaSuccess)
            return e;
        *R.launches += 1;
        for (int l = 0; l < NLISTS; ++l) {
            for (long long off = 0; off < cnt[l]; off += R.batch) {
                int nb = (int)((cnt[l] - off) < R.batch ? (cnt[l] - off) : R.batch);
                if ((e = launch_list(l, A.list[l] + off, nb, nullptr, B, st)) != cudaSuccess)
                    return e;
                *R.launches += 2;
            }
        }
        Lists t = A;
        A = B;
        B = t;
    }
    return cudaSuccess;
}

void *rounds_graph_new() { return new RoundsGraph(); }
void rounds_graph_free(void *g) { delete reinterpret_cast<RoundsGraph *>(g); }

// Moment counts with a work-list Gaunt form (N <= 7).
bool rounds_gaunt_supported(int nm)
{
    return nm == 1 || nm == 4 || nm == 9 || nm == 16 || nm == 25 || nm == 36 || nm == 49 ||
           nm == 64;
}

cudaError_t launch_closure_rounds(const RoundsLaunch &R, bool gaunt)
{
    const int nm = R.P->nm;
    if (gaunt) {
        switch (nm) {
        case 1: return rounds_t<1, 1, true>(R);
        case 4: return rounds_t<1, 2, true>(R);
        case 9: return rounds_t<2, 4, true>(R);
        case 16: return rounds_t<2, 7, true>(R);
        case 25: return rounds_t<4, 11, true>(R);
        case 36: return rounds_t<5, 16, true>(R);
        case 49: return rounds_t<7, 22, true>(R);
        case 64: return rounds_t<8, 29, true>(R);
        default: return cudaErrorInvalidValue;
        }
    }
    switch ((nm + 7) / 8) {
    case 1: return rounds_t<1, 1, false>(R);
    case 2: return rounds_t<2, 1, false>(R);
    case 3: return rounds_t<3, 1, false>(R);
    case 4: return rounds_t<4, 1, false>(R);
    case 5: return rounds_t<5, 1, false>(R);
    case 6: return rounds_t<6, 1, false>(R);
    case 7: return rounds_t<7, 1, false>(R);
    case 8: return rounds_t<8, 1, false>(R);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace c3d
