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

#include <cstdio>

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

// Appends cell c to the list when it still needs a pass.
template <class S>
__device__ void append_if_needed(const S &sl, long long c, int lane, int *listOut,
                                 unsigned int *countOut)
{
    if (lane == 0 && sl.s.need != NEED_NONE) {
        unsigned int pos = atomicAdd(countOut, 1u);
        listOut[pos] = (int)c;
    }
}

} // namespace

constexpr int RW = 8;  // warps (cells) per CTA of the init and pass kernels
constexpr int RWN = 4; // warps (cells) per CTA of the Newton kernel

template <int NT> using TSlot = Slot<NT, true>;

template <int NT>
__global__ void __launch_bounds__(RW * 32)
    rounds_init_kernel(ClosureParams P, long long ncells, const int *__restrict__ cellMap,
                       Outputs O, CellState<NT> *state, int *listOut, unsigned int *countOut)
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
    slot_to_state(sl, state[c], lane);
    append_if_needed(sl, c, lane, listOut, countOut);
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
                             const int *__restrict__ list, int n, CellState<NT> *state,
                             double *__restrict__ momBuf, int *errorFlag)
{
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
                              const int *__restrict__ list, int n, CellState<NT> *state,
                              double *__restrict__ hBuf, int *errorFlag)
{
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

// Newton logic for the listed cells: one warp per cell, RWN cells per CTA, state staged
// in shared memory with H in the tiled layout (TSlot).
// GAUNT: the CTA assembles H_ij = sum_k beta_ijk mom_k (i >= j, the CSR terms of beta in
// the order of src/opt/fobj.cpp:81-99, laid out per tile slot by c3d_set_gaunt) for its
// cells that need a Hessian in one sweep over the tile slots, so that each term is read once
// for RWN cells. A cell's moments sit in its slot's g..rinv vectors, which a Hessian visit
// recomputes afterwards. Otherwise the pass wrote H in tiles to hBuf.
template <int NT, int NT2, bool GAUNT>
__global__ void __launch_bounds__(RWN * 32)
    rounds_newton_kernel(ClosureParams P, double m0, const int *__restrict__ list, int n,
                         CellState<NT> *state, const double *__restrict__ buf,
                         const GauntTerm *__restrict__ stream, int streamLen,
                         Outputs O, int *listOut, unsigned int *countOut)
{
    constexpr int NM2P = 8 * NT2;
    constexpr int NMP = Cfg<NT>::NMP;
    constexpr int LS = TSlot<NT>::LSIZE;
    static_assert(!GAUNT || NM2P <= 4 * NMP, "moments must fit in g, d, alphaOld, rinv");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TSlot<NT> *slots = reinterpret_cast<TSlot<NT> *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pos = blockIdx.x * RWN + warp;
    const bool active = pos < n;
    const long long cell = active ? list[pos] : -1;
    const bool needH = active && state[cell].s.need == NEED_H;
    TSlot<NT> &sl = slots[warp];
    C3D_NCLK_DECL
    if (active) {
        state_to_slot(state[cell], sl, lane, !(GAUNT && needH));
    } else if (lane == 0) {
        sl.s.need = NEED_NONE;
    }
    if (GAUNT) {
        double *mom = sl.scratch(); // g, d, alphaOld, rinv: NM2P <= 4 NMP doubles
        if (needH)
            for (int k = lane; k < NM2P; k += 32)
                mom[k] = buf[(size_t)pos * NM2P + k];
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
    if (!active)
        return;
    C3D_NCLK(O.stats, 0, lane);
    if (sl.s.need == NEED_H) {
        after_hessian(sl, P, O, lane, m0);
        C3D_NCLK(O.stats, 5, lane);
    } else if (sl.s.need == NEED_TRIAL) {
        after_trial(sl, P, O, lane, sl.s.fquad);
        C3D_NCLK(O.stats, 7, lane);
    }
    slot_to_state(sl, state[cell], lane);
    append_if_needed(sl, cell, lane, listOut, countOut);
    C3D_NCLK(O.stats, 6, lane);
}

// ---------------------------------------------------------------- host side

struct RoundsLaunch {
    const ClosureParams *P;
    const double *chunks;      // direct: (NMP+1) x QCP chunks; Gaunt: (NM2P+1) x QCP chunks
    int nm2;                   // Gaunt: extended moments (chunk rows: nm2 + the weight row)
    const GauntTerm *gstream;  // Gaunt: assembly streams, entry s of thread t at s*128 + t
    int streamLen;             // entries per thread
    double m0;                 // M[0][0]
    long long ncells;
    const int *cellMap;        // closure cell i -> grid cell cellMap[i] (null: identity)
    double *u, *alpha;
    int *iters, *iterGamma, *regIdx, *status;
    unsigned long long *failCount, *stats;
    double *gamma, *normG;     // per-cell final gamma and |g| (may be null)
    void *state;               // ncells x rounds_state_bytes(nm)
    int *listA, *listB;        // ncells each
    unsigned int *counts;      // 2 device counters
    unsigned int *hostCount;   // pinned
    double *buf;               // batch x (NM2P or NPK) doubles
    long long batch;           // list entries per pass/Newton launch pair
    int *errorFlag;
    cudaStream_t stream;
    long long *launches;
    long long maxRounds;
};

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
size_t rounds_buf_doubles(int nm, int nm2, bool gaunt)
{
    if (gaunt)
        return (size_t)8 * ((nm2 + 7) / 8);
    const int nt = (nm + 7) / 8;
    return (size_t)64 * nt * (nt + 1) / 2; // the tiled lower triangle
}

template <int NT, int NT2, bool GAUNT> static cudaError_t rounds_t(const RoundsLaunch &R)
{
    const ClosureParams &P = *R.P;
    CellState<NT> *state = reinterpret_cast<CellState<NT> *>(R.state);
    cudaStream_t st = R.stream;
    cudaError_t e;
    size_t slotSmem = RW * sizeof(Slot<NT>);
    e = cudaFuncSetAttribute(rounds_init_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)slotSmem);
    if (e != cudaSuccess)
        return e;
    size_t newtonSmem = RWN * sizeof(TSlot<NT>);
    e = cudaFuncSetAttribute(rounds_newton_kernel<NT, NT2, GAUNT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)newtonSmem);
    if (e != cudaSuccess)
        return e;
    size_t passSmem;
    if (GAUNT) {
        passSmem = GSTAGES * (size_t)(R.nm2 + 1) * QCP * 8 + (size_t)QC * CST2 * 8 +
                   (size_t)(RWP * P.nm + 1) * 8 + GSTAGES * 8;
        e = cudaFuncSetAttribute(rounds_pass_gaunt_kernel<NT, NT2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)passSmem);
    } else {
        passSmem = 3 * (size_t)Cfg<NT>::CHUNK * 8 + (size_t)RW * Cfg<NT>::NMP * 8 + 3 * 8;
        e = cudaFuncSetAttribute(rounds_pass_direct_kernel<NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)passSmem);
    }
    if (e != cudaSuccess)
        return e;
    const double m0 = R.m0;
    const Outputs O{R.u,      R.alpha,     R.iters, R.iterGamma, R.regIdx,
                    R.status, R.failCount, R.stats, R.gamma,     R.normG};

    // round 0: set-up of every cell
    unsigned int *cA = R.counts, *cB = R.counts + 1;
    int *listA = R.listA, *listB = R.listB;
    e = cudaMemsetAsync(cA, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess)
        return e;
    rounds_init_kernel<NT><<<(unsigned)((R.ncells + RW - 1) / RW), RW * 32, slotSmem, st>>>(
        P, R.ncells, R.cellMap, O, state, listA, cA);
    *R.launches += 2;
    e = cudaMemcpyAsync(R.hostCount, cA, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return e;
    long long count = *R.hostCount;
    long long rounds = 0;
    while (count > 0) {
        if (++rounds > R.maxRounds)
            return cudaErrorLaunchTimeout;
        e = cudaMemsetAsync(cB, 0, sizeof(unsigned int), st);
        if (e != cudaSuccess)
            return e;
        for (long long off = 0; off < count; off += R.batch) {
            int nb = (int)((count - off) < R.batch ? (count - off) : R.batch);
            unsigned grid = (unsigned)((nb + RW - 1) / RW);
            if (GAUNT)
                rounds_pass_gaunt_kernel<NT, NT2><<<(unsigned)((nb + RWP - 1) / RWP), RW * 32,
                                                    passSmem, st>>>(
                    P, R.chunks, R.nm2, listA + off, nb, state, R.buf, R.errorFlag);
            else
                rounds_pass_direct_kernel<NT><<<grid, RW * 32, passSmem, st>>>(
                    P, R.chunks, listA + off, nb, state, R.buf, R.errorFlag);
            rounds_newton_kernel<NT, NT2, GAUNT><<<(unsigned)((nb + RWN - 1) / RWN), RWN * 32,
                                                   newtonSmem, st>>>(
                P, m0, listA + off, nb, state, R.buf, R.gstream, R.streamLen, O, listB, cB);
            *R.launches += 2;
            e = cudaGetLastError();
            if (e != cudaSuccess)
                return e;
        }
        *R.launches += 1;
        e = cudaMemcpyAsync(R.hostCount, cB, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return e;
        count = *R.hostCount;
        int *t = listA;
        listA = listB;
        listB = t;
        unsigned int *tc = cA;
        cA = cB;
        cB = tc;
    }
    return cudaSuccess;
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
