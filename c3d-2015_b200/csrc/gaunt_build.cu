// Gaunt coefficient tables built on the device (c3d_gaunt_build, include/c3d_b200.h).
//
// beta_ij (nm2 values per pair i, j < nm) is the least-squares solution of
// M2 beta_ij = m_i .* m_j over the quadrature points, with M2 the nq x nm2 matrix of the
// harmonics up to degree 2N (src/init.cpp:288-316: one Householder QR of M2, then one
// solve per pair); the sparse table keeps |beta| > threshold in (i*nm + j, k) order
// (src/init.cpp:318-336). Here the work is laid out for the GPU:
//  * the QR of the one shared matrix runs in one CTA on a column-major copy (column c
//    contiguous, so every access is coalesced), one warp per trailing column;
//  * the nm^2 solves run one warp per pair: the right-hand side lives in shared memory,
//    the reflectors and R are read from L2 (2 MB at N = 6, Q = 28);
//  * the CSR compaction counts per row, scans, then writes each row with a ballot prefix,
//    so the column order is the host's.
// The sums are warp and block reductions, not the host's sequential loops, so the tables
// agree with the host build (host/tables.c) to rounding, not bit for bit.
#include "../../include/c3d_b200.h"
#include "c3d_common.cuh"

#include <algorithm>
#include <cmath>
#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace c3d {
void set_last_error(const std::string &msg); // reported by c3d_last_error (api.cu)
} // namespace c3d

using namespace c3d;

namespace {

constexpr int QR_THREADS = 1024;
constexpr int SOLVE_SMEM_MAX = 200 * 1024; // dynamic shared memory of one solve CTA

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// In-place Householder QR of the column-major nq x nm2 matrix V (column c at V + c nq,
// nq >= nm2): R on and above the diagonal, the reflectors' tails below it (v_0 = 1
// implicit), tau[nm2]. The reflector of column j follows the host's householder(): beta =
// -sign(alpha) hypot(alpha, |x_tail|), tau = (beta - alpha) / beta, tail / (alpha - beta);
// tau = 0 (no reflection) when the tail is zero or j is the last row.
__global__ void __launch_bounds__(QR_THREADS)
    gaunt_qr_kernel(int nq, int nm2, double *__restrict__ V, double *__restrict__ tau)
{
    __shared__ double red[QR_THREADS / 32];
    __shared__ double sTau, sScale;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = QR_THREADS / 32;
    for (int j = 0; j < nm2; ++j) {
        double *col = V + (size_t)j * nq;
        double ss = 0.0;
        for (int r = j + 1 + tid; r < nq; r += QR_THREADS)
            ss += col[r] * col[r];
        ss = warp_sum(ss);
        if (lane == 0)
            red[warp] = ss;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int w = 0; w < NW; ++w)
                t += red[w];
            const double xnorm = sqrt(t);
            double ta = 0.0, s = 1.0;
            if (xnorm > 0.0 && j < nq - 1) {
                const double alpha = col[j];
                const double beta = -(alpha >= 0.0 ? 1.0 : -1.0) * hypot(alpha, xnorm);
                ta = (beta - alpha) / beta;
                s = alpha - beta;
                col[j] = beta;
            }
            sTau = ta;
            sScale = s;
            tau[j] = ta;
        }
        __syncthreads();
        const double ta = sTau; // the same for every thread: the block skips together
        if (ta == 0.0)
            continue;
        const double s = sScale;
        for (int r = j + 1 + tid; r < nq; r += QR_THREADS)
            col[r] /= s;
        __syncthreads();
        // (I - tau v v^T) on the trailing columns, one warp per column
        for (int c = j + 1 + warp; c < nm2; c += NW) {
            double *cc = V + (size_t)c * nq;
            double d = 0.0;
            for (int r = j + 1 + lane; r < nq; r += 32)
                d += col[r] * cc[r];
            d = (warp_sum(d) + cc[j]) * ta;
            __syncwarp();
            if (lane == 0)
                cc[j] -= d;
            for (int r = j + 1 + lane; r < nq; r += 32)
                cc[r] -= d * col[r];
        }
        __syncthreads();
    }
}

// One warp per pair (i, j), pair = i nm + j: y = m_i .* m_j (M2t holds the first nm
// columns of M2 column-major), y <- Q^T y with the reflectors of V, then R x = y[0, nm2)
// by back substitution; x is row pair of the dense table beta[nm^2][nm2].
__global__ void gaunt_solve_kernel(int nm, int nm2, int nq, const double *__restrict__ M2t,
                                   const double *__restrict__ V, const double *__restrict__ tau,
                                   double *__restrict__ beta)
{
    extern __shared__ double gsy[]; // per warp: y[nq], x[nm2]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pair = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pair >= nm * nm)
        return; // a whole warp; the kernel has no block barrier
    const int i = pair / nm, j = pair % nm;
    double *y = gsy + (size_t)warp * (nq + nm2);
    double *x = y + nq;
    const double *mi = M2t + (size_t)i * nq, *mj = M2t + (size_t)j * nq;
    for (int r = lane; r < nq; r += 32)
        y[r] = mi[r] * mj[r];
    __syncwarp();
    for (int c = 0; c < nm2; ++c) {
        const double ta = tau[c];
        if (ta == 0.0)
            continue;
        const double *v = V + (size_t)c * nq;
        double d = 0.0;
        for (int r = c + 1 + lane; r < nq; r += 32)
            d += v[r] * y[r];
        d = (warp_sum(d) + y[c]) * ta;
        __syncwarp();
        if (lane == 0)
            y[c] -= d;
        for (int r = c + 1 + lane; r < nq; r += 32)
            y[r] -= d * v[r];
        __syncwarp();
    }
    for (int k = nm2 - 1; k >= 0; --k) {
        double s = 0.0;
        for (int l = k + 1 + lane; l < nm2; l += 32)
            s += V[(size_t)l * nq + k] * x[l];
        s = y[k] - warp_sum(s);
        if (lane == 0)
            x[k] = s / V[(size_t)k * nq + k];
        __syncwarp();
    }
    for (int k = lane; k < nm2; k += 32)
        beta[(size_t)pair * nm2 + k] = x[k];
}

// Entries above the threshold per row of the dense table, one warp per row.
__global__ void gaunt_count_kernel(int rows, int nm2, const double *__restrict__ beta, double thr,
                                   int *__restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= rows)
        return;
    int n = 0;
    for (int k = lane; k < nm2; k += 32)
        n += fabs(beta[(size_t)row * nm2 + k]) > thr ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        n += __shfl_xor_sync(0xffffffffu, n, o);
    if (lane == 0)
        cnt[row] = n;
}

// Row pointers from the counts (rows <= 2^16: one thread walks them).
__global__ void gaunt_scan_kernel(int rows, const int *__restrict__ cnt, int *__restrict__ rowPtr)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    int p = 0;
    for (int r = 0; r < rows; ++r) {
        rowPtr[r] = p;
        p += cnt[r];
    }
    rowPtr[rows] = p;
}

// CSR values and columns, one warp per row; a ballot prefix keeps the column order.
__global__ void gaunt_fill_kernel(int rows, int nm2, const double *__restrict__ beta, double thr,
                                  const int *__restrict__ rowPtr, int *__restrict__ colInd,
                                  double *__restrict__ val)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= rows)
        return;
    int p = rowPtr[row];
    for (int k0 = 0; k0 < nm2; k0 += 32) {
        const int k = k0 + lane;
        const double v = k < nm2 ? beta[(size_t)row * nm2 + k] : 0.0;
        const bool keep = k < nm2 && fabs(v) > thr;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int at = p + __popc(m & ((1u << lane) - 1u));
            colInd[at] = k;
            val[at] = v;
        }
        p += __popc(m);
    }
}

} // namespace

extern "C" c3d_status c3d_gaunt_build(int nm, int nm2, int nq, const double *M2, double threshold,
                                      double *beta, int *rowPtr, long long capacity, int *colInd,
                                      double *val, long long *nnz)
{
    if (!M2 || !nnz)
        return set_last_error("c3d_gaunt_build: M2 and nnz are required"), C3D_ERR_INVALID;
    if (nm < 1 || nm2 < nm || nq < nm2 || (long long)nm * nm > (1 << 16))
        return set_last_error("c3d_gaunt_build: need 1 <= nm <= nm2 <= nq and nm^2 <= 65536"),
               C3D_ERR_INVALID;
    if ((size_t)(nq + nm2) * 8 > (size_t)SOLVE_SMEM_MAX)
        return set_last_error("c3d_gaunt_build: nq + nm2 too large for one warp's shared memory"),
               C3D_ERR_INVALID;
    if (!(threshold >= 0.0) || !std::isfinite(threshold))
        return set_last_error("c3d_gaunt_build: threshold must be finite and >= 0"),
               C3D_ERR_INVALID;
    if (rowPtr && (!colInd || !val || capacity < 0))
        return set_last_error("c3d_gaunt_build: rowPtr needs colInd, val and capacity"),
               C3D_ERR_INVALID;
    const int rows = nm * nm;
    // column-major copy of M2: the QR's working matrix, and (its first nm columns) m_i
    std::vector<double> cm((size_t)nq * nm2);
    for (int q = 0; q < nq; ++q)
        for (int k = 0; k < nm2; ++k)
            cm[(size_t)k * nq + q] = M2[(size_t)q * nm2 + k];
    double *dV = nullptr, *dM = nullptr, *dTau = nullptr, *dBeta = nullptr, *dVal = nullptr;
    int *dCnt = nullptr, *dRow = nullptr, *dCol = nullptr;
    cudaStream_t st = nullptr;
    auto release = [&]() {
        if (st)
            cudaStreamSynchronize(st);
        cudaFree(dV);
        cudaFree(dM);
        cudaFree(dTau);
        cudaFree(dBeta);
        cudaFree(dVal);
        cudaFree(dCnt);
        cudaFree(dRow);
        cudaFree(dCol);
        if (st)
            cudaStreamDestroy(st);
    };
    auto cudaFail = [&](cudaError_t e, const char *what) {
        release();
        cudaGetLastError();
        set_last_error(std::string("c3d_gaunt_build: ") + what + ": " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? C3D_ERR_OOM : C3D_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess)
        return st = nullptr, cudaFail(e, "stream");
    if ((e = cudaMalloc(&dV, cm.size() * 8)) != cudaSuccess ||
        (e = cudaMalloc(&dM, (size_t)nm * nq * 8)) != cudaSuccess ||
        (e = cudaMalloc(&dTau, (size_t)nm2 * 8)) != cudaSuccess ||
        (e = cudaMalloc(&dBeta, (size_t)rows * nm2 * 8)) != cudaSuccess ||
        (e = cudaMalloc(&dCnt, (size_t)rows * 4)) != cudaSuccess ||
        (e = cudaMalloc(&dRow, (size_t)(rows + 1) * 4)) != cudaSuccess)
        return cudaFail(e, "device allocation");
    if ((e = cudaMemcpyAsync(dV, cm.data(), cm.size() * 8, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(dM, dV, (size_t)nm * nq * 8, cudaMemcpyDeviceToDevice, st)) !=
            cudaSuccess)
        return cudaFail(e, "copy");
    gaunt_qr_kernel<<<1, QR_THREADS, 0, st>>>(nq, nm2, dV, dTau);
    int wpb = (int)std::min<size_t>(8, (size_t)SOLVE_SMEM_MAX / ((size_t)(nq + nm2) * 8));
    const size_t smem = (size_t)wpb * (nq + nm2) * 8;
    if ((e = cudaFuncSetAttribute(gaunt_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
        return cudaFail(e, "shared memory attribute");
    gaunt_solve_kernel<<<(rows + wpb - 1) / wpb, 32 * wpb, smem, st>>>(nm, nm2, nq, dM, dV, dTau,
                                                                       dBeta);
    gaunt_count_kernel<<<(rows + 7) / 8, 256, 0, st>>>(rows, nm2, dBeta, threshold, dCnt);
    gaunt_scan_kernel<<<1, 32, 0, st>>>(rows, dCnt, dRow);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return cudaFail(e, "launch");
    std::vector<int> hRow((size_t)rows + 1);
    if ((e = cudaMemcpyAsync(hRow.data(), dRow, hRow.size() * 4, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cudaFail(e, "row pointers");
    const long long count = hRow[rows];
    *nnz = count;
    if (beta && (e = cudaMemcpyAsync(beta, dBeta, (size_t)rows * nm2 * 8, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess)
        return cudaFail(e, "dense table");
    if (rowPtr) {
        if (count > capacity) {
            release();
            set_last_error("c3d_gaunt_build: " + std::to_string(count) +
                           " entries above the threshold exceed capacity " +
                           std::to_string(capacity));
            return C3D_ERR_INVALID;
        }
        std::copy(hRow.begin(), hRow.end(), rowPtr);
        if (count > 0) {
            if ((e = cudaMalloc(&dCol, (size_t)count * 4)) != cudaSuccess ||
                (e = cudaMalloc(&dVal, (size_t)count * 8)) != cudaSuccess)
                return cudaFail(e, "device allocation");
            gaunt_fill_kernel<<<(rows + 7) / 8, 256, 0, st>>>(rows, nm2, dBeta, threshold, dRow,
                                                              dCol, dVal);
            if ((e = cudaGetLastError()) != cudaSuccess ||
                (e = cudaMemcpyAsync(colInd, dCol, (size_t)count * 4, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(val, dVal, (size_t)count * 8, cudaMemcpyDeviceToHost, st)) !=
                    cudaSuccess)
                return cudaFail(e, "sparse table");
        }
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cudaFail(e, "synchronize");
    release();
    return C3D_OK;
}
