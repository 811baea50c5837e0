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
// arithmetic bit for bit (unfused operations in its order). The flux sums
// over directions in the reference's order, with fused multiply-adds.
#include "c3d_common.cuh"

namespace c3d {


// ---------------------------------------------------------------- ghost fill

// Two periodic ghost layers per face over interior ranges of the other two axes
// (no edges or corners). The three face groups read only interior cells, so
// they run as one launch.
__global__ void ghost_fill_kernel(GridDims g, double *__restrict__ u)
{
    const int nm = g.nm;
    const long long fx = 4LL * g.ny * g.nz, fy = 4LL * g.nx * g.nz, fz = 4LL * g.nx * g.ny;
    const long long total = (fx + fy + fz) * nm;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = (int)(e % nm);
        long long f = e / nm;
        long long dst, src;
        if (f < fx) {
            int side = (int)(f / (2LL * g.ny * g.nz)); // 0: low ghosts, 1: high ghosts
            long long r = f % (2LL * g.ny * g.nz);
            int l = (int)(r / ((long long)g.ny * g.nz));
            long long r2 = r % ((long long)g.ny * g.nz);
            int j = 2 + (int)(r2 / g.nz), k = 2 + (int)(r2 % g.nz);
            if (side == 0) {
                dst = g.cell(l, j, k);
                src = g.cell(g.nx + l, j, k);
            } else {
                dst = g.cell(g.nx + 2 + l, j, k);
                src = g.cell(2 + l, j, k);
            }
        } else if (f < fx + fy) {
            f -= fx;
            int side = (int)(f / (2LL * g.nx * g.nz));
            long long r = f % (2LL * g.nx * g.nz);
            int l = (int)(r / ((long long)g.nx * g.nz));
            long long r2 = r % ((long long)g.nx * g.nz);
            int i = 2 + (int)(r2 / g.nz), k = 2 + (int)(r2 % g.nz);
            if (side == 0) {
                dst = g.cell(i, l, k);
                src = g.cell(i, g.ny + l, k);
            } else {
                dst = g.cell(i, g.ny + 2 + l, k);
                src = g.cell(i, 2 + l, k);
            }
        } else {
            f -= fx + fy;
            int side = (int)(f / (2LL * g.nx * g.ny));
            long long r = f % (2LL * g.nx * g.ny);
            int l = (int)(r / ((long long)g.nx * g.ny));
            long long r2 = r % ((long long)g.nx * g.ny);
            int i = 2 + (int)(r2 / g.ny), j = 2 + (int)(r2 % g.ny);
            if (side == 0) {
                dst = g.cell(i, j, l);
                src = g.cell(i, j, g.nz + l);
            } else {
                dst = g.cell(i, j, g.nz + 2 + l);
                src = g.cell(i, j, 2 + l);
            }
        }
        u[dst * nm + m] = u[src * nm + m];
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

// Interior-cell index -> grid cell index.
__device__ __forceinline__ long long interior_cell(const GridDims &g, long long n)
{
    int k = (int)(n % g.nz);
    long long r = n / g.nz;
    int j = (int)(r % g.ny);
    int i = (int)(r / g.ny);
    return g.cell(i + 2, j + 2, k + 2);
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

// ---------------------------------------------------------------- kinetic flux

// psi[(q - q0) * nall + c] = exp(alpha_c . m_q) (M_N) or alpha_c . m_q (P_N), for all
// cells c and q0 <= q < q0 + nqc. The dot product runs in the reference's order
// (moment index ascending, unfused), src/flux_kinetic.cpp:21-37.
template <int NM>
__global__ void __launch_bounds__(128)
    ansatz_kernel(GridDims g, const double *__restrict__ alpha, const double *__restrict__ M, int q0,
                  int nqc, int isPn, double *__restrict__ psi)
{
    constexpr int TB = 128;
    extern __shared__ double sh[];
    double *sM = sh;             // nqc x NM
    double *sA = sh + nqc * NM;  // TB x NM
    const long long nall = g.nall();
    for (int e = threadIdx.x; e < nqc * NM; e += TB)
        sM[e] = M[(long long)q0 * NM + e];
    long long c0 = (long long)blockIdx.x * TB;
    long long n = nall - c0 < TB ? nall - c0 : TB;
    for (long long e = threadIdx.x; e < n * NM; e += TB)
        sA[e] = alpha[c0 * NM + e];
    __syncthreads();
    if (threadIdx.x >= n)
        return;
    double a[NM];
#pragma unroll
    for (int i = 0; i < NM; ++i)
        a[i] = sA[threadIdx.x * NM + i];
    long long c = c0 + threadIdx.x;
    for (int q = 0; q < nqc; ++q) {
        double z = 0.0;
#pragma unroll
        for (int i = 0; i < NM; ++i)
            z = __dadd_rn(z, __dmul_rn(a[i], sM[q * NM + i]));
        psi[(long long)q * nall + c] = isPn ? z : exp(z);
    }
}

__device__ __forceinline__ double sgn1(double x) { return x >= 0.0 ? 1.0 : -1.0; }

// minmod / slopefit, src/flux_kinetic.cpp:45-60 (MIN/MAX/SIGN macros of src/utils.h:12-14).
__device__ __forceinline__ double minmod(double x, double y)
{
    double s = sgn1(x);
    double ax = fabs(x), b = y * s;
    double mn = ax < b ? ax : b;
    double mx = 0.0 > mn ? 0.0 : mn;
    return s * mx;
}
__device__ __forceinline__ double slopefit(double th, double l, double c, double r)
{
    return minmod(th * (r - c), minmod(0.5 * (r - l), th * (c - l)));
}

// Upwind MUSCL difference along one axis, src/flux_kinetic.cpp:130-189.
__device__ __forceinline__ double axis_flux(double om, double w, double th, const double *p,
                                            long long c, long long s)
{
    double k1, k2, k3, k4, f;
    if (om > 0) {
        k1 = p[c - 2 * s];
        k2 = p[c - s];
        k3 = p[c];
        k4 = p[c + s];
        f = k3 + 0.5 * slopefit(th, k2, k3, k4) - k2 - 0.5 * slopefit(th, k1, k2, k3);
    } else {
        k1 = p[c - s];
        k2 = p[c];
        k3 = p[c + s];
        k4 = p[c + 2 * s];
        f = k3 - 0.5 * slopefit(th, k2, k3, k4) - k2 + 0.5 * slopefit(th, k1, k2, k3);
    }
    return f * om * w;
}

// flux_m(c) (+)= sum_{q in chunk} m_q[m] (Fx/dx + Fy/dy + Fz/dz), one thread per interior
// cell, moments in registers. Directions are staged through shared memory SUB at a time
// (7 KB for M_6), so several blocks share an SM. 1/dx is precomputed (exact for the
// power-of-two spacings of the benchmark grids, within one rounding otherwise).
// accumulate = 0 on the first chunk.
template <int NM>
__global__ void __launch_bounds__(128)
    kinetic_stencil_kernel(GridDims g, const double *__restrict__ psi, const double *__restrict__ M,
                           const double *__restrict__ w, const double *__restrict__ xi,
                           const double *__restrict__ eta, const double *__restrict__ mu, int q0,
                           int nqc, double rdx, double rdy, double rdz, double theta,
                           int accumulate, double *__restrict__ flux)
{
    constexpr int SUB = 16;
    __shared__ double sM[SUB * NM];
    __shared__ double sO[SUB * 4]; // xi, eta, mu, w
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool active = n < g.ninterior();
    const long long nall = g.nall();
    long long c = active ? interior_cell(g, n) : 0;
    const long long sx = (long long)g.nyg() * g.nzg(), sy = g.nzg(), sz = 1;
    double acc[NM];
    if (accumulate && active) {
#pragma unroll
        for (int m = 0; m < NM; ++m)
            acc[m] = flux[c * NM + m];
    } else {
#pragma unroll
        for (int m = 0; m < NM; ++m)
            acc[m] = 0.0;
    }
    for (int s0 = 0; s0 < nqc; s0 += SUB) {
        int ns = nqc - s0 < SUB ? nqc - s0 : SUB;
        __syncthreads();
        for (int e = threadIdx.x; e < ns * NM; e += blockDim.x)
            sM[e] = M[(long long)(q0 + s0) * NM + e];
        for (int q = threadIdx.x; q < ns; q += blockDim.x) {
            sO[4 * q + 0] = xi[q0 + s0 + q];
            sO[4 * q + 1] = eta[q0 + s0 + q];
            sO[4 * q + 2] = mu[q0 + s0 + q];
            sO[4 * q + 3] = w[q0 + s0 + q];
        }
        __syncthreads();
        if (!active)
            continue;
        for (int q = 0; q < ns; ++q) {
            const double *p = psi + (long long)(s0 + q) * nall;
            double wq = sO[4 * q + 3];
            double fx = axis_flux(sO[4 * q + 0], wq, theta, p, c, sx);
            double fy = axis_flux(sO[4 * q + 1], wq, theta, p, c, sy);
            double fz = axis_flux(sO[4 * q + 2], wq, theta, p, c, sz);
            double sv = fx * rdx + fy * rdy + fz * rdz;
#pragma unroll
            for (int m = 0; m < NM; ++m)
                acc[m] = fma(sM[q * NM + m], sv, acc[m]);
        }
    }
    if (!active)
        return;
#pragma unroll
    for (int m = 0; m < NM; ++m)
        flux[c * NM + m] = acc[m];
}

// ---------------------------------------------------------------- kinetic flux on the tensor pipe

__device__ __forceinline__ void dmma_g(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// psi[(q - q0) * nall + c] = exp(z) (M_N) or z (P_N) with z = alpha_c . m_q, for a tile of
// 64 cells x 32 directions per CTA: Z = A M^T on the FP64 tensor pipe (m8n8k4; warp w owns
// cells 8w..8w+7, four 8-direction tiles, K = moments in steps of 4).
template <int NT>
__global__ void __launch_bounds__(256)
    ansatz_dmma_kernel(GridDims g, const double *__restrict__ alpha, const double *__restrict__ M,
                       int q0, int nqc, int isPn, double *__restrict__ psi)
{
    constexpr int NMP = 8 * NT;
    constexpr int KS = (NMP + 3) / 4;      // k-steps of 4 moments
    constexpr int AS = 4 * KS + 4;         // row stride of the alpha tile (== 4 mod 16 doubles
    constexpr int MS = 4 * KS + 4;         //   when 4*KS is a multiple of 16; conflict-light)
    extern __shared__ double ansatzSmem[]; // sA[64 * AS], sM[32 * MS]
    double *sA = ansatzSmem;
    double *sM = ansatzSmem + 64 * AS;
    const int nm = g.nm;
    const long long nall = g.nall();
    const long long c0 = (long long)blockIdx.x * 64;
    const int qb = blockIdx.y * 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < 64 * AS; e += 256) {
        int r = e / AS, m = e % AS;
        long long c = c0 + r;
        sA[e] = (c < nall && m < nm) ? alpha[c * nm + m] : 0.0;
    }
    for (int e = tid; e < 32 * MS; e += 256) {
        int r = e / MS, m = e % MS;
        int q = qb + r;
        sM[e] = (q < nqc && m < nm) ? M[(long long)(q0 + q) * nm + m] : 0.0;
    }
    __syncthreads();
    double acc[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j)
        acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < KS; ++kk) {
        double a = sA[(8 * warp + (lane >> 2)) * AS + 4 * kk + (lane & 3)];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double b = sM[(8 * j + (lane >> 2)) * MS + 4 * kk + (lane & 3)];
            dmma_g(acc[j][0], acc[j][1], a, b);
        }
    }
    const long long c = c0 + 8 * warp + (lane >> 2);
    if (c >= nall)
        return;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int q = qb + 8 * j + 2 * (lane & 3) + e2;
            if (q < nqc) {
                double z = acc[j][e2];
                psi[(long long)q * nall + c] = isPn ? z : exp(z);
            }
        }
}

// flux(c) (+)= sum_q m_q (Fx/dx + Fy/dy + Fz/dz) for 64 interior cells (consecutive in the
// interior numbering) per CTA: per 32-direction chunk the limited upwind differences
// S[q][cell] go to shared memory, then F += S^T M on the FP64 tensor pipe (warp w owns
// cells 8w..8w+7 and every 8-moment tile).
template <int NT>
__global__ void __launch_bounds__(256)
    kinetic_dmma_kernel(GridDims g, const double *__restrict__ psi, const double *__restrict__ M,
                        const double *__restrict__ w, const double *__restrict__ xi,
                        const double *__restrict__ eta, const double *__restrict__ mu, int q0,
                        int nqc, double rdx, double rdy, double rdz, double theta,
                        int accumulate, double *__restrict__ flux)
{
    constexpr int NMP = 8 * NT;
    constexpr int CS = 68; // S tile row stride (cells)
    constexpr int MS = NMP + 4 + ((NMP + 4) % 16 == 4 ? 0 : (20 - (NMP + 4) % 16) % 16);
    __shared__ double sS[32 * CS];
    __shared__ double sM[32 * MS];
    __shared__ double sO[32 * 4];
    __shared__ long long sCell[64];
    const int nm = g.nm;
    const long long nall = g.nall(), nint = g.ninterior();
    const long long n0 = (long long)blockIdx.x * 64;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long sx = (long long)g.nyg() * g.nzg(), sy = g.nzg(), sz = 1;
    if (tid < 64)
        sCell[tid] = (n0 + tid < nint) ? interior_cell(g, n0 + tid) : -1;
    double acc[NT][2];
    const long long myc = n0 + 8 * warp + (lane >> 2);
    __syncthreads();
    if (accumulate && myc < nint) {
        long long c = sCell[8 * warp + (lane >> 2)];
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2) {
                int m = 8 * j + 2 * (lane & 3) + e2;
                acc[j][e2] = (m < nm) ? flux[c * nm + m] : 0.0;
            }
    } else {
#pragma unroll
        for (int j = 0; j < NT; ++j)
            acc[j][0] = acc[j][1] = 0.0;
    }
    for (int qb = 0; qb < nqc; qb += 32) {
        int nq = nqc - qb < 32 ? nqc - qb : 32;
        __syncthreads();
        for (int e = tid; e < 32 * MS; e += 256) {
            int r = e / MS, m = e % MS;
            sM[e] = (r < nq && m < nm) ? M[(long long)(q0 + qb + r) * nm + m] : 0.0;
        }
        if (tid < 32) {
            int q = q0 + qb + tid;
            bool ok = tid < nq;
            sO[4 * tid + 0] = ok ? xi[q] : 0.0;
            sO[4 * tid + 1] = ok ? eta[q] : 0.0;
            sO[4 * tid + 2] = ok ? mu[q] : 0.0;
            sO[4 * tid + 3] = ok ? w[q] : 0.0;
        }
        __syncthreads();
        // stencil: thread handles cell (tid % 64) for directions tid/64 + 4i
        {
            const int cl = tid & 63;
            const long long c = sCell[cl];
            for (int qq = tid >> 6; qq < 32; qq += 4) {
                double sv = 0.0;
                if (c >= 0 && qq < nq) {
                    const double *p = psi + (long long)(qb + qq) * nall;
                    double wq = sO[4 * qq + 3];
                    double fx = axis_flux(sO[4 * qq + 0], wq, theta, p, c, sx);
                    double fy = axis_flux(sO[4 * qq + 1], wq, theta, p, c, sy);
                    double fz = axis_flux(sO[4 * qq + 2], wq, theta, p, c, sz);
                    sv = fx * rdx + fy * rdy + fz * rdz;
                }
                sS[qq * CS + cl] = sv;
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            double a = sS[(4 * kk + (lane & 3)) * CS + 8 * warp + (lane >> 2)];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                double b = sM[(4 * kk + (lane & 3)) * MS + 8 * j + (lane >> 2)];
                dmma_g(acc[j][0], acc[j][1], a, b);
            }
        }
    }
    if (myc >= nint)
        return;
    long long c = sCell[8 * warp + (lane >> 2)];
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
            int m = 8 * j + 2 * (lane & 3) + e2;
            if (m < nm)
                flux[c * nm + m] = acc[j][e2];
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

cudaError_t launch_ghost_fill(const GridDims &g, double *u, int numSMs, cudaStream_t st)
{
    long long total = (4LL * g.ny * g.nz + 4LL * g.nx * g.nz + 4LL * g.nx * g.ny) * g.nm;
    ghost_fill_kernel<<<grid_for(total, 256, numSMs), 256, 0, st>>>(g, u);
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

template <int NT>
static cudaError_t kinetic_t(const GridDims &g, const double *alpha, const double *M,
                             const double *w, const double *xi, const double *eta, const double *mu,
                             int nq, int qChunk, double dx, double dy, double dz, double theta,
                             int isPn, double *psi, double *flux, cudaStream_t st)
{
    for (int q0 = 0; q0 < nq; q0 += qChunk) {
        int nqc = nq - q0 < qChunk ? nq - q0 : qChunk;
        dim3 ga((unsigned)((g.nall() + 63) / 64), (unsigned)((nqc + 31) / 32));
        constexpr int KS = (8 * NT + 3) / 4;
        const size_t smem = (size_t)(64 + 32) * (4 * KS + 4) * sizeof(double);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(ansatz_dmma_kernel<NT>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess)
                return e;
        }
        ansatz_dmma_kernel<NT><<<ga, 256, smem, st>>>(g, alpha, M, q0, nqc, isPn, psi);
        kinetic_dmma_kernel<NT><<<(unsigned)((g.ninterior() + 63) / 64), 256, 0, st>>>(
            g, psi, M, w, xi, eta, mu, q0, nqc, 1.0 / dx, 1.0 / dy, 1.0 / dz, theta, q0 > 0 ? 1 : 0,
            flux);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

cudaError_t launch_kinetic_flux(const GridDims &g, const double *alpha, const double *M,
                                const double *w, const double *xi, const double *eta,
                                const double *mu, int nq, int qChunk, double dx, double dy,
                                double dz, double theta, int isPn, double *psi, double *flux,
                                cudaStream_t st)
{
#define C3D_NT_CASE(NT)                                                                            \
    case NT:                                                                                       \
        return kinetic_t<NT>(g, alpha, M, w, xi, eta, mu, nq, qChunk, dx, dy, dz, theta, isPn,     \
                             psi, flux, st);
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

// Directions per materialised-ansatz chunk (bounded by the HBM budget only).
int kinetic_max_chunk(int nm)
{
    (void)nm;
    return 1 << 20;
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
