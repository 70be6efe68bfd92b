// Device set-up of the two-level preconditioner's coarse space (the dense
// steps of build_coarse in plan.cpp, which the host keeps for batches):
//   coarse_assemble_kernel  A_c = P^T K P from the FP64 element matrices,
//                           one thread per element, FP64 atomics into A_c
//   coarse_factor_kernel    one block: right-looking Cholesky of A_c with
//                           numerically dependent modes dropped (pivot <=
//                           1e-13 max diagonal), the inverse of L, and
//                           A_c^-1 = L^-T L^-1
//   coarse_rows_kernel      each part's rows of A_c^-1 (FP64 and FP32)
// P holds one aggregate per part with the plate's three rigid-body modes
// (w = 1; w = dy, theta_x = 1/h; w = dx, theta_y = -1/h about the
// aggregate centre, h its size), zero on constrained DOFs.
#pragma once

#include <cstdint>

namespace pg {

template <int NPE>
__global__ void coarse_assemble_kernel(int Ne, int C, const float* __restrict__ nodes,
                                       const uint32_t* __restrict__ elements, const uint8_t* __restrict__ cons,
                                       const int* __restrict__ owner, const double* __restrict__ geom,
                                       const double* __restrict__ ke64, double* __restrict__ Ac) {
    constexpr int ND = 3 * NPE;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const double* K = ke64 + (size_t)e * ND * ND;
    double Ph[NPE][3][3];
    int ag[NPE];
    for (int i = 0; i < NPE; i++) {
        const int n = (int)elements[(size_t)e * NPE + i];
        const int a = owner[n];
        ag[i] = a;
        const double ih = geom[3 * a + 2];
        const double dx = ((double)nodes[2 * n] - geom[3 * a]) * ih;
        const double dy = ((double)nodes[2 * n + 1] - geom[3 * a + 1]) * ih;
        const double v[3][3] = {{1.0, dy, dx}, {0.0, ih, 0.0}, {0.0, 0.0, -ih}};
        for (int d = 0; d < 3; d++)
            for (int m = 0; m < 3; m++) Ph[i][d][m] = cons[3 * n + d] ? 0.0 : v[d][m];
    }
    for (int i = 0; i < NPE; i++)
        for (int j = 0; j < NPE; j++) {
            double T[3][3];  // K_ij Phi_j
            for (int d = 0; d < 3; d++)
                for (int m = 0; m < 3; m++) {
                    double acc = 0.0;
                    for (int f = 0; f < 3; f++) acc += K[(3 * i + d) * ND + 3 * j + f] * Ph[j][f][m];
                    T[d][m] = acc;
                }
            for (int mi = 0; mi < 3; mi++)
                for (int mj = 0; mj < 3; mj++) {
                    double acc = 0.0;
                    for (int d = 0; d < 3; d++) acc += Ph[i][d][mi] * T[d][mj];
                    if (acc != 0.0) atomicAdd(Ac + (size_t)(3 * ag[i] + mi) * C + 3 * ag[j] + mj, acc);
                }
        }
}

constexpr int kCoarseThreads = 1024;

// Dynamic shared memory of coarse_factor_kernel: a column of C doubles, and
// two 32 x 65 tiles for the product of phase 3.
__host__ __device__ constexpr size_t coarse_factor_smem(int C) {
    return (size_t)(C > 2 * 32 * 65 ? C : 2 * 32 * 65) * sizeof(double);
}

// Block-wide maximum of v (every thread receives it).
__device__ __forceinline__ double block_max(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
    return m;
}

// One block of kCoarseThreads threads, dynamic shared memory coarse_factor_smem(C).
// L, Lt and Ainv ([C][C], row-major) start zeroed; keep [C] receives 1 for
// kept modes; *dropped the count of dropped ones.
//   1. right-looking Cholesky of A_c in L (lower triangle), column by
//      column: the pivot, the column scaled below it (staged in shared
//      memory), then the trailing update row by row (a warp per row,
//      lanes along the row, so every access is coalesced); a mode whose
//      pivot is <= 1e-13 max diagonal is dropped (its column zero)
//   2. Y = L^-1 by forward substitution over all columns at once, kept
//      transposed (Lt[c][r] = Y[r][c]): at step i row i of Y is scaled by
//      1 / L_ii and subtracted from the rows below (warps over columns c,
//      lanes along r); dropped rows are zero
//   3. A_c^-1 = Y^T Y: entry (i, j), j <= i, is Lt[i] . Lt[j] over k >= i,
//      in 32 x 32 tiles staged through shared memory
__global__ void __launch_bounds__(kCoarseThreads) coarse_factor_kernel(int C, const double* __restrict__ Ac,
                                                                       double* L, double* Lt, double* Ainv,
                                                                       int* keep, int* dropped) {
    extern __shared__ double col[];  // [C] (phases 1, 2), two tiles (phase 3)
    __shared__ double red[kCoarseThreads / 32];
    __shared__ double s_inv;
    __shared__ int s_keep;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    double mx = 0.0;
    for (int i = tid; i < C; i += blockDim.x) mx = fmax(mx, Ac[(size_t)i * C + i]);
    const double dmax = block_max(mx, red);
    for (int i = warp; i < C; i += nw)
        for (int k = lane; k <= i; k += 32) L[(size_t)i * C + k] = Ac[(size_t)i * C + k];
    int nd = 0;
    __syncthreads();
    // 1. Cholesky
    for (int j = 0; j < C; j++) {
        if (tid == 0) {
            const double d = L[(size_t)j * C + j];
            s_keep = d > 1e-13 * dmax;
            keep[j] = s_keep;
            const double ljj = s_keep ? sqrt(d) : 0.0;
            L[(size_t)j * C + j] = ljj;
            s_inv = s_keep ? 1.0 / ljj : 0.0;
        }
        __syncthreads();
        const bool kj = s_keep != 0;
        nd += kj ? 0 : 1;
        const double inv = s_inv;
        for (int i = j + 1 + tid; i < C; i += blockDim.x) {
            const double v = L[(size_t)i * C + j] * inv;  // 0 for a dropped mode
            L[(size_t)i * C + j] = v;
            col[i] = v;
        }
        __syncthreads();
        if (kj)
            for (int i = j + 1 + warp; i < C; i += nw) {
                const double ci = col[i];
                double* li = L + (size_t)i * C;
                for (int k = j + 1 + lane; k <= i; k += 32) li[k] -= ci * col[k];
            }
        __syncthreads();
    }
    if (tid == 0) *dropped = nd;
    // 2. Y = L^-1, transposed into Lt
    for (int i = tid; i < C; i += blockDim.x) Lt[(size_t)i * C + i] = keep[i] ? 1.0 : 0.0;
    __syncthreads();
    for (int i = 0; i < C; i++) {
        const double lii = L[(size_t)i * C + i];
        const double inv = lii > 0.0 ? 1.0 / lii : 0.0;
        // row i of Y (column i of Lt, entries c <= i) scaled; below-diagonal
        // column i of L staged
        for (int c = tid; c <= i; c += blockDim.x) Lt[(size_t)c * C + i] *= inv;
        for (int r = i + 1 + tid; r < C; r += blockDim.x) col[r] = L[(size_t)r * C + i];
        __syncthreads();
        for (int c = warp; c <= i; c += nw) {
            double* ltc = Lt + (size_t)c * C;
            const double yic = ltc[i];
            if (yic != 0.0)
                for (int r = i + 1 + lane; r < C; r += 32) ltc[r] -= col[r] * yic;
        }
        __syncthreads();
    }
    // 3. A_c^-1 = L^-T L^-1: entry (i, j), j <= i, is Lt[i] . Lt[j] over
    //    k >= i; 32 x 32 tiles of entries (a thread each), the rows of Lt
    //    they need staged in shared memory 64 columns at a time
    __syncthreads();
    double* ta = col;                 // [32][65] rows I0 .. I0 + 31 of Lt
    double* tb = col + 32 * 65;       // [32][65] rows J0 .. J0 + 31
    const int ty = tid >> 5, tx = tid & 31;  // entry (I0 + ty, J0 + tx)
    const int nt = (C + 31) / 32;
    for (int I = 0; I < nt; I++)
        for (int J = 0; J <= I; J++) {
            const int I0 = 32 * I, J0 = 32 * J;
            double acc = 0.0;
            for (int k0 = I0; k0 < C; k0 += 64) {
                for (int q = tid; q < 32 * 64; q += blockDim.x) {
                    const int rr = q >> 6, kk = q & 63, k = k0 + kk;
                    const int ia = I0 + rr, ib = J0 + rr;
                    ta[rr * 65 + kk] = (ia < C && k < C) ? Lt[(size_t)ia * C + k] : 0.0;
                    tb[rr * 65 + kk] = (ib < C && k < C) ? Lt[(size_t)ib * C + k] : 0.0;
                }
                __syncthreads();
#pragma unroll 8
                for (int kk = 0; kk < 64; kk++) acc += ta[ty * 65 + kk] * tb[tx * 65 + kk];
                __syncthreads();
            }
            const int i = I0 + ty, j = J0 + tx;
            if (i < C && j <= i) {
                Ainv[(size_t)i * C + j] = acc;
                Ainv[(size_t)j * C + i] = acc;
            }
        }
}

// Part rows of A_c^-1: out64/out32[r][k] = Ainv[src[r]][k].
__global__ void coarse_rows_kernel(int rows, int C, const int* __restrict__ src, const double* __restrict__ Ainv,
                                   double* __restrict__ out64, float* __restrict__ out32) {
    const long total = (long)rows * C;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int r = (int)(q / C), k = (int)(q - (long)r * C);
        const double v = Ainv[(size_t)src[r] * C + k];
        out64[q] = v;
        out32[q] = (float)v;
    }
}

}  // namespace pg
