// Device set-up of the two-level preconditioner's coarse space (the dense
// steps of build_coarse in plan.cpp, which the host keeps for batches):
//   coarse_assemble_kernel  A_c = P^T K P from the FP64 element matrices,
//                           one thread per element, FP64 atomics into A_c
//   coarse_factor_kernel    one block: left-looking Cholesky of A_c with
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

// sum_{k in [k0, k1)} a[k] b[k] in four interleaved partial sums
__device__ __forceinline__ double cdot4(const double* a, const double* b, int k0, int k1) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
        s0 += a[k] * b[k];
        s1 += a[k + 1] * b[k + 1];
        s2 += a[k + 2] * b[k + 2];
        s3 += a[k + 3] * b[k + 3];
    }
    for (; k < k1; k++) s0 += a[k] * b[k];
    return (s0 + s1) + (s2 + s3);
}

constexpr int kCoarseThreads = 1024;

// One block of kCoarseThreads threads.  L, Lt and Ainv ([C][C]) start
// zeroed; keep [C] receives 1 for kept modes; *dropped the count of
// dropped ones.
__global__ void __launch_bounds__(kCoarseThreads) coarse_factor_kernel(int C, const double* __restrict__ Ac,
                                                                       double* L, double* Lt, double* Ainv,
                                                                       int* keep, int* dropped) {
    __shared__ double red[kCoarseThreads / 32];
    __shared__ double s_val;
    __shared__ int s_keep, s_dropped;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // largest diagonal entry
    double mx = 0.0;
    for (int i = tid; i < C; i += blockDim.x) mx = fmax(mx, Ac[(size_t)i * C + i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
        s_val = m;
        s_dropped = 0;
    }
    __syncthreads();
    const double dmax = s_val;
    __syncthreads();
    // left-looking Cholesky, column by column
    for (int j = 0; j < C; j++) {
        const double* lj = L + (size_t)j * C;
        double part = 0.0;
        for (int k = tid; k < j; k += blockDim.x) part += lj[k] * lj[k];
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
            const double d = Ac[(size_t)j * C + j] - s;
            s_keep = d > 1e-13 * dmax;
            keep[j] = s_keep;
            if (s_keep) {
                s_val = sqrt(d);
                L[(size_t)j * C + j] = s_val;
            } else {
                s_dropped++;
            }
        }
        __syncthreads();
        if (s_keep) {
            const double ljj = s_val;
            for (int i = j + 1 + tid; i < C; i += blockDim.x) {
                const double* li = L + (size_t)i * C;
                L[(size_t)i * C + j] = (Ac[(size_t)i * C + j] - cdot4(li, lj, 0, j)) / ljj;
            }
        }
        __syncthreads();
    }
    if (tid == 0) *dropped = s_dropped;
    // inverse of L, kept transposed (Lt[j][k] = (L^-1)[k][j]): column j of
    // L^-1 by forward substitution, one thread per column
    for (int j = tid; j < C; j += blockDim.x) {
        if (!keep[j]) continue;
        double* lt = Lt + (size_t)j * C;
        lt[j] = 1.0 / L[(size_t)j * C + j];
        for (int i = j + 1; i < C; i++) {
            if (!keep[i]) continue;
            const double* li = L + (size_t)i * C;
            lt[i] = -cdot4(li, lt, j, i) / li[i];
        }
    }
    __syncthreads();
    // A_c^-1 = L^-T L^-1: entry (i, j), j <= i, is Lt[i] . Lt[j] over k >= i
    const long pairs = (long)C * (C + 1) / 2;
    for (long q = tid; q < pairs; q += blockDim.x) {
        // q -> (i, j) with q = i (i + 1) / 2 + j
        int i = (int)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
        while ((long)i * (i + 1) / 2 > q) i--;
        while ((long)(i + 1) * (i + 2) / 2 <= q) i++;
        const int j = (int)(q - (long)i * (i + 1) / 2);
        const double s = cdot4(Lt + (size_t)i * C, Lt + (size_t)j * C, i, C);
        Ainv[(size_t)i * C + j] = s;
        Ainv[(size_t)j * C + i] = s;
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
