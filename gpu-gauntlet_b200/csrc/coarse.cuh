// Device set-up of the two-level preconditioner's coarse space (the dense
// steps of build_coarse in plan.cpp, which the host keeps for batches):
//   coarse_assemble_kernel  A_c = P^T K P from the FP64 element matrices,
//                           one thread per element, FP64 atomics into A_c
//   coarse_factor_kernel    one block: blocked right-looking Cholesky of
//                           A_c with numerically dependent modes dropped
//                           (pivot <= 1e-13 max diagonal), the inverse of L
//                           and A_c^-1 = L^-T L^-1 (coarse_factor_tiles_kernel:
//                           the same unblocked, for C past shared memory)
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

// Dynamic shared memory of coarse_factor_tiles_kernel: two columns of C
// doubles, and two 32 x 65 tiles for the product of phase 3.
__host__ __device__ constexpr size_t coarse_factor_smem(int C) {
    return (size_t)(2 * C > 2 * 32 * 65 ? 2 * C : 2 * 32 * 65) * sizeof(double);
}

// Panel widths of coarse_factor_kernel (Cholesky, inverse of L) and its
// dynamic shared memory: a C x 32 panel of L; a 16-row panel of L^-1 and the
// matching 16 columns of L, C x 17 each.
constexpr int kPanelChol = 32, kPanelInv = 16;
__host__ __device__ constexpr size_t coarse_factor_blocked_smem(int C) {
    const size_t a = (size_t)C * (kPanelChol + 1), b = 2 * (size_t)C * (kPanelInv + 1), c = 2 * 32 * 65;
    return (a > b ? (a > c ? a : c) : (b > c ? b : c)) * sizeof(double);
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

// A_c^-1 = L^-T L^-1 from Lt (Lt[c][r] = (L^-1)[r][c]): entry (i, j),
// j <= i, is Lt[i] . Lt[j] over k >= i; 32 x 32 tiles of entries, one block
// of kCoarseThreads threads per tile (a thread per entry), the rows of Lt
// the tile needs staged in shared memory 64 columns at a time.  Grid: the
// nt (nt + 1) / 2 tiles of the lower triangle, nt = ceil(C / 32).
__global__ void __launch_bounds__(kCoarseThreads) coarse_inverse_kernel(int C, const double* __restrict__ Lt,
                                                                        double* __restrict__ Ainv) {
    __shared__ double ta[32 * 65];  // rows I0 .. I0 + 31 of Lt
    __shared__ double tb[32 * 65];  // rows J0 .. J0 + 31
    const int tid = threadIdx.x;
    const int ty = tid >> 5, tx = tid & 31;  // entry (I0 + ty, J0 + tx)
    const int p = blockIdx.x;
    int I = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while (I * (I + 1) / 2 > p) I--;
    while ((I + 1) * (I + 2) / 2 <= p) I++;
    const int J = p - I * (I + 1) / 2;
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

// The unblocked form of coarse_factor_kernel, for a C whose panels do not
// fit in shared memory.  One block of kCoarseThreads threads, dynamic
// shared memory coarse_factor_smem(C).
// L and Lt ([C][C], row-major) start zeroed; keep [C] receives 1 for
// kept modes; *dropped the count of dropped ones.
//   1. right-looking Cholesky of A_c in L (lower triangle), column by
//      column: the pivot, the column scaled below it (staged in shared
//      memory), then the trailing update; a mode whose pivot is <= 1e-13
//      max diagonal is dropped (its column zero).  The next column of the
//      trailing matrix is also kept in shared memory (written by the update),
//      so pivot and scaling read no global memory
//   2. Y = L^-1 by forward substitution over all columns at once, kept
//      transposed (Lt[c][r] = Y[r][c]): at step i row i of Y is scaled by
//      1 / L_ii (and staged) and subtracted from the rows below; dropped
//      rows are zero
// then A_c^-1 = Y^T Y by coarse_inverse_kernel.  The updates of 1 and 2 run over 32 x 32 tiles of their region (warp w,
// lane l: entry (32 I + w, 32 K + l), so every access is coalesced), four
// tiles per round with all loads issued before the stores: the matrices are
// L2-resident and each round costs one L2 round trip.
__device__ __forceinline__ void tile_cursor_next(int& I, int& K, int tri, int nK) {
    if (++K > (tri ? I : nK - 1)) {
        K = 0;
        ++I;
    }
}

__global__ void __launch_bounds__(kCoarseThreads) coarse_factor_tiles_kernel(int C, const double* __restrict__ Ac,
                                                                             double* L, double* Lt, int* keep,
                                                                             int* dropped) {
    extern __shared__ double col[];  // [C] col, [C] nxt (phases 1, 2); two tiles (phase 3)
    double* nxt = col + C;
    __shared__ double red[kCoarseThreads / 32];
    __shared__ double s_inv;
    __shared__ int s_keep;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    double mx = 0.0;
    for (int i = tid; i < C; i += blockDim.x) mx = fmax(mx, Ac[(size_t)i * C + i]);
    const double dmax = block_max(mx, red);
    for (int i = warp; i < C; i += nw)
        for (int k = lane; k <= i; k += 32) L[(size_t)i * C + k] = Ac[(size_t)i * C + k];
    for (int i = tid; i < C; i += blockDim.x) nxt[i] = Ac[(size_t)i * C];
    int nd = 0;
    __syncthreads();
    // 1. Cholesky
    for (int j = 0; j < C; j++) {
        if (tid == 0) {
            const double d = nxt[j];
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
            const double v = nxt[i] * inv;  // 0 for a dropped mode
            L[(size_t)i * C + j] = v;
            col[i] = v;
        }
        __syncthreads();
        const int base = j + 1, m = C - base;
        if (kj && m > 0) {
            // trailing lower triangle rows/columns base .. C-1
            const int nt = (m + 31) >> 5;
            int I = 0, K = 0;
            while (I < nt) {
                double *p0 = nullptr, *p1 = nullptr, *p2 = nullptr, *p3 = nullptr;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
                int n0 = -1, n1 = -1, n2 = -1, n3 = -1;  // row whose next-column entry this is
                auto take = [&](double*& pp, double& ff, int& nn) {
                    if (I >= nt) return;
                    const int i = base + 32 * I + warp, k = base + 32 * K + lane;
                    if (i < C && k <= i) {
                        pp = L + (size_t)i * C + k;
                        ff = col[i] * col[k];
                        if (k == base) nn = i;
                    }
                    tile_cursor_next(I, K, 1, 0);
                };
                take(p0, f0, n0);
                take(p1, f1, n1);
                take(p2, f2, n2);
                take(p3, f3, n3);
                const double v0 = p0 ? *p0 - f0 : 0.0, v1 = p1 ? *p1 - f1 : 0.0;
                const double v2 = p2 ? *p2 - f2 : 0.0, v3 = p3 ? *p3 - f3 : 0.0;
                if (p0) { *p0 = v0; if (n0 >= 0) nxt[n0] = v0; }
                if (p1) { *p1 = v1; if (n1 >= 0) nxt[n1] = v1; }
                if (p2) { *p2 = v2; if (n2 >= 0) nxt[n2] = v2; }
                if (p3) { *p3 = v3; if (n3 >= 0) nxt[n3] = v3; }
            }
        } else if (m > 0) {
            // dropped mode: no update; the next column as it stands
            for (int i = base + tid; i < C; i += blockDim.x) nxt[i] = L[(size_t)i * C + base];
        }
        __syncthreads();
    }
    if (tid == 0) *dropped = nd;
    // 2. Y = L^-1, transposed into Lt; nxt holds row i of Y (entries c <= i)
    for (int i = tid; i < C; i += blockDim.x) Lt[(size_t)i * C + i] = keep[i] ? 1.0 : 0.0;
    __syncthreads();
    for (int i = 0; i < C; i++) {
        const double lii = L[(size_t)i * C + i];
        const double inv = lii > 0.0 ? 1.0 / lii : 0.0;
        for (int c = tid; c <= i; c += blockDim.x) {
            const double y = Lt[(size_t)c * C + i] * inv;
            Lt[(size_t)c * C + i] = y;
            nxt[c] = y;
        }
        for (int r = i + 1 + tid; r < C; r += blockDim.x) col[r] = L[(size_t)r * C + i];
        __syncthreads();
        // Lt[c][r] -= L[r][i] Y[i][c] over c <= i (tile rows) and r > i (tile columns)
        const int base = i + 1, mr = C - base;
        if (mr > 0) {
            const int ntI = (i + 1 + 31) >> 5, ntK = (mr + 31) >> 5;
            int I = 0, K = 0;
            while (I < ntI) {
                double *p0 = nullptr, *p1 = nullptr, *p2 = nullptr, *p3 = nullptr;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
                auto take = [&](double*& pp, double& ff) {
                    if (I >= ntI) return;
                    const int c = 32 * I + warp, r = base + 32 * K + lane;
                    if (c <= i && r < C && nxt[c] != 0.0) {
                        pp = Lt + (size_t)c * C + r;
                        ff = col[r] * nxt[c];
                    }
                    tile_cursor_next(I, K, 0, ntK);
                };
                take(p0, f0);
                take(p1, f1);
                take(p2, f2);
                take(p3, f3);
                const double v0 = p0 ? *p0 - f0 : 0.0, v1 = p1 ? *p1 - f1 : 0.0;
                const double v2 = p2 ? *p2 - f2 : 0.0, v3 = p3 ? *p3 - f3 : 0.0;
                if (p0) *p0 = v0;
                if (p1) *p1 = v1;
                if (p2) *p2 = v2;
                if (p3) *p3 = v3;
            }
        }
        __syncthreads();
    }
}

// One block of kCoarseThreads threads (32 warps), dynamic shared memory
// coarse_factor_blocked_smem(C).  L and Lt ([C][C], row-major) start
// zeroed; keep [C] receives 1 for kept modes; *dropped the count of dropped
// ones.  Blocked, so the O(C^3) work runs from shared memory and each entry
// of the global matrices is read and written once per panel:
//   1. right-looking Cholesky of A_c in L (lower triangle), 32-column
//      panels: the panel (all rows below its top) is loaded into shared
//      memory and factored there column by column (a mode whose pivot is
//      <= 1e-13 max diagonal is dropped: its column zero), written back,
//      and the trailing lower triangle gets the panel's rank-32 update
//      (32 x 32 tiles, four tiles' loads in flight per thread)
//   2. Y = L^-1, kept transposed (Lt[c][r] = Y[r][c]), by forward
//      substitution in 16-row panels: the panel's rows of Y and the
//      matching columns of L in shared memory, the panel solved there, then
//      the rank-16 update of the rows below
// then A_c^-1 = Y^T Y by coarse_inverse_kernel
__global__ void __launch_bounds__(kCoarseThreads) coarse_factor_kernel(int C, const double* __restrict__ Ac,
                                                                       double* L, double* Lt, int* keep,
                                                                       int* dropped) {
    extern __shared__ double cf_smem[];
    double* sm = cf_smem;
    __shared__ double red[kCoarseThreads / 32];
    __shared__ double s_inv;
    __shared__ int s_keep;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int nt = blockDim.x;
    double mx = 0.0;
    for (int i = tid; i < C; i += nt) mx = fmax(mx, Ac[(size_t)i * C + i]);
    const double dmax = block_max(mx, red);
    for (int i = warp; i < C; i += nw)
        for (int k = lane; k <= i; k += 32) L[(size_t)i * C + k] = Ac[(size_t)i * C + k];
    for (int i = tid; i < C; i += nt) Lt[(size_t)i * C + i] = 1.0;  // Y starts as the identity
    int nd = 0;
    __syncthreads();
    // 1. Cholesky
    constexpr int W1 = kPanelChol, S1 = W1 + 1;
    double* P = sm;  // P[r][q] = L[p0 + r][p0 + q], r < C - p0
    for (int p0 = 0; p0 < C; p0 += W1) {
        const int w = min(W1, C - p0), rows = C - p0;
        for (int r = warp; r < rows; r += nw)
            if (lane < w) P[r * S1 + lane] = lane <= r ? L[(size_t)(p0 + r) * C + p0 + lane] : 0.0;
        __syncthreads();
        for (int s = 0; s < w; s++) {
            if (tid == 0) {
                const double d = P[s * S1 + s];
                s_keep = d > 1e-13 * dmax;
                keep[p0 + s] = s_keep;
                const double ljj = s_keep ? sqrt(d) : 0.0;
                P[s * S1 + s] = ljj;
                s_inv = s_keep ? 1.0 / ljj : 0.0;
            }
            __syncthreads();
            const bool kj = s_keep != 0;
            nd += kj ? 0 : 1;
            const double inv = s_inv;
            for (int r = s + 1 + tid; r < rows; r += nt) P[r * S1 + s] *= inv;  // 0 for a dropped mode
            __syncthreads();
            if (kj) {
                const int c = s + 1 + lane;
                if (c < w)
                    for (int r = c + warp; r < rows; r += nw) P[r * S1 + c] -= P[r * S1 + s] * P[c * S1 + s];
            }
            __syncthreads();
        }
        for (int r = warp; r < rows; r += nw)
            if (lane < w && lane <= r) L[(size_t)(p0 + r) * C + p0 + lane] = P[r * S1 + lane];
        // rank-w update of the trailing lower triangle (rows and columns >= p0 + w)
        const int base = p0 + w, m = C - base;
        if (m > 0) {
            const int ntl = (m + 31) >> 5;
            int I = 0, K = 0;
            while (I < ntl) {
                double *p_0 = nullptr, *p_1 = nullptr, *p_2 = nullptr, *p_3 = nullptr;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
                auto take = [&](double*& pp, double& ff) {
                    if (I >= ntl) return;
                    const int i = base + 32 * I + warp, k = base + 32 * K + lane;
                    if (i < C && k <= i) {
                        pp = L + (size_t)i * C + k;
                        const double* pi = P + (i - p0) * S1;
                        const double* pk = P + (k - p0) * S1;
                        double acc = 0.0;
                        for (int q = 0; q < w; q++) acc += pi[q] * pk[q];
                        ff = acc;
                    }
                    tile_cursor_next(I, K, 1, 0);
                };
                take(p_0, f0);
                take(p_1, f1);
                take(p_2, f2);
                take(p_3, f3);
                const double v0 = p_0 ? *p_0 - f0 : 0.0, v1 = p_1 ? *p_1 - f1 : 0.0;
                const double v2 = p_2 ? *p_2 - f2 : 0.0, v3 = p_3 ? *p_3 - f3 : 0.0;
                if (p_0) *p_0 = v0;
                if (p_1) *p_1 = v1;
                if (p_2) *p_2 = v2;
                if (p_3) *p_3 = v3;
            }
        }
        __syncthreads();
    }
    if (tid == 0) *dropped = nd;
    // 2. Y = L^-1 (transposed in Lt)
    constexpr int W2 = kPanelInv, S2 = W2 + 1;
    double* Yp = sm;           // Yp[c][s] = Y[p0 + s][c], c < p0 + w
    double* Lp = sm + C * S2;  // Lp[r][s] = L[p0 + r][p0 + s], r < C - p0
    for (int p0 = 0; p0 < C; p0 += W2) {
        const int w = min(W2, C - p0), ncol = p0 + w, rows = C - p0;
        for (int q = tid; q < ncol * w; q += nt) {
            const int c = q / w, s = q - c * w;
            Yp[c * S2 + s] = Lt[(size_t)c * C + p0 + s];
        }
        for (int q = tid; q < rows * w; q += nt) {
            const int r = q / w, s = q - r * w;
            Lp[r * S2 + s] = L[(size_t)(p0 + r) * C + p0 + s];
        }
        __syncthreads();
        for (int s = 0; s < w; s++) {
            const double lss = Lp[s * S2 + s];
            const double inv = lss > 0.0 ? 1.0 / lss : 0.0;  // a dropped row of Y is zero
            for (int c = tid; c < ncol; c += nt) Yp[c * S2 + s] *= inv;
            __syncthreads();
            const int s2 = s + 1 + lane;
            if (s2 < w)
                for (int c = warp; c < ncol; c += nw) Yp[c * S2 + s2] -= Lp[s2 * S2 + s] * Yp[c * S2 + s];
            __syncthreads();
        }
        for (int q = tid; q < ncol * w; q += nt) {
            const int c = q / w, s = q - c * w;
            Lt[(size_t)c * C + p0 + s] = Yp[c * S2 + s];
        }
        // rank-w update of the rows below: Y[r][c] -= sum_s L[r][p0 + s] Y[p0 + s][c]
        const int base = p0 + w, mr = C - base;
        if (mr > 0) {
            const int ntI = (ncol + 31) >> 5, ntK = (mr + 31) >> 5;
            int I = 0, K = 0;
            while (I < ntI) {
                double *p_0 = nullptr, *p_1 = nullptr, *p_2 = nullptr, *p_3 = nullptr;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
                auto take = [&](double*& pp, double& ff) {
                    if (I >= ntI) return;
                    const int c = 32 * I + warp, r = base + 32 * K + lane;
                    if (c < ncol && r < C) {
                        pp = Lt + (size_t)c * C + r;
                        const double* yc = Yp + c * S2;
                        const double* lr = Lp + (r - p0) * S2;
                        double acc = 0.0;
                        for (int q = 0; q < w; q++) acc += lr[q] * yc[q];
                        ff = acc;
                    }
                    tile_cursor_next(I, K, 0, ntK);
                };
                take(p_0, f0);
                take(p_1, f1);
                take(p_2, f2);
                take(p_3, f3);
                const double v0 = p_0 ? *p_0 - f0 : 0.0, v1 = p_1 ? *p_1 - f1 : 0.0;
                const double v2 = p_2 ? *p_2 - f2 : 0.0, v3 = p_3 ? *p_3 - f3 : 0.0;
                if (p_0) *p_0 = v0;
                if (p_1) *p_1 = v1;
                if (p_2) *p_2 = v2;
                if (p_3) *p_3 = v3;
            }
        }
        __syncthreads();
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
