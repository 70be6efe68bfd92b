// Device kernels of the plate solver.
//
//   ke_kernel          element stiffness, FP64 (and an FP32 copy), per element
//   binv_kernel        3x3 block diagonal, constrained rule, FP64 inversion
//   applyk_*_kernel    y = K x colour by colour (test hook, reference layout)
//   pcg_kernel         persistent cooperative PCG: the whole solve in one
//                      launch, one grid-wide wait per iteration
//
// PCG form.  The reference runs textbook PCG (pcg.ts:98-215) with three
// reductions per iteration.  Here the Chronopoulos-Gear recurrence computes
// the same iterates in exact arithmetic with one reduction per iteration:
//   w = A u;  gamma = (r,u), delta = (w,u), rho = (r,r)     [one reduction]
//   beta = gamma/gamma_prev;  alpha = gamma/(delta - beta*gamma/alpha_prev)
//   p = u + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;  u = M^-1 r
// (delta - beta*gamma/alpha_prev equals p.Ap, the reference's breakdown
// quantity).  Each thread block owns a node set; it also keeps copies of
// r, u, p, s for its ghost nodes (nodes of its elements owned elsewhere)
// and updates them with the same arithmetic as their owners, so after the
// single wait it only needs the owners' w of its ghosts -- published before
// the wait -- and no second halo exchange.
#pragma once

#include <cstdint>

#include "element.cuh"

namespace pg {

struct PcgResult {
    int status;
    int iterations;
    int converged;
    int stop_reason;
    double final_residual;
    double true_rel_residual;
    double b_norm;
    int reliable_updates;
    int wait_failures;
};

struct PcgArgs {
    int G, npe, C, Nn;
    const int* node_off;
    const int* nown;
    const int* nodes;
    const int* elem_off;
    const int* color_off;
    const int* elems;
    const int* lnode;
    const double* ke64;   // [Ne][nd*nd]
    const float* ke32;    // [Ne][nd*nd]
    const double* binv64; // [Nn][9]
    const float* binv32;  // [Nn][9]
    const uint8_t* cons;  // [3Nn]
    const float* F;       // [3Nn]
    double* x;            // [3Nn]
    double* xch64;        // [2][3Nn]
    float* xch32;         // [2][3Nn]
    double* partials;     // [2][G][4]
    unsigned int* bar;
    int* abort_flag;
    PcgResult* res;
    double tol;
    int maxit;
    int stop_rule;
    unsigned long long timeout_ns;
    int ke_smem;
    int sm_nloc, sm_nown, sm_nel;  // shared-memory strides (max over parts)
    int reliable_interval;
    double reliable_delta;
};

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------

__global__ void ke_kernel(int Ne, int npe, const float* __restrict__ nodes,
                          const uint32_t* __restrict__ elements, double E, double nu, double t,
                          const float* __restrict__ elem_t, double* __restrict__ ke64,
                          float* __restrict__ ke32) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    double c[8];
    for (int k = 0; k < npe; k++) {
        const uint32_t n = elements[(size_t)e * npe + k];
        c[2 * k] = nodes[2 * n];
        c[2 * k + 1] = nodes[2 * n + 1];
    }
    const double te = elem_t ? (double)elem_t[e] : t;
    double Ke[144];
    const int kk = npe == 4 ? 144 : 81;
    if (npe == 4)
        q4_ke(c, E, nu, te, Ke);
    else
        dkt_ke(c, E, nu, te, Ke);
    for (int i = 0; i < kk; i++) {
        ke64[(size_t)e * kk + i] = Ke[i];
        if (ke32) ke32[(size_t)e * kk + i] = (float)Ke[i];
    }
}

// computeBlockDiagonal + invertBlockDiagonal (solver.ts:188-304), per node.
__global__ void binv_kernel(int Nn, int npe, const int* __restrict__ inc_ptr,
                            const int* __restrict__ inc_idx, const double* __restrict__ ke64,
                            const uint8_t* __restrict__ cons, double* __restrict__ binv64,
                            float* __restrict__ binv32) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    const int nd = 3 * npe, kk = nd * nd;
    double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = inc_ptr[n]; q < inc_ptr[n + 1]; q++) {
        const int e = inc_idx[q] >> 2, k = inc_idx[q] & 3;
        const double* K = ke64 + (size_t)e * kk;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) b[r * 3 + c] += K[(3 * k + r) * nd + 3 * k + c];
    }
    const bool wc = cons[3 * n], xc = cons[3 * n + 1], yc = cons[3 * n + 2];
    double o[9];
    bool ident = wc && xc && yc;
    if (!ident) {
        if (wc) { b[0] = 1; b[1] = 0; b[2] = 0; b[3] = 0; b[6] = 0; }
        if (xc) { b[4] = 1; b[1] = 0; b[7] = 0; b[3] = 0; b[5] = 0; }
        if (yc) { b[8] = 1; b[2] = 0; b[5] = 0; b[6] = 0; b[7] = 0; }
        const double a00 = b[0], a01 = b[1], a02 = b[2], a10 = b[3], a11 = b[4], a12 = b[5];
        const double a20 = b[6], a21 = b[7], a22 = b[8];
        const double det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
                           a02 * (a10 * a21 - a11 * a20);
        if (fabs(det) < 1e-30) {
            ident = true;
        } else {
            const double id = 1.0 / det;
            o[0] = id * (a11 * a22 - a12 * a21);
            o[1] = id * (a02 * a21 - a01 * a22);
            o[2] = id * (a01 * a12 - a02 * a11);
            o[3] = id * (a12 * a20 - a10 * a22);
            o[4] = id * (a00 * a22 - a02 * a20);
            o[5] = id * (a02 * a10 - a00 * a12);
            o[6] = id * (a10 * a21 - a11 * a20);
            o[7] = id * (a01 * a20 - a00 * a21);
            o[8] = id * (a00 * a11 - a01 * a10);
        }
    }
    for (int i = 0; i < 9; i++) {
        const double v = ident ? ((i % 4 == 0) ? 1.0 : 0.0) : o[i];
        binv64[(size_t)n * 9 + i] = v;
        if (binv32) binv32[(size_t)n * 9 + i] = (float)v;
    }
}

// One colour of y += K x (elements of a colour share no node: no atomics).
__global__ void applyk_color_kernel(int cnt, const uint32_t* __restrict__ list, int npe,
                                    const uint32_t* __restrict__ elements,
                                    const double* __restrict__ ke64, const double* __restrict__ x,
                                    double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t e = list[i];
    const int nd = 3 * npe;
    int dof[12];
    double xl[12];
    for (int k = 0; k < npe; k++)
        for (int d = 0; d < 3; d++) {
            dof[3 * k + d] = (int)elements[(size_t)e * npe + k] * 3 + d;
            xl[3 * k + d] = x[dof[3 * k + d]];
        }
    const double* K = ke64 + (size_t)e * nd * nd;
    for (int r = 0; r < nd; r++) {
        double s = 0;
        for (int c = 0; c < nd; c++) s += K[r * nd + c] * xl[c];
        y[dof[r]] += s;
    }
}

__global__ void bc_copy_kernel(int n, const uint8_t* __restrict__ cons,
                               const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && cons[i]) y[i] = x[i];
}

// ---------------------------------------------------------------------------
// grid-wide wait with a time limit
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Every block arrives once per wait; the wait ends when the arrival count
// reaches target = waits_so_far * G.  A block that sees the abort flag, or
// waits longer than timeout_ns, returns false (and raises the flag), so a
// lost block ends the kernel with PG_ETIMEOUT instead of a hang.
__device__ bool grid_wait(const PcgArgs& a, unsigned int target, int* s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        red_release_add(a.bar, 1u);
        int ok = 1;
        const unsigned long long t0 = gtimer();
        while (ld_acquire(a.bar) < target) {
            if (*(volatile int*)a.abort_flag) { ok = 0; break; }
            if (gtimer() - t0 >= a.timeout_ns) {
                atomicExch(a.abort_flag, 1);
                atomicAdd(&a.res->wait_failures, 1);
                ok = 0;
                break;
            }
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// ---------------------------------------------------------------------------
// block / grid reductions (fixed order: identical bits in every block)
// ---------------------------------------------------------------------------

template <int K>
__device__ void block_sum(double (&v)[K], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) red[warp * K + k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            v[k] = lane < nw ? red[lane * K + k] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
    __syncthreads();
}

// Sums slot values k < K over all G blocks; result in out[k] (shared).
template <int K>
__device__ void grid_sum(const double* __restrict__ slots, int G, double* out) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double v[K];
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = 0.0;
        for (int b = lane; b < G; b += 32)
#pragma unroll
            for (int k = 0; k < K; k++) v[k] += __ldcg(slots + (size_t)b * 4 + k);
#pragma unroll
        for (int k = 0; k < K; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < K; k++) out[k] = v[k];
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// element-by-element K.u for the owned rows of a block
// ---------------------------------------------------------------------------

__device__ __forceinline__ int sym_index(int i, int j, int nd) {
    if (i > j) { const int t = i; i = j; j = t; }
    return i * nd - (i * (i - 1)) / 2 + (j - i);
}

// y[owned dofs] += sum over part elements of Ke u_e, colour by colour; one
// thread per (element, row); rows of ghost nodes are skipped.
template <typename T, int NPE>
__device__ void matvec_owned(const T* __restrict__ u, T* __restrict__ y, int no, int nel, int C,
                             const int* __restrict__ coff, const int* __restrict__ ln,
                             const T* __restrict__ kes, const T* __restrict__ keg,
                             const int* __restrict__ elems, bool ks) {
    constexpr int ND = 3 * NPE, KK = ND * ND;
    for (int c = 0; c < C; c++) {
        const int cs = coff[c], cnt = coff[c + 1] - cs;
        for (int t = threadIdx.x; t < cnt * ND; t += blockDim.x) {
            const int row = t / cnt, el = cs + (t - row * cnt);
            const int rn = ln[el * NPE + row / 3];
            if (rn >= no) continue;
            int nn[NPE];
#pragma unroll
            for (int k = 0; k < NPE; k++) nn[k] = ln[el * NPE + k] * 3;
            T acc = T(0);
            if (ks) {
#pragma unroll
                for (int col = 0; col < ND; col++)
                    acc += kes[sym_index(row, col, ND) * nel + el] * u[nn[col / 3] + col % 3];
            } else {
                const T* K = keg + (size_t)elems[el] * KK + row * ND;
#pragma unroll
                for (int col = 0; col < ND; col++) acc += __ldg(K + col) * u[nn[col / 3] + col % 3];
            }
            y[rn * 3 + row % 3] += acc;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// persistent PCG (FP64)
// ---------------------------------------------------------------------------

enum { STOP_CONVERGED = 0, STOP_MAX_ITER = 1, STOP_BREAKDOWN = 2, STOP_ZERO_RHS = 3 };
enum { ST_OK = 0, ST_TIMEOUT = 4, ST_NONFINITE = 5 };

template <int NPE>
__global__ void __launch_bounds__(512, 1) pcg_fp64_kernel(PcgArgs a) {
    constexpr int ND = 3 * NPE;
    extern __shared__ __align__(16) unsigned char smem[];
    const int g = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int n0 = a.node_off[g], nloc = a.node_off[g + 1] - n0, no = a.nown[g];
    const int e0 = a.elem_off[g], nel = a.elem_off[g + 1] - e0;
    const int C = a.C;
    const int* __restrict__ gnodes = a.nodes + n0;
    const int* __restrict__ gelems = a.elems + e0;

    // shared-memory carve-up (doubles first, then ints and bytes)
    double* r = (double*)smem;
    double* u = r + 3 * a.sm_nloc;
    double* p = u + 3 * a.sm_nloc;
    double* s = p + 3 * a.sm_nloc;
    double* w = s + 3 * a.sm_nloc;
    double* x = w + 3 * a.sm_nloc;
    double* bi = x + 3 * a.sm_nown;
    double* red = bi + 9 * a.sm_nloc;
    double* scal = red + 32 * 4;
    double* kes = scal + 8;
    int* ln = (int*)(kes + (a.ke_smem ? (size_t)a.sm_nel * (ND * (ND + 1) / 2) : 0));
    int* coff = ln + NPE * a.sm_nel;
    int* iflag = coff + (C + 1);
    unsigned char* cm = (unsigned char*)(iflag + 4);

    // ---- load the part ----
    for (int k = tid; k < 3 * nloc; k += nt) {
        const int gd = gnodes[k / 3] * 3 + k % 3;
        const unsigned char c = a.cons[gd];
        cm[k] = c;
        r[k] = c ? 0.0 : (double)a.F[gd];
        p[k] = 0.0;
        s[k] = 0.0;
        if (k < 3 * no) x[k] = 0.0;
    }
    for (int k = tid; k < 9 * nloc; k += nt) bi[k] = a.binv64[(size_t)gnodes[k / 9] * 9 + k % 9];
    for (int k = tid; k < NPE * nel; k += nt) ln[k] = a.lnode[(size_t)e0 * NPE + k];
    for (int k = tid; k <= C; k += nt) coff[k] = a.color_off[(size_t)g * (C + 1) + k] - e0;
    if (a.ke_smem) {
        constexpr int NS = ND * (ND + 1) / 2;
        for (int k = tid; k < NS * nel; k += nt) {
            const int el = k % nel, q = k / nel;
            int i = 0, rem = q;
            while (rem >= ND - i) { rem -= ND - i; i++; }
            kes[k] = a.ke64[(size_t)gelems[el] * ND * ND + i * ND + i + rem];
        }
    }
    __syncthreads();
    for (int nd = tid; nd < nloc; nd += nt) {
        const double* B = bi + 9 * nd;
        const double r0 = r[3 * nd], r1 = r[3 * nd + 1], r2 = r[3 * nd + 2];
        u[3 * nd] = B[0] * r0 + B[1] * r1 + B[2] * r2;
        u[3 * nd + 1] = B[3] * r0 + B[4] * r1 + B[5] * r2;
        u[3 * nd + 2] = B[6] * r0 + B[7] * r1 + B[8] * r2;
    }
    __syncthreads();

    double gamma_prev = 1.0, alpha_prev = 1.0, bnorm = 0.0;
    unsigned int waits = 0;
    int it = 0, par = 0, stop = -1, status = ST_OK, iters = 0;
    double final_res = 0.0;

    for (;; it++) {
        // ---- w = A u on owned rows ----
        for (int k = tid; k < 3 * no; k += nt) w[k] = 0.0;
        __syncthreads();
        matvec_owned<double, NPE>(u, w, no, nel, C, coff, ln, kes, a.ke64, gelems, a.ke_smem != 0);
        double v[3] = {0.0, 0.0, 0.0};
        double* xo = a.xch64 + (size_t)par * 3 * a.Nn;
        for (int k = tid; k < 3 * no; k += nt) {
            if (cm[k]) w[k] = u[k];
            v[0] += r[k] * u[k];
            v[1] += w[k] * u[k];
            v[2] += r[k] * r[k];
            __stcg(xo + gnodes[k / 3] * 3 + k % 3, w[k]);
        }
        block_sum<3>(v, red);
        if (tid == 0) {
            double* slot = a.partials + ((size_t)par * a.G + g) * 4;
            __stcg(slot, v[0]);
            __stcg(slot + 1, v[1]);
            __stcg(slot + 2, v[2]);
        }
        if (!grid_wait(a, (++waits) * a.G, iflag)) { status = ST_TIMEOUT; break; }
        grid_sum<3>(a.partials + (size_t)par * a.G * 4, a.G, scal);
        const double gamma = scal[0], delta = scal[1], rho = scal[2];

        // ---- decisions (identical in every block) ----
        const double rn = sqrt(rho);
        if (!isfinite(gamma) || !isfinite(delta) || !isfinite(rho)) { status = ST_NONFINITE; break; }
        if (it == 0) {
            bnorm = rn;
            if (bnorm < 1e-30) { stop = STOP_ZERO_RHS; iters = 0; final_res = 0.0; break; }
        } else if ((a.stop_rule == 0 && rn < a.tol) || rn / bnorm < a.tol) {
            stop = STOP_CONVERGED; iters = it; final_res = rn; break;
        }
        if (it >= a.maxit) { stop = STOP_MAX_ITER; iters = it; final_res = rn; break; }
        const double beta = it == 0 ? 0.0 : gamma / gamma_prev;
        const double pap = it == 0 ? delta : delta - beta * gamma / alpha_prev;
        if (fabs(pap) < 1e-30) { stop = STOP_BREAKDOWN; iters = it + 1; final_res = rn; break; }
        const double alpha = gamma / pap;
        gamma_prev = gamma;
        alpha_prev = alpha;

        // ---- ghost w from their owners ----
        for (int k = 3 * no + tid; k < 3 * nloc; k += nt) w[k] = __ldcg(xo + gnodes[k / 3] * 3 + k % 3);
        __syncthreads();
        // ---- vector updates on owned and ghost DOFs ----
        for (int k = tid; k < 3 * nloc; k += nt) {
            const double pk = u[k] + beta * p[k];
            const double sk = w[k] + beta * s[k];
            p[k] = pk;
            s[k] = sk;
            if (k < 3 * no) x[k] += alpha * pk;
            r[k] -= alpha * sk;
        }
        __syncthreads();
        for (int nd = tid; nd < nloc; nd += nt) {
            const double* B = bi + 9 * nd;
            const double r0 = r[3 * nd], r1 = r[3 * nd + 1], r2 = r[3 * nd + 2];
            u[3 * nd] = B[0] * r0 + B[1] * r1 + B[2] * r2;
            u[3 * nd + 1] = B[3] * r0 + B[4] * r1 + B[5] * r2;
            u[3 * nd + 2] = B[6] * r0 + B[7] * r1 + B[8] * r2;
        }
        __syncthreads();
        par ^= 1;
    }

    // ---- write x; FP64 true residual F - K x ----
    for (int k = tid; k < 3 * no; k += nt) a.x[gnodes[k / 3] * 3 + k % 3] = x[k];
    if (status == ST_OK) {
        par ^= 1;
        double* xo = a.xch64 + (size_t)par * 3 * a.Nn;
        for (int k = tid; k < 3 * no; k += nt) __stcg(xo + gnodes[k / 3] * 3 + k % 3, x[k]);
        if (!grid_wait(a, (++waits) * a.G, iflag)) {
            status = ST_TIMEOUT;
        } else {
            // p <- x on owned and ghost DOFs
            for (int k = tid; k < 3 * nloc; k += nt)
                p[k] = k < 3 * no ? x[k] : __ldcg(xo + gnodes[k / 3] * 3 + k % 3);
            for (int k = tid; k < 3 * no; k += nt) w[k] = 0.0;
            __syncthreads();
            matvec_owned<double, NPE>(p, w, no, nel, C, coff, ln, kes, a.ke64, gelems, a.ke_smem != 0);
            double v[2] = {0.0, 0.0};
            for (int k = tid; k < 3 * no; k += nt) {
                const double f = cm[k] ? 0.0 : (double)a.F[gnodes[k / 3] * 3 + k % 3];
                const double kx = cm[k] ? p[k] : w[k];
                const double d = (cm[k] ? 0.0 : f) - (cm[k] ? kx : w[k]);
                v[0] += d * d;
                v[1] += f * f;
            }
            block_sum<2>(v, red);
            double* slots = a.partials + (size_t)par * a.G * 4;
            if (tid == 0) {
                __stcg(slots + (size_t)g * 4, v[0]);
                __stcg(slots + (size_t)g * 4 + 1, v[1]);
            }
            if (!grid_wait(a, (++waits) * a.G, iflag)) {
                status = ST_TIMEOUT;
            } else if (g == 0) {
                grid_sum<2>(slots, a.G, scal);
                if (tid == 0) {
                    a.res->true_rel_residual = scal[1] > 0 ? sqrt(scal[0] / scal[1]) : 0.0;
                }
            }
        }
    }
    if (g == 0 && tid == 0) {
        a.res->status = status;
        a.res->iterations = iters;
        a.res->converged = (stop == STOP_CONVERGED || stop == STOP_ZERO_RHS) ? 1 : 0;
        a.res->stop_reason = stop < 0 ? STOP_MAX_ITER : stop;
        a.res->final_residual = final_res;
        a.res->b_norm = bnorm;
    }
}

}  // namespace pg
