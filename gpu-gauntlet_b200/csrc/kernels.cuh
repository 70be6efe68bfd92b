// Device kernels of the plate solver.
//
//   ke_kernel          element stiffness, FP64 (and an FP32 copy), per element
//   binv_kernel        3x3 block diagonal, constrained rule, FP64 inversion
//   task_ke_kernel     the per-task 3 x 3npe blocks the PCG kernels read
//   applyk_*_kernel    y = K x colour by colour (test hook, reference layout;
//                      also the FP64 K x of the set-up and correction steps)
//   power_start_kernel, binv_apply_kernel
//                      lambda_max(D^-1 K) power steps for the Chebyshev smoother
//   residual_*_kernel, add_kernel
//                      FP64 correction after a stagnated mixed solve
//   elem_moments_kernel, node_moments_kernel
//                      nodal bending moments
//   pcg_kernel         persistent cooperative PCG: the whole solve in one
//                      launch, one grid-wide wait per iteration
//   pcg_batch_kernel   many plates, one team of blocks per plate queue
//   (pcg_multi_kernel, several load cases of one plate in lockstep, is in
//   multi.cuh)
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
    int nonfinite_it;          // reduction index where a non-finite value appeared
    int reductions;            // grid-wide reductions performed
    double nonfinite_vals[3];  // gamma, delta, rho at that reduction
    long long phase_cycles[8];  // block 0, see PhaseClock
    unsigned last_tag;         // largest round tag this launch may have written
};

// Byte offsets of the shared-memory arrays of one block (computed on the
// host from the plan's maxima; T is the inner vector type).
struct SmemLayout {
    int r, u, p, s, w, B, yt, kt;  // T
    int x, xl, ytd, red, scal, sp;  // double
    int qw, cs, cv;                 // double, per coarse row of the part: A_c^-1 P^T w,
                                    // A_c^-1 P^T s and c = A_c^-1 P^T r (two copies of cs, cv)
    int ctl;                        // int[4]: decision broadcast
    int clk;                        // long long[8]: phase timers
    int nb, ainv;                   // T: per-node basis data, A_c^-1 rows
    int nslot;                      // int
    int gid, tptr;                 // int
    int tnode;                     // uint16
    int cm;                        // uint8
    int total;
};

// Copies of every block's partial sums in the exchange buffer: each block
// reads one copy, which spreads the pollers of a slot line over kRep lines.
constexpr int kRep = 8;

struct PcgArgs {
    int G, NT, Nn;
    int npe;                     // 3 (DKT) or 4 (Q4): the batch kernel's dispatch
    const int* node_off;
    const int* nown;
    const int* nodes;
    const int* task_off;
    const int* tp_off;
    const int* tptr;
    const uint16_t* task_nodes;  // [NT][npe] -> staged [npe][part tasks]
    const double* kt64;          // [3*nd][NT] task blocks, FP64
    const float* kt32;           // [3*nd][NT] task blocks, FP32
    const double* binv64;        // [Nn][9]
    const float* binv32;         // [Nn][9]
    const uint8_t* cons;         // [3Nn]
    const float* F;              // [3Nn]
    double* x;                   // [3Nn]
    unsigned long long* llv;     // [2][3Nn][2] tagged w / r values of the owners
    unsigned long long* llx;     // [3Nn][2] tagged x values (FP64 residual rounds)
    unsigned long long* llp;     // [2][kRep][G][16] tagged partial sums (kRep copies)
    int* abort_flag;
    PcgResult* res;
    double tol;
    int maxit;
    int stop_rule;
    // round tags of this launch start at tag0 + 1: the exchange buffers keep
    // older tags from earlier launches of the plan, which never match
    unsigned tag0;
    unsigned long long timeout_ns;
    int ke_smem;                 // Ke blocks in shared memory: 0 none, 1 owned tasks, 2 all
    int timing;
    int test_stall;  // test hook: block 0 waits once for a tag nobody writes
    // two-level preconditioner (coarse = 1): u = M_bj r + P A_c^-1 P^T r
    int coarse;
    int C;                      // coarse DOFs, 3 per part
    const int* cagg_off;        // [G+1] aggregates touching each part's nodes
    const int* node_slot;       // per part-local node: slot in its part's aggregate list
    const double* node_basis;   // per part-local node: dx, dy, 1/h
    const int* ainv_off;        // [G+1] first A_c^-1 row of each part
    const double* ainv64;       // [rows][C]
    const float* ainv32;        // [rows][C]
    int ainv_smem;
    int reliable_interval;
    double reliable_delta;
    // polynomial smoother (smoother = 1; needs a plan with a 2-ring halo):
    // u = a D^-1 r - b D^-1 K D^-1 r (the degree-2 Chebyshev step for
    // D^-1 K) in place of u = D^-1 r
    int smoother;
    const int* n1;                  // [G] owned + ring-1 nodes of each part
    double cheb_a, cheb_b;
    int trace_it;                   // iteration traced (-1: none)
    unsigned long long* trace;      // [G][4] globaltimer: start, published, exchanged, end
    SmemLayout L;
};

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------

template <int NPE>
__global__ void ke_kernel(int Ne, const float* __restrict__ nodes,
                          const uint32_t* __restrict__ elements, double E, double nu, double t,
                          const float* __restrict__ elem_t, double* __restrict__ ke64,
                          float* __restrict__ ke32) {
    constexpr int KK = 9 * NPE * NPE;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    double c[2 * NPE];
#pragma unroll
    for (int k = 0; k < NPE; k++) {
        const uint32_t n = elements[(size_t)e * NPE + k];
        c[2 * k] = nodes[2 * n];
        c[2 * k + 1] = nodes[2 * n + 1];
    }
    const double te = elem_t ? (double)elem_t[e] : t;
    double Ke[KK];
    if constexpr (NPE == 4)
        q4_ke(c, E, nu, te, Ke);
    else
        dkt_ke(c, E, nu, te, Ke);
    for (int i = 0; i < KK; i++) {
        ke64[(size_t)e * KK + i] = Ke[i];
        if (ke32) ke32[(size_t)e * KK + i] = (float)Ke[i];
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

// Start vector of the lambda_max(D^-1 K) power iteration: 1 + 0.5 sin(0.7 i),
// 0 on constrained DOFs.
__global__ void power_start_kernel(int n, const uint8_t* __restrict__ cons, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = cons[i] ? 0.0 : 1.0 + 0.5 * sin(0.7 * (double)i);
}

// z = D^-1 y node by node, D^-1 the 3x3 block inverses (FP64).
__global__ void binv_apply_kernel(int Nn, const double* __restrict__ binv, const double* __restrict__ y,
                                  double* __restrict__ z) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Nn) return;
    const double* B = binv + 9 * (size_t)k;
    const double y0 = y[3 * k], y1 = y[3 * k + 1], y2 = y[3 * k + 2];
#pragma unroll
    for (int d = 0; d < 3; d++) z[3 * k + d] = B[3 * d] * y0 + B[3 * d + 1] * y1 + B[3 * d + 2] * y2;
}

// One power step z = D^-1 K x, node by node: (K x)_n gathered from the
// node's incident elements (FP64 element matrices, constrained rows the
// identity), then the node's 3x3 block inverse.  One launch per step in
// place of the colour-ordered K x, the identity rows and the block apply.
template <int NPE>
__global__ void power_step_kernel(int Nn, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                                  const uint32_t* __restrict__ elements, const double* __restrict__ ke64,
                                  const uint8_t* __restrict__ cons, const double* __restrict__ binv,
                                  const double* __restrict__ x, double* __restrict__ z) {
    constexpr int ND = 3 * NPE;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    double y[3] = {0.0, 0.0, 0.0};
    for (int q = inc_ptr[n]; q < inc_ptr[n + 1]; q++) {
        const int e = inc_idx[q] >> 2, k = inc_idx[q] & 3;
        const double* K = ke64 + (size_t)e * ND * ND + 3 * k * ND;
        for (int b = 0; b < NPE; b++) {
            const int m = (int)elements[(size_t)e * NPE + b];
            const double x0 = x[3 * m], x1 = x[3 * m + 1], x2 = x[3 * m + 2];
            for (int d = 0; d < 3; d++)
                y[d] += K[d * ND + 3 * b] * x0 + K[d * ND + 3 * b + 1] * x1 + K[d * ND + 3 * b + 2] * x2;
        }
    }
    for (int d = 0; d < 3; d++)
        if (cons[3 * n + d]) y[d] = x[3 * n + d];
    const double* B = binv + 9 * (size_t)n;
#pragma unroll
    for (int d = 0; d < 3; d++) z[3 * n + d] = B[3 * d] * y[0] + B[3 * d + 1] * y[1] + B[3 * d + 2] * y[2];
}

// r = F - y narrowed to FP32, 0 on constrained rows (y = K x): the load of
// an FP64 correction solve K d = F - K x.  r may be F itself.
__global__ void residual_f32_kernel(int n, const uint8_t* cons, const float* F, const double* y, float* r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = cons[i] ? 0.0f : (float)((double)F[i] - y[i]);
}

// x += a
__global__ void add_kernel(int n, const double* __restrict__ a, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += a[i];
}

// out[0] += sum (F - y)^2, out[1] += sum F^2 over the unconstrained rows
// (y = K x): the true residual of x.  out must start at zero.
__global__ void residual_norms_kernel(int n, const uint8_t* __restrict__ cons, const float* __restrict__ F,
                                      const double* __restrict__ y, double* out) {
    double a = 0.0, b = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!cons[i]) {
            const double f = (double)F[i], r = f - y[i];
            a += r * r;
            b += f * f;
        }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, a);
        atomicAdd(out + 1, b);
    }
}

// ---------------------------------------------------------------------------
// tagged exchange between blocks (no grid barrier)
// ---------------------------------------------------------------------------
// A value a block publishes for other blocks is stored as 64-bit words
// {32-bit payload, 32-bit round tag}; an aligned 64-bit store is
// single-copy atomic, so a reader that sees the current round's tag also
// sees that round's payload -- no fence, no arrival counter, no second
// load.  FP64 values take two words (low and high halves).  Each block
// waits only for the words it needs: every block's partial sums, and its
// own ghosts' values.  Every wait has a time limit: past it the block
// raises the abort flag and the kernel ends with PG_ETIMEOUT.

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// 128-bit forms (p 16-byte aligned).  Each 64-bit half carries its own tag,
// so a reader that sees the two halves from different rounds rejects the
// pair: the pair needs no 128-bit single-copy atomicity.
__device__ __forceinline__ void ld_relaxed2(const unsigned long long* p, unsigned long long& a,
                                            unsigned long long& b) {
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}

__device__ __forceinline__ void st_relaxed2(unsigned long long* p, unsigned long long a,
                                            unsigned long long b) {
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

template <typename T>
struct Tag;

template <>
struct Tag<float> {
    static constexpr int W = 1;
    __device__ static __forceinline__ void put(unsigned long long* p, float v, unsigned f) {
        st_relaxed(p, ((unsigned long long)f << 32) | __float_as_uint(v));
    }
    __device__ static __forceinline__ bool get(const unsigned long long* p, unsigned f, float& v) {
        const unsigned long long a = ld_relaxed(p);
        if ((unsigned)(a >> 32) != f) return false;
        v = __uint_as_float((unsigned)a);
        return true;
    }
};

template <>
struct Tag<double> {
    static constexpr int W = 2;
    __device__ static __forceinline__ void put(unsigned long long* p, double v, unsigned f) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v);
        st_relaxed2(p, ((unsigned long long)f << 32) | (b & 0xffffffffull),
                    ((unsigned long long)f << 32) | (b >> 32));
    }
    __device__ static __forceinline__ bool get(const unsigned long long* p, unsigned f, double& v) {
        unsigned long long a, b;
        ld_relaxed2(p, a, b);
        if ((unsigned)(a >> 32) != f || (unsigned)(b >> 32) != f) return false;
        v = __longlong_as_double((long long)((b << 32) | (a & 0xffffffffull)));
        return true;
    }
};

// 1/x for the PCG scalars: the hardware's approximate reciprocal
// (rcp.approx.ftz.f64) refined by three Newton-Raphson steps
// r <- r + r (1 - x r), each of which about doubles the number of correct
// bits, so the result is within a few ulp of 1/x for normal x.  Shorter than
// a correctly rounded division on the thread-0 path every block waits on.
__device__ __forceinline__ double recip(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const double e = __fma_rn(-x, r, 1.0);
        r = __fma_rn(r, e, r);
    }
    return r;
}

// Time limit of one wait (a spin loop of one thread).  The clock starts at
// the wait's first time check (after 32 failed reads), so a wait that is
// already satisfied costs no timer read.
struct Waiter {
    unsigned long long t0, limit;
    int* abort_flag;
    int* failures;
    unsigned spins;
    __device__ __forceinline__ void start(unsigned long long lim, int* ab, int* fails) {
        limit = lim;
        abort_flag = ab;
        failures = fails;
        spins = 0;
        t0 = 0;
    }
    // false when the wait must give up (time limit, or another block gave up)
    __device__ __forceinline__ bool keep_going() {
        if ((++spins & 31u) != 0) return true;
        const unsigned long long now = gtimer();
        if (spins == 32u) t0 = now;
        if (*(volatile int*)abort_flag) return false;
        if (now - t0 >= limit) {
            atomicExch(abort_flag, 1);
            atomicAdd(failures, 1);
            return false;
        }
        return true;
    }
};

template <typename T>
__device__ __forceinline__ bool poll(const unsigned long long* p, unsigned f, T& v, Waiter& wt) {
    wt.spins = 0;
    while (!Tag<T>::get(p, f, v))
        if (!wt.keep_going()) return false;
    return true;
}

// ---------------------------------------------------------------------------
// block / grid reductions (fixed order: identical bits in every block)
// ---------------------------------------------------------------------------

// Sums KM values (KM a power of two <= 32) over the 32 lanes of a warp by
// recursive halving: at each of the first log2(KM) steps a lane keeps half
// of its values and adds the partner's copy of that half (one shuffle per
// kept value), then the single remaining value is summed over the lanes
// that share it.  Lane l ends with the warp total of value l / (32 / KM):
// KM - 1 + 5 - log2(KM) shuffles instead of 5 KM.  Fixed order.
template <int KM>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[KM]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int lv = 0; (KM >> (lv + 1)) >= 1; lv++) {
        const int h = KM >> (lv + 1), o = 16 >> lv;
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const double keep = up ? v[h + i] : v[i];
            const double send = up ? v[i] : v[h + i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    double t = v[0];
#pragma unroll
    for (int o = 16 / KM; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

// Block-wide totals of the first K (<= KM) of the KM values v, published
// as this block's partial sums: copy r < kRep goes to slots
// pb[r][g][2k, 2k+1].  Every block reads the copy g % kRep, so each slot
// line has about G / kRep readers instead of G.  After the warps' own
// reduce-scatter, lane l of warp 0 adds value k = l mod KM over warps
// l / KM, l / KM + 32 / KM, ... and the 32 / KM lanes of one value finish
// with an xor butterfly: IEEE addition is commutative, so every one of them
// holds the same bits, and each writes its share of the copies.  All
// threads call it; it has one barrier, and warp 0 alone works after it, so
// `red` must not be written again before a later barrier.
template <int KM>
__device__ void block_publish(double (&v)[KM], double* red, unsigned long long* pb, int G, int g,
                              int K, unsigned f) {
    constexpr int SH = 32 / KM;  // lanes that share one value after the reduce-scatter
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double t = warp_reduce_scatter<KM>(v);
    if (lane % SH == 0) red[warp * KM + lane / SH] = t;
    __syncthreads();
    if (warp != 0) return;
    const int k = lane % KM, w0 = lane / KM;
    double tk = 0.0;
    for (int w = w0; w < nw; w += SH) tk += red[w * KM + k];
#pragma unroll
    for (int o = KM; o < 32; o <<= 1) tk += __shfl_xor_sync(0xffffffffu, tk, o);
    if (k < K)
        for (int r = w0; r < kRep; r += SH) Tag<double>::put(pb + ((size_t)r * G + g) * 16 + 2 * k, tk, f);
}

// One exchange round, all threads of the block: waits for the K tagged
// FP64 partial sums of every block (slots of 16 words; staged to
// sp[G * K]) and for the tagged values of this block's ghost DOFs in vector
// buffer vb (written to dst[3 * no .. 3 * nloc)).  Items 0 .. ng - 1 are
// the ghosts, which their owners publish before their partial sums, then
// the partials.  Each thread takes items tid, tid + nt, tid + 2 nt, ...
// with S in flight, and refills a slot with its next item as soon as the
// slot's item has arrived: a ghost frees its slot after one round trip, so
// every partial is being polled by the time the partials come in, and the
// round costs about one L2 round trip after the last block published.
// The block that publishes last finds every other item already there; with
// S slots per thread it reads them in ceil(items / (S nt)) round trips.
// Returns false if a wait gave up.
template <typename T, int S>
__device__ bool exchange_round_s(const unsigned long long* __restrict__ pb, int G, int K,
                               const unsigned long long* __restrict__ vb, T* dst, int no, int nloc,
                               const int* __restrict__ gid, int g, unsigned f, double* sp,
                               Waiter& wt) {
    constexpr int TW = Tag<T>::W;
    const int ng = 3 * (nloc - no), n = ng + G * K, nt = blockDim.x;
    pb += (size_t)(g % kRep) * G * 16;  // the copy of the partials part g reads
    auto addr = [&](int i) -> const unsigned long long* {
        if (i < ng) {
            const int k = 3 * no + i;
            return vb + (size_t)(3 * gid[k / 3] + k % 3) * TW;
        }
        const int q = i - ng;
        return pb + (size_t)(q / K) * 16 + 2 * (q % K);
    };
    // S slots: item index (>= n when empty) and its address
    int it[S];
    const unsigned long long* pp[S];
#pragma unroll
    for (int s = 0; s < S; s++) {
        it[s] = threadIdx.x + s * nt;
        pp[s] = it[s] < n ? addr(it[s]) : nullptr;
    }
    int next = threadIdx.x + S * nt;
    wt.spins = 0;
    for (;;) {
        unsigned long long lo[S], hi[S];
        bool any = false;
#pragma unroll
        for (int s = 0; s < S; s++) {
            lo[s] = hi[s] = 0;
            if (it[s] >= n) continue;
            any = true;
            if (it[s] >= ng || TW == 2) {
                ld_relaxed2(pp[s], lo[s], hi[s]);
            } else {
                lo[s] = ld_relaxed(pp[s]);
                hi[s] = lo[s];
            }
        }
        if (!any) break;
        bool moved = false;
#pragma unroll
        for (int s = 0; s < S; s++) {
            if (it[s] >= n) continue;
            if ((unsigned)(lo[s] >> 32) != f || (unsigned)(hi[s] >> 32) != f) continue;
            const int i = it[s];
            if (i >= ng) {
                sp[i - ng] = __longlong_as_double((long long)((hi[s] << 32) | (lo[s] & 0xffffffffull)));
            } else if constexpr (TW == 2) {
                dst[3 * no + i] = (T)__longlong_as_double((long long)((hi[s] << 32) | (lo[s] & 0xffffffffull)));
            } else {
                dst[3 * no + i] = (T)__uint_as_float((unsigned)lo[s]);
            }
            it[s] = next;
            next += nt;
            pp[s] = it[s] < n ? addr(it[s]) : nullptr;
            moved = true;
        }
        if (!moved && !wt.keep_going()) return false;
    }
    return true;
}

// exchange_round_s with two slots per thread while the round's items fit
// in two per thread (block Jacobi: 3 partials per block), else, when XS
// allows, three (the two-level preconditioner's 6 partials per block and
// the ghosts make about 2.5 items per thread on the 60k-DOF plate, and the
// block that publishes last then reads them in one round trip, not two).
// Measured on that plate, in A/B runs on one B200: with XS = 3 the mixed-
// precision two-level solves run 0.9% (Chebyshev) and 1.8% faster, and the
// mixed block-Jacobi solves, whose rounds keep two slots, 0.9-1.8% slower
// (the larger kernel); in the FP64 kernels the third slot's code made block
// Jacobi 2.4% slower, and in the batch kernel it costs spills, so those
// keep XS = 2.
template <typename T, int XS = 3>
__device__ __forceinline__ bool exchange_round(const unsigned long long* __restrict__ pb, int G, int K,
                                               const unsigned long long* __restrict__ vb, T* dst, int no,
                                               int nloc, const int* __restrict__ gid, int g, unsigned f,
                                               double* sp, Waiter& wt) {
    const int n = 3 * (nloc - no) + G * K;
    if constexpr (XS >= 3)
        if (n > 2 * (int)blockDim.x) return exchange_round_s<T, 3>(pb, G, K, vb, dst, no, nloc, gid, g, f, sp, wt);
    return exchange_round_s<T, 2>(pb, G, K, vb, dst, no, nloc, gid, g, f, sp, wt);
}

// Warp 0: adds the first K of each block's `stride` staged partials
// (sp[G][stride]) in block order (the same bits in every block) into out[K].
template <int K>
__device__ __forceinline__ void sum_partials(const double* __restrict__ sp, int G, int stride,
                                             double* out) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = 0.0;
    for (int b = lane; b < G; b += 32)
#pragma unroll
        for (int k = 0; k < K; k++) v[k] += sp[b * stride + k];
#pragma unroll
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) out[k] = v[k];
}

// ---------------------------------------------------------------------------
// task matvec: the owned rows of K u, one (element, owned node) per thread
// ---------------------------------------------------------------------------

// Task block layout: entry (row r of the node, column c of the rotated
// element) of task t sits at kt[(r * ND + c) * stride + t], so consecutive
// threads read consecutive words.  Task node ids sit at tn[j * ts + t];
// results go to yt[r * ys + t].  Tasks t >= ksplit read their blocks from
// kt2 (stride2) instead of kt (stride): the ring-1 tasks of a 2-ring plan
// when only the owned tasks' blocks are staged in shared memory.
template <int NPE, typename T, typename KT>
__device__ __forceinline__ void task_matvec(const T* __restrict__ u, T* __restrict__ yt, int ys,
                                            int count, const uint16_t* __restrict__ tn, int ts,
                                            const KT* __restrict__ kt, size_t stride,
                                            int ksplit = 1 << 30,
                                            const KT* __restrict__ kt2 = nullptr,
                                            size_t stride2 = 0) {
    constexpr int ND = 3 * NPE;
    // FP64 blocks split the last partial pass into task rows; FP32 blocks do
    // not (measured on the 60k-DOF plate: the split saves 2% in FP64 and
    // costs 6% in mixed precision, whose whole-task pass is cheaper)
    constexpr bool split = sizeof(T) == 8;
    const int nt = blockDim.x, full = (!split || count <= nt) ? count : count - count % nt;
    // whole tasks while every thread has one
    for (int t = threadIdx.x; t < full; t += nt) {
        const KT* kb = t < ksplit ? kt + t : kt2 + t;
        const size_t ks = t < ksplit ? stride : stride2;
        T a0 = T(0), a1 = T(0), a2 = T(0);
#pragma unroll
        for (int j = 0; j < NPE; j++) {
            const int b = 3 * (int)tn[j * ts + t];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const T v = u[b + d];
                const int c = 3 * j + d;
                a0 += (T)kb[(size_t)(0 * ND + c) * ks] * v;
                a1 += (T)kb[(size_t)(1 * ND + c) * ks] * v;
                a2 += (T)kb[(size_t)(2 * ND + c) * ks] * v;
            }
        }
        yt[t] = a0;
        yt[ys + t] = a1;
        yt[2 * ys + t] = a2;
    }
    // the remaining rem < nt tasks one row per thread (3 rem rows), so the
    // last pass costs about a third of a task instead of a whole one (FP64)
    const int rem = count - full;
    for (int q = threadIdx.x; q < 3 * rem; q += nt) {
        const int t = full + q % rem, r = q / rem;
        const KT* kb = t < ksplit ? kt + t : kt2 + t;
        const size_t ks = t < ksplit ? stride : stride2;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < NPE; j++) {
            const int b = 3 * (int)tn[j * ts + t];
#pragma unroll
            for (int d = 0; d < 3; d++) acc += (T)kb[(size_t)(r * ND + 3 * j + d) * ks] * u[b + d];
        }
        yt[r * ys + t] = acc;
    }
}

// Bending moments at each element's centroid (postprocess.ts:59-264):
// curvatures from the rotations (Q4: shape derivatives at xi = eta = 0
// through the Jacobian; DKT: linear-triangle derivatives), M = D (k_x +
// nu k_y, k_y + nu k_x, (1 - nu) k_xy / 2) with the plate's uniform D.
// em[e] = {Mx, My, Mxy, weight}; weight 0 marks a degenerate triangle
// (|2A| < 1e-15), which the reference leaves out of the nodal averages.
template <int NPE>
__global__ void elem_moments_kernel(int Ne, const float* __restrict__ nodes,
                                    const uint32_t* __restrict__ el, double D, double nu,
                                    const double* __restrict__ x, double4* __restrict__ em) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const uint32_t* en = el + (size_t)e * NPE;
    double dNdx[NPE], dNdy[NPE];
    if constexpr (NPE == 4) {
        const double dXi[4] = {-0.25, 0.25, 0.25, -0.25}, dEta[4] = {-0.25, -0.25, 0.25, 0.25};
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const double xi = nodes[2 * en[i]], yi = nodes[2 * en[i] + 1];
            J11 += dXi[i] * xi;
            J12 += dXi[i] * yi;
            J21 += dEta[i] * xi;
            J22 += dEta[i] * yi;
        }
        const double inv = 1.0 / (J11 * J22 - J12 * J21);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            dNdx[i] = inv * (J22 * dXi[i] - J12 * dEta[i]);
            dNdy[i] = inv * (-J21 * dXi[i] + J11 * dEta[i]);
        }
    } else {
        const double x1 = nodes[2 * en[0]], y1 = nodes[2 * en[0] + 1];
        const double x2 = nodes[2 * en[1]], y2 = nodes[2 * en[1] + 1];
        const double x3 = nodes[2 * en[2]], y3 = nodes[2 * en[2] + 1];
        const double twoA = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
        if (fabs(twoA) < 1e-15) {
            em[e] = make_double4(0.0, 0.0, 0.0, 0.0);
            return;
        }
        const double inv = 1.0 / twoA;
        dNdx[0] = (y2 - y3) * inv; dNdy[0] = (x3 - x2) * inv;
        dNdx[1] = (y3 - y1) * inv; dNdy[1] = (x1 - x3) * inv;
        dNdx[2] = (y1 - y2) * inv; dNdy[2] = (x2 - x1) * inv;
    }
    double kx = 0, ky = 0, kxy = 0;
#pragma unroll
    for (int i = 0; i < NPE; i++) {
        const double tx = x[3 * (size_t)en[i] + 1], ty = x[3 * (size_t)en[i] + 2];
        kx += dNdx[i] * ty;
        ky += -dNdy[i] * tx;
        kxy += dNdy[i] * ty - dNdx[i] * tx;
    }
    em[e] = make_double4(D * (kx + nu * ky), D * (ky + nu * kx), D * (1 - nu) * kxy / 2, 1.0);
}

// Nodal averages of the element moments, summed in element order over each
// node's incidence list (postprocess.ts:132-155).  M: [3][Nn] Mx, My, Mxy.
__global__ void node_moments_kernel(int Nn, const int* __restrict__ inc_ptr,
                                    const int* __restrict__ inc_idx, const double4* __restrict__ em,
                                    double* __restrict__ M) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    double sx = 0, sy = 0, sxy = 0, c = 0;
    for (int q = inc_ptr[n]; q < inc_ptr[n + 1]; q++) {
        const double4 m = em[inc_idx[q] / 4];
        if (m.w == 0.0) continue;
        sx += m.x;
        sy += m.y;
        sxy += m.z;
        c += 1.0;
    }
    M[n] = c > 0 ? sx / c : 0.0;
    M[Nn + n] = c > 0 ? sy / c : 0.0;
    M[2 * (size_t)Nn + n] = c > 0 ? sxy / c : 0.0;
}

// Task blocks of every task from the element matrices (setup, per solve):
// the owned node's 3 rows, columns rotated to start at the owned node.
template <int NPE>
__global__ void task_ke_kernel(int NT, const int* __restrict__ task_elem,
                               const uint8_t* __restrict__ task_pos,
                               const double* __restrict__ ke64, double* __restrict__ kt64,
                               float* __restrict__ kt32) {
    constexpr int ND = 3 * NPE, KK = ND * ND;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NT) return;
    const int e = task_elem[t], k = task_pos[t];
    const double* K = ke64 + (size_t)e * KK;
    for (int r = 0; r < 3; r++)
        for (int j = 0; j < NPE; j++)
            for (int d = 0; d < 3; d++) {
                const double v = K[(3 * k + r) * ND + 3 * ((k + j) % NPE) + d];
                const size_t o = (size_t)(r * ND + 3 * j + d) * NT + t;
                kt64[o] = v;
                if (kt32) kt32[o] = (float)v;
            }
}

// ---------------------------------------------------------------------------
// persistent PCG
// ---------------------------------------------------------------------------

enum { STOP_CONVERGED = 0, STOP_MAX_ITER = 1, STOP_BREAKDOWN = 2, STOP_ZERO_RHS = 3, STOP_STAGNATED = 4 };
enum { ACT_UPDATE = 0, ACT_STOP = 1, ACT_RU = 2, ACT_NONFINITE = 3 };
enum { ST_OK = 0, ST_TIMEOUT = 4, ST_NONFINITE = 5 };

// Threads per block: at most kMaxThreads (the launch bound of the 96-register
// build); up to kLeanThreads a build with 128 registers per thread runs
// instead (no spills); the batch and load-case kernels always run
// kBatchThreads / kMultiThreads.
constexpr int kMaxThreads = 576;
constexpr int kLeanThreads = 512;
constexpr int kBatchThreads = 512;
constexpr int kMultiThreads = 512;  // the load-case kernel (128 registers)

// Per-phase SM cycles of thread 0 of block 0, when timing is requested:
// 0 K.u, 1 gather + dots + publish w, 2 block reduction and publishing the
// partials, 3 the Chebyshev smoother's K t, 4 exchange wait, 5 the barrier
// after the decision, 6 thread 0's decision, 7 vector updates (and the
// residual replacement rounds of the mixed mode).
struct PhaseClock {
    bool on;
    long long last;
    long long* t;  // 8 accumulators in shared memory
    __device__ __forceinline__ void start(bool enable, long long* acc) {
        on = enable;
        t = acc;
        if (on)
            for (int k = 0; k < 8; k++) t[k] = 0;
        last = on ? clock64() : 0;
    }
    __device__ __forceinline__ void lap(int k) {
        if (!on) return;
        const long long now = clock64();
        t[k] += now - last;
        last = now;
    }
};

// Owned-node gather of task results: w_n = sum of the node's task rows.
template <typename T>
__device__ __forceinline__ void gather3(const T* __restrict__ yt, int ntask, int ta, int tb,
                                        T& w0, T& w1, T& w2) {
    w0 = T(0);
    w1 = T(0);
    w2 = T(0);
    for (int t = ta; t < tb; t++) {
        w0 += yt[t];
        w1 += yt[ntask + t];
        w2 += yt[2 * ntask + t];
    }
}

__device__ __forceinline__ void block_jacobi3(const float* Bn, const float* rv, float* u) {
    u[0] = Bn[0] * rv[0] + Bn[1] * rv[1] + Bn[2] * rv[2];
    u[1] = Bn[3] * rv[0] + Bn[4] * rv[1] + Bn[5] * rv[2];
    u[2] = Bn[6] * rv[0] + Bn[7] * rv[1] + Bn[8] * rv[2];
}
__device__ __forceinline__ void block_jacobi3(const double* Bn, const double* rv, double* u) {
    u[0] = Bn[0] * rv[0] + Bn[1] * rv[1] + Bn[2] * rv[2];
    u[1] = Bn[3] * rv[0] + Bn[4] * rv[1] + Bn[5] * rv[2];
    u[2] = Bn[6] * rv[0] + Bn[7] * rv[1] + Bn[8] * rv[2];
}

// Polynomial smoother at one node: with t = D^-1 r in un and the node's
// task results K t in yt[ta, tb), un = ca t - cb D_n^-1 (K t); constrained
// rows of K are the identity.
template <typename T>
__device__ __forceinline__ void smooth_node(T* un, const T* __restrict__ yt, int ys, int ta, int tb,
                                            const T* Bn, const unsigned char* cn, T ca, T cb) {
    T k3[3];
    gather3(yt, ys, ta, tb, k3[0], k3[1], k3[2]);
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (cn[d]) k3[d] = un[d];
    T v[3];
    block_jacobi3(Bn, k3, v);
#pragma unroll
    for (int d = 0; d < 3; d++) un[d] = ca * un[d] - cb * v[d];
}

// Restriction of a nodal 3-vector to the node's aggregate modes (P^T v):
// mode 0 w = 1; mode 1 w = dy, thx = 1/h; mode 2 w = dx, thy = -1/h,
// constrained DOFs excluded.
template <typename V, typename T>
__device__ __forceinline__ void restrict3(const V* v, const unsigned char* c, const T* bas,
                                          double* acc) {
    const double w = c[0] ? 0.0 : (double)v[0], tx = c[1] ? 0.0 : (double)v[1];
    const double ty = c[2] ? 0.0 : (double)v[2];
    acc[0] += w;
    acc[1] += (double)bas[1] * w + (double)bas[2] * tx;
    acc[2] += (double)bas[0] * w - (double)bas[2] * ty;
}

// u += P c for one node (c = the 3 coarse values of its aggregate).
template <typename T>
__device__ __forceinline__ void prolong3(const double* cvn, const unsigned char* c, const T* bas,
                                         T* u) {
    if (!c[0]) u[0] += (T)(cvn[0] + (double)bas[1] * cvn[1] + (double)bas[0] * cvn[2]);
    if (!c[1]) u[1] += (T)((double)bas[2] * cvn[1]);
    if (!c[2]) u[2] -= (T)((double)bas[2] * cvn[2]);
}

// out[q] = sum_j Ai[q][j] y_j for the part's coarse rows q < rows, where
// y_{3b+m} = (T) sp[b * stride + off + m] is the restriction of block b's
// aggregate staged by the exchange (no contiguous copy needed).  Warps
// w0.. take two rows each (16 lanes per row, lane l reading the 3 columns
// of blocks l, l + 16, ...), then a 16-lane shuffle reduction: fixed order,
// so every block computes the same bits for the same row.
template <typename T>
__device__ __forceinline__ void coarse_apply(const T* __restrict__ Ai, int G, int rows,
                                             const double* __restrict__ sp, int stride, int off,
                                             double* __restrict__ out, int w0) {
    const int lane = threadIdx.x & 31, warp = (int)(threadIdx.x >> 5) - w0;
    const int nw = (int)(blockDim.x >> 5) - w0;
    if (warp < 0) return;
    const int half = lane >> 4, hl = lane & 15, C = 3 * G;
    for (int q0 = 2 * warp; q0 < rows; q0 += 2 * nw) {
        const int q = q0 + half;
        T acc0 = T(0), acc1 = T(0), acc2 = T(0);
        if (q < rows) {
            const T* row = Ai + (size_t)q * C;
            for (int b = hl; b < G; b += 16) {
                const double* y = sp + b * stride + off;
                acc0 += row[3 * b] * (T)y[0];
                acc1 += row[3 * b + 1] * (T)y[1];
                acc2 += row[3 * b + 2] * (T)y[2];
            }
        }
        double acc = (double)acc0 + (double)acc1 + (double)acc2;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (hl == 0 && q < rows) out[q] = acc;
    }
}

// The whole PCG solve.  T = double: plain FP64.  T = float (MIXED): inner
// iterations in FP32 with FP64 dot products, FP64 solution x, and FP64
// true-residual replacement r = F - K x ("reliable update") whenever the
// recursive residual has fallen by reliable_delta, after reliable_interval
// updates, or when it meets the tolerance (convergence is then decided on
// the true residual).
//
// Exchange rounds: round e (e = 1, 2, ...) carries every block's partial
// sums and the owners' values of one vector (w, or the replaced r), in
// buffers [e & 1]; x rounds (for the FP64 residual) use their own tags.
// A block overwrites buffer [e & 1] only after it has seen every block's
// round e - 1 partials, and every block reads round e - 2 before it
// publishes round e - 1, so no reader can still need the old values.
template <int NPE, typename T, bool MIXED, int XS = (MIXED ? 3 : 2)>
__device__ __forceinline__ void pcg_body(const PcgArgs& a, const int g, unsigned char* sm) {
    constexpr int ND = 3 * NPE, TW = Tag<T>::W;
    const SmemLayout& L = a.L;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n0 = a.node_off[g], nloc = a.node_off[g + 1] - n0, no = a.nown[g];
    // tasks [0, nta) of the part; the owned nodes' are [0, ntm) (all of them
    // unless the plan has a 2-ring halo: then ring-1 nodes' tasks follow)
    const int t0 = a.task_off[g], nta = a.task_off[g + 1] - t0;
    const int nn1 = a.n1[g], ntm = a.tptr[a.tp_off[g] + no];
    const bool cheb = a.smoother == 1;
    const T ca = (T)a.cheb_a, cbc = (T)a.cheb_b;
    const size_t N3 = 3 * (size_t)a.Nn;

    T* r = (T*)(sm + L.r);
    T* u = (T*)(sm + L.u);
    T* p = (T*)(sm + L.p);
    T* s = (T*)(sm + L.s);
    T* w = (T*)(sm + L.w);
    T* B = (T*)(sm + L.B);
    T* yt = (T*)(sm + L.yt);
    T* kts = (T*)(sm + L.kt);
    double* x = (double*)(sm + L.x);
    double* red = (double*)(sm + L.red);
    double* scal = (double*)(sm + L.scal);
    double* sp = (double*)(sm + L.sp);
    int* gid = (int*)(sm + L.gid);
    int* tptr = (int*)(sm + L.tptr);
    uint16_t* tn = (uint16_t*)(sm + L.tnode);
    unsigned char* cm = (unsigned char*)(sm + L.cm);
    // coarse state per row of this part: c = A_c^-1 P^T r and cs = A_c^-1 P^T s
    // in two copies (copy cb is current; an update writes copy cb ^ 1, so
    // nodes can read the current copy while the new one is written), and
    // qw = A_c^-1 P^T w of the current round
    double* qw = (double*)(sm + L.qw);
    double* csb = (double*)(sm + L.cs);
    double* cvb = (double*)(sm + L.cv);
    int* ctl = (int*)(sm + L.ctl);  // [0] action, [1] final residual needed
    T* nb = (T*)(sm + L.nb);
    int* nslot = (int*)(sm + L.nslot);
    const int rows = a.coarse ? 3 * (a.cagg_off[g + 1] - a.cagg_off[g]) : 0;
    const T* aig = a.coarse ? (MIXED ? (const T*)a.ainv32 : (const T*)a.ainv64) + (size_t)a.ainv_off[g] * a.C
                            : nullptr;
    T* ais = (T*)(sm + L.ainv);
    const T* Ai = a.ainv_smem ? (const T*)ais : aig;
    const int KP = a.coarse ? 6 : 3;  // partial sums per block in a main round
    // FP64 views for the true residual: own arrays in MIXED mode (ytd may
    // share the dead yt / w / u space),
    // the (then dead) p / yt arrays in FP64 mode
    double* xl = MIXED ? (double*)(sm + L.xl) : (double*)p;
    double* ytd = MIXED ? (double*)(sm + L.ytd) : (double*)yt;
    const T* ktg = MIXED ? (const T*)a.kt32 : (const T*)a.kt64;
    const T* Bg = MIXED ? (const T*)a.binv32 : (const T*)a.binv64;

    // ---- load the part ----
    for (int i = tid; i < nloc; i += nt) gid[i] = a.nodes[n0 + i];
    for (int i = tid; i <= nn1; i += nt) tptr[i] = a.tptr[a.tp_off[g] + i];
    for (int i = tid; i < NPE * nta; i += nt) {
        const int t = i % nta, j = i / nta;
        tn[i] = a.task_nodes[(size_t)(t0 + t) * NPE + j];
    }
    // Ke blocks staged in shared memory: none, the owned tasks' (ke_smem 1)
    // or every task's (2)
    const int nk = a.ke_smem == 2 ? nta : ntm;
    if (a.ke_smem)
        for (int i = tid; i < 3 * ND * nk; i += nt) {
            const int t = i % nk, q = i / nk;
            kts[i] = ktg[(size_t)q * a.NT + t0 + t];
        }
    if (a.coarse) {
        for (int i = tid; i < nloc; i += nt) {
            nslot[i] = a.node_slot[n0 + i];
#pragma unroll
            for (int q = 0; q < 3; q++) nb[3 * i + q] = (T)a.node_basis[3 * (size_t)(n0 + i) + q];
        }
        for (int j = tid; j < rows; j += nt) csb[j] = 0.0;
        if (a.ainv_smem)
            for (int i = tid; i < rows * a.C; i += nt) ais[i] = aig[i];
    }
    __syncthreads();
    for (int n = tid; n < nloc; n += nt) {
        const int G3 = 3 * gid[n];
        T rv[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const unsigned char c = a.cons[G3 + d];
            cm[3 * n + d] = c;
            rv[d] = c ? T(0) : (T)a.F[G3 + d];
            r[3 * n + d] = rv[d];
            p[3 * n + d] = T(0);
            s[3 * n + d] = T(0);
            if (n < no) x[3 * n + d] = 0.0;
        }
        T* Bn = B + 9 * n;
#pragma unroll
        for (int q = 0; q < 9; q++) Bn[q] = Bg[(size_t)gid[n] * 9 + q];
        block_jacobi3(Bn, rv, u + 3 * n);
    }
    __syncthreads();

    const T* kt = a.ke_smem ? kts : ktg + t0;
    const size_t kstride = a.ke_smem ? (size_t)nk : (size_t)a.NT;
    // the smoother's K t also runs ring-1 tasks, whose blocks may stay in global memory
    const int ksplit = a.ke_smem == 1 ? ntm : (1 << 30);
    if (cheb) {
        // u0 = a t - b D^-1 K t, t = D^-1 r0 (u holds t on every local node)
        task_matvec<NPE, T, T>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0, (size_t)a.NT);
        __syncthreads();
        for (int n = tid; n < nn1; n += nt)
            smooth_node(u + 3 * n, yt, nta, tptr[n], tptr[n + 1], B + 9 * n, cm + 3 * n, ca, cbc);
        __syncthreads();
    }
    PhaseClock clk;
    clk.start(a.timing && g == 0 && tid == 0, (long long*)(sm + L.clk));
    Waiter wt;
    wt.start(a.timeout_ns, a.abort_flag, &a.res->wait_failures);
    unsigned e = a.tag0 + 1, xe = a.tag0 + 1;  // round tags
    int status = ST_OK;

    // ---- two-level: u0 = M_bj r0 + P A_c^-1 P^T r0 (one exchange round) ----
    if (a.coarse) {
        double v0[4] = {0.0, 0.0, 0.0, 0.0};
        for (int n = tid; n < no; n += nt) restrict3(r + 3 * n, cm + 3 * n, nb + 3 * n, v0);
        unsigned long long* pb0 = a.llp + (size_t)(e & 1) * kRep * a.G * 16;
        block_publish<4>(v0, red, pb0, a.G, g, 3, e);
        const bool ok = exchange_round<T, XS>(pb0, a.G, 3, nullptr, w, no, no, gid, g, e, sp, wt);
        if (__syncthreads_or(!ok)) {
            status = ST_TIMEOUT;
        } else {
            coarse_apply<T>(Ai, a.G, rows, sp, 3, 0, cvb, 0);
            __syncthreads();
            for (int n = tid; n < nloc; n += nt) prolong3(cvb + 3 * nslot[n], cm + 3 * n, nb + 3 * n, u + 3 * n);
            __syncthreads();
        }
        e++;
    }

    // decision state (thread 0): reciprocals of the previous gamma and
    // alpha, and squared thresholds, so the step to the barrier has one
    // division and no square root
    double inv_gamma = 1.0, inv_alpha = 1.0, bnorm = 0.0, rn_ref = 0.0;
    const double thr_abs = a.tol * a.tol;
    double thr_rel = 0.0, thr_ru = 0.0;
    int cb = 0;  // current copy of the coarse state
    double best_trn = INFINITY;  // mixed: smallest FP64 residual seen at a replacement
    int stall = 0;               // replacements since it last halved
    int it = 0, stop = -1, xupd = 0, xupd_ref = 0, nru = 0;
    double final_res = 0.0, true_rel = -1.0;
    bool first = true;

    for (; status == ST_OK; it++) {
        const bool tr = it == a.trace_it && tid == 0;
        if (tr) a.trace[4 * g] = gtimer();
        // ---- w = A u on owned rows ----
        task_matvec<NPE, T, T>(u, yt, nta, ntm, tn, nta, kt, kstride);
        __syncthreads();
        clk.lap(0);
        // ---- gather, BC rows, dot products, publish w ----
        double v[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        unsigned long long* vb = a.llv + (size_t)(e & 1) * N3 * 2;
        unsigned long long* pb = a.llp + (size_t)(e & 1) * kRep * a.G * 16;
        for (int k = tid; k < 3 * no; k += nt) {
            const int n = k / 3, d = k - 3 * n;
            const int tb = tptr[n + 1];
            T wk = T(0);
            for (int t = tptr[n]; t < tb; t++) wk += yt[d * nta + t];
            const bool c = cm[k] != 0;
            const T uk = u[k], rk = r[k];
            if (c) wk = uk;
            w[k] = wk;
            v[0] += (double)rk * (double)uk;
            v[1] += (double)wk * (double)uk;
            v[2] += (double)rk * (double)rk;
            Tag<T>::put(vb + (size_t)(3 * gid[n] + d) * TW, wk, e);
            if (a.coarse && !c) {
                const T* bs = nb + 3 * n;  // dx, dy, 1/h
                const double wd = (double)wk;
                if (d == 0) {
                    v[3] += wd;
                    v[4] += (double)bs[1] * wd;
                    v[5] += (double)bs[0] * wd;
                } else if (d == 1) {
                    v[4] += (double)bs[2] * wd;
                } else {
                    v[5] -= (double)bs[2] * wd;
                }
            }
        }
        clk.lap(1);
        if (a.coarse) {
            block_publish<8>(v, red, pb, a.G, g, 6, e);
        } else {
            double v4[4] = {v[0], v[1], v[2], 0.0};
            block_publish<4>(v4, red, pb, a.G, g, 3, e);
        }
        if (tr) a.trace[4 * g + 1] = gtimer();
        clk.lap(2);
        // ---- exchange: every block's partials and this block's ghost w ----
        {
            bool ok = exchange_round<T, XS>(pb, a.G, KP, vb, w, no, nloc, gid, g, e, sp, wt);
            if (a.test_stall && it == 0 && tid == 0) {
                double never;  // a tag no block writes: the wait must run out
                ok = ok && poll<double>(a.llp + (size_t)kRep * a.G * 32, 0xffffffffu, never, wt);
            }
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            sum_partials<3>(sp, a.G, KP, scal);
        }
        e++;
        clk.lap(4);
        // ---- decisions: thread 0 decides (warp 0 just summed the partials),
        //      the block follows after one barrier ----
        __syncwarp();
        if (tid == 0) {
            const double gamma = scal[0], delta = scal[1], rho = scal[2];
            int act = ACT_UPDATE;
            if (!isfinite(gamma) || !isfinite(delta) || !isfinite(rho)) {
                if (g == 0) {
                    a.res->nonfinite_it = it;
                    a.res->nonfinite_vals[0] = gamma;
                    a.res->nonfinite_vals[1] = delta;
                    a.res->nonfinite_vals[2] = rho;
                }
                act = ACT_NONFINITE;
            } else if (first && rho < 1e-60) {
                bnorm = sqrt(rho);
                stop = STOP_ZERO_RHS; final_res = 0.0; true_rel = 0.0; act = ACT_STOP;
            } else {
                // ||r|| < tol  <=>  rho < tol^2, and so on for the other tests
                if (first) {
                    bnorm = sqrt(rho);
                    rn_ref = bnorm;
                    thr_rel = a.tol * bnorm * (a.tol * bnorm);
                    thr_ru = a.reliable_delta * rn_ref * (a.reliable_delta * rn_ref);
                } else {
                    const bool conv = (a.stop_rule == 0 && rho < thr_abs) || rho < thr_rel;
                    if (MIXED && (conv || rho <= thr_ru || xupd - xupd_ref >= a.reliable_interval))
                        act = ACT_RU;
                    else if (!MIXED && conv) {
                        stop = STOP_CONVERGED; final_res = sqrt(rho); act = ACT_STOP;
                    }
                }
                if (act == ACT_UPDATE && xupd >= a.maxit) {
                    stop = STOP_MAX_ITER; final_res = sqrt(rho); act = ACT_STOP;
                }
                if (act == ACT_UPDATE) {
                    const double beta = first ? 0.0 : gamma * inv_gamma;
                    const double pap = first ? delta : delta - beta * gamma * inv_alpha;
                    if (fabs(pap) < 1e-30) {
                        stop = STOP_BREAKDOWN; xupd++; final_res = sqrt(rho); act = ACT_STOP;
                    } else {
                        // two independent reciprocals; only alpha gates the barrier
                        const double alpha = gamma * recip(pap);
                        inv_gamma = recip(gamma);
                        inv_alpha = pap * inv_gamma;
                        first = false;
                        xupd++;
                        scal[3] = alpha;
                        scal[4] = beta;
                    }
                }
            }
            ctl[0] = act;
            ctl[1] = (act == ACT_STOP && true_rel < 0.0) ? 1 : 0;
            clk.lap(6);
        }
        // meanwhile warps 1.. apply A_c^-1 to this round's P^T w
        if (a.coarse) coarse_apply<T>(Ai, a.G, rows, sp, 6, 3, qw, 1);
        __syncthreads();
        const int act = ctl[0];
        if (tr) a.trace[4 * g + 2] = gtimer();
        if (act == ACT_NONFINITE) { status = ST_NONFINITE; break; }
        if (act == ACT_STOP) break;
        clk.lap(5);

        if (MIXED && act == ACT_RU) {
            // ---- reliable update: r = F - K x in FP64 ----
            for (int n = tid; n < no; n += nt)
#pragma unroll
                for (int d = 0; d < 3; d++)
                    Tag<double>::put(a.llx + (size_t)(3 * gid[n] + d) * 2, x[3 * n + d], xe);
            bool ok = true;
            for (int k = tid; k < 3 * nloc && ok; k += nt) {
                if (k < 3 * no) { xl[k] = x[k]; continue; }
                double xv;
                ok = poll<double>(a.llx + (size_t)(3 * gid[k / 3] + k % 3) * 2, xe, xv, wt);
                xl[k] = xv;
            }
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            xe++;
            task_matvec<NPE, double, double>(xl, ytd, ntm, ntm, tn, nta, a.kt64 + t0, (size_t)a.NT);
            __syncthreads();
            double vt[4] = {0.0, 0.0, 0.0, 0.0};
            const int KR = a.coarse ? 4 : 1;
            unsigned long long* rb = a.llv + (size_t)(e & 1) * N3 * 2;
            unsigned long long* qb = a.llp + (size_t)(e & 1) * kRep * a.G * 16;
            for (int n = tid; n < no; n += nt) {
                double kx[3], rtv[3];
                gather3(ytd, ntm, tptr[n], tptr[n + 1], kx[0], kx[1], kx[2]);
                const int G3 = 3 * gid[n];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int k = 3 * n + d;
                    const double rt = cm[k] ? -xl[k] : (double)a.F[G3 + d] - kx[d];
                    vt[0] += rt * rt;
                    rtv[d] = rt;
                    r[k] = (T)rt;
                    Tag<T>::put(rb + (size_t)(G3 + d) * TW, (T)rt, e);
                }
                if (a.coarse) restrict3(rtv, cm + 3 * n, nb + 3 * n, vt + 1);
            }
            block_publish<4>(vt, red, qb, a.G, g, KR, e);
            ok = exchange_round<T, XS>(qb, a.G, KR, rb, r, no, nloc, gid, g, e, sp, wt);
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            sum_partials<1>(sp, a.G, KR, scal);
            // c = A_c^-1 P^T r from the true residual (cs is unchanged)
            if (a.coarse) coarse_apply<T>(Ai, a.G, rows, sp, 4, 1, cvb + cb * rows, 0);
            __syncthreads();
            e++;
            for (int n = tid; n < nloc; n += nt) {
                block_jacobi3(B + 9 * n, r + 3 * n, u + 3 * n);
                if (a.coarse && !cheb)
                    prolong3(cvb + cb * rows + 3 * nslot[n], cm + 3 * n, nb + 3 * n, u + 3 * n);
            }
            if (cheb) {
                __syncthreads();
                task_matvec<NPE, T, T>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0, (size_t)a.NT);
                __syncthreads();
                for (int n = tid; n < nn1; n += nt) {
                    smooth_node(u + 3 * n, yt, nta, tptr[n], tptr[n + 1], B + 9 * n, cm + 3 * n, ca, cbc);
                    if (a.coarse)
                        prolong3(cvb + cb * rows + 3 * nslot[n], cm + 3 * n, nb + 3 * n, u + 3 * n);
                }
            }
            if (tid == 0) {
                const double trn = sqrt(scal[0]);
                int act2 = ACT_UPDATE;
                nru++;
                rn_ref = trn;
                thr_ru = a.reliable_delta * rn_ref * (a.reliable_delta * rn_ref);
                xupd_ref = xupd;
                if (!isfinite(trn)) {
                    act2 = ACT_NONFINITE;
                } else if ((a.stop_rule == 0 && trn < a.tol) || trn / bnorm < a.tol) {
                    stop = STOP_CONVERGED; final_res = trn; true_rel = trn / bnorm; act2 = ACT_STOP;
                } else if (xupd >= a.maxit) {
                    stop = STOP_MAX_ITER; final_res = trn; true_rel = trn / bnorm; act2 = ACT_STOP;
                } else if (trn < 0.5 * best_trn) {
                    best_trn = trn;
                    stall = 0;
                } else if (++stall >= 3) {
                    // three replacements in a row without halving the FP64
                    // residual: the FP32 inner iterations no longer reduce
                    // the error (condition number near 1 / FP32 epsilon)
                    stop = STOP_STAGNATED; final_res = trn; true_rel = trn / bnorm; act2 = ACT_STOP;
                }
                ctl[0] = act2;
                ctl[1] = 0;
            }
            __syncthreads();
            if (ctl[0] == ACT_NONFINITE) { status = ST_NONFINITE; break; }
            if (ctl[0] == ACT_STOP) break;
            clk.lap(7);
            // the next round runs on buffers [e & 1]; the other pair may still be read
            continue;
        }

        // ---- vector updates; two-level: with cs = A_c^-1 P^T s and
        //      c = A_c^-1 P^T r, P^T s = P^T w + beta P^T s and
        //      P^T r_new = P^T r - alpha P^T s give cs = qw + beta cs and
        //      c_new = c - alpha cs, so u = M_bj r_new + P c_new needs no
        //      coarse solve after the decision ----
        const double alpha = scal[3], beta = scal[4];
        const T bt = (T)beta, at = (T)alpha;
        if (cheb) {
            // s, r on every local node, p and x on owned nodes, t = D^-1 r
            // into u; then K t on owned and ring-1 rows and
            // u = a t - b D^-1 K t (+ P c_new, c by the recurrences below)
            const double* cso = csb + cb * rows;
            const double* cvo = cvb + cb * rows;
            if (a.coarse && tid < rows) {
                const double c1 = __fma_rn(beta, cso[tid], qw[tid]);
                csb[(cb ^ 1) * rows + tid] = c1;
                cvb[(cb ^ 1) * rows + tid] = __fma_rn(-alpha, c1, cvo[tid]);
            }
            for (int n = tid; n < nloc; n += nt) {
                T rv[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int k = 3 * n + d;
                    const T sk = w[k] + bt * s[k];
                    s[k] = sk;
                    if (n < no) {
                        const T pk = u[k] + bt * p[k];
                        p[k] = pk;
                        x[k] += alpha * (double)pk;
                    }
                    rv[d] = r[k] - at * sk;
                    r[k] = rv[d];
                }
                block_jacobi3(B + 9 * n, rv, u + 3 * n);
            }
            __syncthreads();
            clk.lap(7);
            task_matvec<NPE, T, T>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0, (size_t)a.NT);
            __syncthreads();
            clk.lap(3);
            for (int n = tid; n < nn1; n += nt) {
                smooth_node(u + 3 * n, yt, nta, tptr[n], tptr[n + 1], B + 9 * n, cm + 3 * n, ca, cbc);
                if (a.coarse) {
                    const int sl = 3 * nslot[n];
                    double c3[3];
#pragma unroll
                    for (int m = 0; m < 3; m++)
                        c3[m] = __fma_rn(-alpha, __fma_rn(beta, cso[sl + m], qw[sl + m]), cvo[sl + m]);
                    prolong3(c3, cm + 3 * n, nb + 3 * n, u + 3 * n);
                }
            }
            if (a.coarse) cb ^= 1;
            __syncthreads();
            clk.lap(7);
            if (tr) a.trace[4 * g + 3] = gtimer();
        } else if (a.coarse) {
            const double* cso = csb + cb * rows;
            const double* cvo = cvb + cb * rows;
            if (tid < rows) {
                const double c1 = __fma_rn(beta, cso[tid], qw[tid]);
                csb[(cb ^ 1) * rows + tid] = c1;
                cvb[(cb ^ 1) * rows + tid] = __fma_rn(-alpha, c1, cvo[tid]);
            }
            for (int n = tid; n < nloc; n += nt) {
                T rv[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int k = 3 * n + d;
                    const T pk = u[k] + bt * p[k];
                    const T sk = w[k] + bt * s[k];
                    p[k] = pk;
                    s[k] = sk;
                    if (n < no) x[k] += alpha * (double)pk;
                    rv[d] = r[k] - at * sk;
                    r[k] = rv[d];
                }
                block_jacobi3(B + 9 * n, rv, u + 3 * n);
                const int sl = 3 * nslot[n];
                double c3[3];
#pragma unroll
                for (int m = 0; m < 3; m++)
                    c3[m] = __fma_rn(-alpha, __fma_rn(beta, cso[sl + m], qw[sl + m]), cvo[sl + m]);
                prolong3(c3, cm + 3 * n, nb + 3 * n, u + 3 * n);
            }
            cb ^= 1;
            __syncthreads();
            clk.lap(7);
            if (tr) a.trace[4 * g + 3] = gtimer();
        } else {
            // p, s, x, r updates and u = M_bj r on owned and ghost nodes
            for (int n = tid; n < nloc; n += nt) {
                T rv[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int k = 3 * n + d;
                    const T pk = u[k] + bt * p[k];
                    const T sk = w[k] + bt * s[k];
                    p[k] = pk;
                    s[k] = sk;
                    if (n < no) x[k] += alpha * (double)pk;
                    rv[d] = r[k] - at * sk;
                    r[k] = rv[d];
                }
                block_jacobi3(B + 9 * n, rv, u + 3 * n);
            }
            __syncthreads();
            clk.lap(7);
            if (tr) a.trace[4 * g + 3] = gtimer();
        }
    }

    // ---- write x; FP64 true residual ||F - K x|| unless already known ----
    for (int n = tid; n < no; n += nt)
#pragma unroll
        for (int d = 0; d < 3; d++) a.x[3 * gid[n] + d] = x[3 * n + d];
    if (status == ST_OK && ctl[1]) {
        for (int n = tid; n < no; n += nt)
#pragma unroll
            for (int d = 0; d < 3; d++)
                Tag<double>::put(a.llx + (size_t)(3 * gid[n] + d) * 2, x[3 * n + d], xe);
        bool ok = true;
        for (int k = tid; k < 3 * nloc && ok; k += nt) {
            if (k < 3 * no) { xl[k] = x[k]; continue; }
            double xv;
            ok = poll<double>(a.llx + (size_t)(3 * gid[k / 3] + k % 3) * 2, xe, xv, wt);
            xl[k] = xv;
        }
        if (__syncthreads_or(!ok)) {
            status = ST_TIMEOUT;
        } else {
            if (MIXED || !a.ke_smem)
                task_matvec<NPE, double, double>(xl, ytd, ntm, ntm, tn, nta, a.kt64 + t0, (size_t)a.NT);
            else
                task_matvec<NPE, double, double>(xl, ytd, ntm, ntm, tn, nta, (const double*)kts, kstride);
            __syncthreads();
            double v[2] = {0.0, 0.0};
            for (int n = tid; n < no; n += nt) {
                double kx[3];
                gather3(ytd, ntm, tptr[n], tptr[n + 1], kx[0], kx[1], kx[2]);
                const int G3 = 3 * gid[n];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int k = 3 * n + d;
                    const double f = cm[k] ? 0.0 : (double)a.F[G3 + d];
                    const double rt = cm[k] ? -xl[k] : f - kx[d];
                    v[0] += rt * rt;
                    v[1] += f * f;
                }
            }
            unsigned long long* pb = a.llp + (size_t)(e & 1) * kRep * a.G * 16;
            block_publish<2>(v, red, pb, a.G, g, 2, e);
            if (g == 0) {
                ok = exchange_round<T, XS>(pb, a.G, 2, nullptr, w, no, no, gid, g, e, sp, wt);
                if (__syncthreads_or(!ok)) {
                    status = ST_TIMEOUT;
                } else {
                    sum_partials<2>(sp, a.G, 2, scal);
                    __syncthreads();
                    if (tid == 0) true_rel = scal[1] > 0 ? sqrt(scal[0] / scal[1]) : 0.0;
                }
            }
        }
    }
    if (g == 0 && tid == 0) {
        a.res->status = status;
        a.res->iterations = xupd;
        a.res->converged = (stop == STOP_CONVERGED || stop == STOP_ZERO_RHS) ? 1 : 0;
        a.res->stop_reason = stop < 0 ? STOP_MAX_ITER : stop;
        a.res->final_residual = final_res;
        a.res->true_rel_residual = true_rel < 0.0 ? 0.0 : true_rel;
        a.res->b_norm = bnorm;
        a.res->reliable_updates = nru;
        a.res->reductions = (int)(e - 1 - a.tag0);
        a.res->last_tag = e > xe ? e : xe;
        for (int k = 0; k < 8; k++) a.res->phase_cycles[k] = clk.on ? clk.t[k] : 0;
    }
}

// One plate on the whole grid: part g = block g; MAXT: the launch bound.
template <int NPE, typename T, bool MIXED, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) pcg_kernel(const __grid_constant__ PcgArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    pcg_body<NPE, T, MIXED>(a, blockIdx.x, sm);
}

// Many independent plates of one element type (NPE) in one launch.  The
// grid is cut into teams of consecutive blocks; teams of one size form a
// class with one queue of plates (largest estimated work first).  A free
// team takes its class's next plate: team block 0 claims a queue position
// with an atomic counter and logs it in the team's claim slot k (tag
// k + 1), where the team's other blocks read it.  Each plate is
// partitioned into as many parts as the team has blocks and has its own
// exchange buffers, so teams never wait on each other.  Team block 0
// stamps each plate's start and end (globaltimer).
struct BatchArgs {
    const PcgArgs* plates;          // [count], npe 3 or 4, one precision for all
    const int* block_team;          // [grid] team of each block
    const int* team_base;           // [teams] first block of each team
    const int* team_class;          // [teams] class of each team
    const int* class_off;           // [classes + 1] into class_queue
    const int* class_queue;         // plate ids, class by class
    const int* log_off;             // [teams + 1] each team's claim slots
    int* class_next;                // [classes] next queue position (zero at launch)
    unsigned long long* claims;     // claim slots (zero at launch)
    unsigned long long* times;      // [count][2] start / end of each plate
    int* abort_flag;
    int* claim_failures;            // waits for a claim that gave up
    unsigned long long timeout_ns;  // limit of one wait for a claim
};

template <int NPE, typename T, bool MIXED>
__global__ void __launch_bounds__(kBatchThreads, 1) pcg_batch_kernel(const __grid_constant__ BatchArgs b) {
    extern __shared__ __align__(16) unsigned char sm[];
    volatile int* s_plate = (volatile int*)sm;  // between plates the shared memory is free
    const int g = (int)blockIdx.x - b.team_base[b.block_team[blockIdx.x]];
    for (int k = 0;; k++) {
        if (threadIdx.x == 0) {
            // the team's class queue and claim slots, re-read each time so
            // that only g and k stay live across the plate's solve
            const int team = b.block_team[blockIdx.x], cls = b.team_class[team];
            const int q0 = b.class_off[cls], qn = b.class_off[cls + 1] - q0;
            const int lo = b.log_off[team];
            unsigned pos = (unsigned)qn;  // past the end: no plate
            if (k < b.log_off[team + 1] - lo) {
                unsigned long long* slot = b.claims + lo + k;
                if (g == 0) {
                    pos = (unsigned)atomicAdd(b.class_next + cls, 1);
                    st_relaxed(slot, ((unsigned long long)(k + 1) << 32) | pos);
                } else {
                    Waiter wt;
                    wt.start(b.timeout_ns, b.abort_flag, b.claim_failures);
                    for (;;) {
                        const unsigned long long v = ld_relaxed(slot);
                        if ((unsigned)(v >> 32) == (unsigned)(k + 1)) {
                            pos = (unsigned)v;
                            break;
                        }
                        if (!wt.keep_going()) break;
                    }
                }
            }
            *s_plate = pos < (unsigned)qn ? b.class_queue[q0 + pos] : -1;
        }
        __syncthreads();
        const int pi = *s_plate;
        __syncthreads();  // read by all before the plate's data overwrite it
        if (pi < 0) break;
        const PcgArgs& a = b.plates[pi];
        if (g == 0 && threadIdx.x == 0) b.times[2 * pi] = gtimer();
        // a plate with fewer parts than the team has blocks leaves the rest idle
        if (g < a.G) pcg_body<NPE, T, MIXED, 2>(a, g, sm);
        __syncthreads();  // shared memory is reloaded for the next plate
        if (g == 0 && threadIdx.x == 0) b.times[2 * pi + 1] = gtimer();
    }
}

}  // namespace pg
