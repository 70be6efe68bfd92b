// Load cases of one plate solved together: NR right-hand sides of the same
// operator advance in lockstep through one persistent launch.
//
// Every per-DOF vector of the single solve (r, u, p, s, w, x and the task
// results) holds NR values per DOF, case-interleaved ([dof][case]), so the
// element matvec reads each Ke coefficient once for NR vectors and the
// coarse correction applies each A_c^-1 row to NR restrictions.  One
// exchange round per iteration carries every case's partial sums and ghost
// values, so the grid-wide wait -- the dominant cost of a single 60k-DOF
// solve -- is paid once for NR cases.
//
// Each case keeps its own PCG scalars (alpha, beta, stop state, residual
// reference), decided by lane `case` of warp 0.  A case that has stopped
// continues with alpha = beta = 0, which leaves its x, r and coarse state
// unchanged.  In mixed precision a residual replacement runs when any case
// asks for one: the round computes every case's FP64 residual, but only the
// cases that asked replace r and their coarse state (the others keep their
// recurrences untouched and only use the true residual for an early
// convergence test).
//
// Threads of the case-interleaved loops handle item q = (dof or node) * NR +
// case with a block size that is a multiple of NR, so each thread works on
// one case (threadIdx.x % NR) throughout.
#pragma once

#include "kernels.cuh"

namespace pg {

// Words of one block's partial-sum slot: up to 6 sums per case, 2 tagged
// words per FP64 sum.
template <int NR>
constexpr int multi_slot_words() { return 2 * 6 * NR; }

// NR consecutive values (one per case) as one aligned access.
template <typename T, int NR>
struct alignas(sizeof(T) * NR <= 16 ? sizeof(T) * NR : 16) CaseVec {
    T v[NR];
};

// Task matvec for NR case-interleaved vectors: yt[(r * ys + t) * NR + k] =
// row r of task t's block times case k of u.  Whole tasks, one per thread.
template <int NPE, typename T, typename KT, int NR>
__device__ __forceinline__ void task_matvec_multi(const T* __restrict__ u, T* __restrict__ yt, int ys,
                                                  int count, const uint16_t* __restrict__ tn, int ts,
                                                  const KT* __restrict__ kt, size_t stride,
                                                  int ksplit = 1 << 30,
                                                  const KT* __restrict__ kt2 = nullptr,
                                                  size_t stride2 = 0) {
    constexpr int ND = 3 * NPE;
    using V = CaseVec<T, NR>;
    for (int t = threadIdx.x; t < count; t += blockDim.x) {
        const KT* kb = t < ksplit ? kt + t : kt2 + t;
        const size_t ks = t < ksplit ? stride : stride2;
        T a0[NR], a1[NR], a2[NR];
#pragma unroll
        for (int k = 0; k < NR; k++) a0[k] = a1[k] = a2[k] = T(0);
#pragma unroll
        for (int j = 0; j < NPE; j++) {
            const int b = 3 * (int)tn[j * ts + t];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int c = 3 * j + d;
                const T k0 = (T)kb[(size_t)(0 * ND + c) * ks];
                const T k1 = (T)kb[(size_t)(1 * ND + c) * ks];
                const T k2 = (T)kb[(size_t)(2 * ND + c) * ks];
                const V uv = *reinterpret_cast<const V*>(u + (size_t)(b + d) * NR);
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    a0[k] += k0 * uv.v[k];
                    a1[k] += k1 * uv.v[k];
                    a2[k] += k2 * uv.v[k];
                }
            }
        }
        V o0, o1, o2;
#pragma unroll
        for (int k = 0; k < NR; k++) {
            o0.v[k] = a0[k];
            o1.v[k] = a1[k];
            o2.v[k] = a2[k];
        }
        *reinterpret_cast<V*>(yt + ((size_t)0 * ys + t) * NR) = o0;
        *reinterpret_cast<V*>(yt + ((size_t)1 * ys + t) * NR) = o1;
        *reinterpret_cast<V*>(yt + ((size_t)2 * ys + t) * NR) = o2;
    }
}

// Block totals of KP sums per case (each thread holds the KP sums of its
// case threadIdx.x % NR), published as this block's partial sums: value
// m * NR + k of block g goes to every replica r < kRep at words
// pb[(r * G + g) * SW + 2 (m * NR + k)].  All threads call it; one barrier,
// then warp 0 alone works, so `red` must not be written again before a
// later barrier.
template <int NR, int KP>
__device__ void block_publish_multi(double (&v)[KP], double* red, unsigned long long* pb, int G, int g,
                                    unsigned f) {
    constexpr int SW = multi_slot_words<NR>(), K = KP * NR;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int m = 0; m < KP; m++)
#pragma unroll
        for (int o = 16; o >= NR; o >>= 1) v[m] += __shfl_xor_sync(0xffffffffu, v[m], o);
    if (lane < NR)
#pragma unroll
        for (int m = 0; m < KP; m++) red[warp * K + m * NR + lane] = v[m];
    __syncthreads();
    if (warp != 0 || lane >= K) return;
    double t = 0.0;
    for (int w = 0; w < nw; w++) t += red[w * K + lane];
#pragma unroll
    for (int r = 0; r < kRep; r++) Tag<double>::put(pb + ((size_t)r * G + g) * SW + 2 * lane, t, f);
}

// One exchange round for NR cases: the K = KP * NR partial sums of every
// block (staged to sp[G][K]) and case k of each ghost DOF of vector buffer
// vb (words ((dof * NR + k) * TW), written to dst[dof_local * NR + k] for
// local DOFs [3 no, 3 nloc)).  Items: the ghost values first (their owners
// publish them before their partial sums), then the partials; each thread
// takes items tid, tid + nt, ... with S in flight, refilling a slot with
// its next item as soon as the slot's item has arrived.  Returns false if a
// wait gave up.
template <typename T, int NR, int S = 4>
__device__ bool exchange_round_multi(const unsigned long long* __restrict__ pb, int G, int K,
                                     const unsigned long long* __restrict__ vb, T* dst, int no, int nloc,
                                     const int* __restrict__ gid, int g, unsigned f, double* sp,
                                     Waiter& wt) {
    constexpr int TW = Tag<T>::W, SW = multi_slot_words<NR>();
    const int ng = 3 * (nloc - no) * NR, n = ng + G * K, nt = blockDim.x;
    pb += (size_t)(g % kRep) * G * SW;
    auto addr = [&](int i) -> const unsigned long long* {
        if (i < ng) {
            const int k3 = 3 * no + i / NR;
            return vb + ((size_t)(3 * gid[k3 / 3] + k3 % 3) * NR + i % NR) * TW;
        }
        const int q = i - ng;
        return pb + (size_t)(q / K) * SW + 2 * (q % K);
    };
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
                dst[3 * no * NR + i] = (T)__longlong_as_double((long long)((hi[s] << 32) | (lo[s] & 0xffffffffull)));
            } else {
                dst[3 * no * NR + i] = (T)__uint_as_float((unsigned)lo[s]);
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

// out[q * NR + k] = sum_j Ai[q][j] y_j^(k) for the part's coarse rows, with
// y_{3b+m}^(k) = sp[b * stride + off + m * NR + k].  Warps w0.. take two
// rows each (16 lanes per row), fixed order as in the single solve.  Only
// the cases in `mask` are written.
template <typename T, int NR>
__device__ __forceinline__ void coarse_apply_multi(const T* __restrict__ Ai, int G, int rows,
                                                   const double* __restrict__ sp, int stride, int off,
                                                   double* __restrict__ out, int w0,
                                                   unsigned mask = 0xffffffffu) {
    const int lane = threadIdx.x & 31, warp = (int)(threadIdx.x >> 5) - w0;
    const int nw = (int)(blockDim.x >> 5) - w0;
    if (warp < 0) return;
    const int half = lane >> 4, hl = lane & 15, C = 3 * G;
    for (int q0 = 2 * warp; q0 < rows; q0 += 2 * nw) {
        const int q = q0 + half;
        T acc[3][NR];
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int k = 0; k < NR; k++) acc[m][k] = T(0);
        if (q < rows) {
            const T* row = Ai + (size_t)q * C;
            for (int b = hl; b < G; b += 16) {
                const double* y = sp + b * stride + off;
#pragma unroll
                for (int m = 0; m < 3; m++) {
                    const T am = row[3 * b + m];
#pragma unroll
                    for (int k = 0; k < NR; k++) acc[m][k] += am * (T)y[m * NR + k];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NR; k++) {
            double s = (double)acc[0][k] + (double)acc[1][k] + (double)acc[2][k];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (hl == 0 && q < rows && ((mask >> k) & 1u)) out[q * NR + k] = s;
        }
    }
}

// Per-case decision state (lane k of warp 0 holds case k's).
struct CaseState {
    double inv_gamma, inv_alpha, bnorm, rn_ref, thr_rel, thr_ru, best_trn, final_res, true_rel;
    int xupd, xupd_ref, nru, stall, stop, status;
    bool first, done, asked;
};

template <int NPE, typename T, bool MIXED, int NR>
__device__ __forceinline__ void pcg_multi_body(const PcgArgs& a, const int g, unsigned char* sm) {
    constexpr int ND = 3 * NPE, TW = Tag<T>::W, SW = multi_slot_words<NR>();
    const SmemLayout& L = a.L;
    const int tid = threadIdx.x, nt = blockDim.x, kc = tid % NR;
    const int lane = tid & 31;
    const int n0 = a.node_off[g], nloc = a.node_off[g + 1] - n0, no = a.nown[g];
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
    double* scal = (double*)(sm + L.scal);  // [0, 3NR) dots, [3NR, 4NR) alpha, [4NR, 5NR) beta
    double* sp = (double*)(sm + L.sp);
    int* gid = (int*)(sm + L.gid);
    int* tptr = (int*)(sm + L.tptr);
    uint16_t* tn = (uint16_t*)(sm + L.tnode);
    unsigned char* cm = (unsigned char*)(sm + L.cm);
    double* qw = (double*)(sm + L.qw);
    double* csb = (double*)(sm + L.cs);
    double* cvb = (double*)(sm + L.cv);
    int* ctl = (int*)(sm + L.ctl);  // [0] action, [1] final residuals needed, [2] cases replacing r
    T* nb = (T*)(sm + L.nb);
    int* nslot = (int*)(sm + L.nslot);
    const int rows = a.coarse ? 3 * (a.cagg_off[g + 1] - a.cagg_off[g]) : 0;
    const int RN = rows * NR;
    const T* aig = a.coarse ? (MIXED ? (const T*)a.ainv32 : (const T*)a.ainv64) + (size_t)a.ainv_off[g] * a.C
                            : nullptr;
    T* ais = (T*)(sm + L.ainv);
    const T* Ai = a.ainv_smem ? (const T*)ais : aig;
    const int KP = a.coarse ? 6 : 3;
    // FP64 views for the true residual: own arrays in MIXED mode (ytd may
    // share the yt / w / u space), the (then dead) p / yt arrays in FP64
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
        for (int j = tid; j < RN; j += nt) csb[j] = 0.0;
        if (a.ainv_smem)
            for (int i = tid; i < rows * a.C; i += nt) ais[i] = aig[i];
    }
    __syncthreads();
    for (int n = tid; n < nloc; n += nt) {
        const int G3 = 3 * gid[n];
#pragma unroll
        for (int d = 0; d < 3; d++) cm[3 * n + d] = a.cons[G3 + d];
#pragma unroll
        for (int q = 0; q < 9; q++) B[9 * n + q] = Bg[(size_t)gid[n] * 9 + q];
    }
    __syncthreads();
    for (int q = tid; q < nloc * NR; q += nt) {
        const int n = q / NR, G3 = 3 * gid[n];
        T rv[3], uv[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const int i = (3 * n + d) * NR + kc;
            rv[d] = cm[3 * n + d] ? T(0) : (T)a.F[kc * N3 + G3 + d];
            r[i] = rv[d];
            p[i] = T(0);
            s[i] = T(0);
            if (n < no) x[i] = 0.0;
        }
        block_jacobi3(B + 9 * n, rv, uv);
#pragma unroll
        for (int d = 0; d < 3; d++) u[(3 * n + d) * NR + kc] = uv[d];
    }
    __syncthreads();

    const T* kt = a.ke_smem ? kts : ktg + t0;
    const size_t kstride = a.ke_smem ? (size_t)nk : (size_t)a.NT;
    const int ksplit = a.ke_smem == 1 ? ntm : (1 << 30);
    // u = ca t - cb D^-1 (K t) at node n of case kc (t in u, K t in yt)
    auto smooth = [&](int n) {
        T k3[3] = {T(0), T(0), T(0)}, tv[3], v3[3];
        for (int t = tptr[n]; t < tptr[n + 1]; t++)
#pragma unroll
            for (int d = 0; d < 3; d++) k3[d] += yt[((size_t)d * nta + t) * NR + kc];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            tv[d] = u[(3 * n + d) * NR + kc];
            if (cm[3 * n + d]) k3[d] = tv[d];
        }
        block_jacobi3(B + 9 * n, k3, v3);
#pragma unroll
        for (int d = 0; d < 3; d++) u[(3 * n + d) * NR + kc] = ca * tv[d] - cbc * v3[d];
    };
    // u += P c at node n of case kc, c3 = its aggregate's coarse values
    auto prolong = [&](int n, const double* c3) {
        T uv[3];
#pragma unroll
        for (int d = 0; d < 3; d++) uv[d] = u[(3 * n + d) * NR + kc];
        prolong3(c3, cm + 3 * n, nb + 3 * n, uv);
#pragma unroll
        for (int d = 0; d < 3; d++) u[(3 * n + d) * NR + kc] = uv[d];
    };
    if (cheb) {
        task_matvec_multi<NPE, T, T, NR>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0, (size_t)a.NT);
        __syncthreads();
        for (int q = tid; q < nn1 * NR; q += nt) smooth(q / NR);
        __syncthreads();
    }
    PhaseClock clk;
    clk.start(a.timing && g == 0 && tid == 0, (long long*)(sm + L.clk));
    Waiter wt;
    wt.start(a.timeout_ns, a.abort_flag, &a.res->wait_failures);
    unsigned e = a.tag0 + 1, xe = a.tag0 + 1;
    int status = ST_OK;

    // ---- two-level: u0 += P A_c^-1 P^T r0 for every case ----
    if (a.coarse) {
        double v0[3] = {0.0, 0.0, 0.0};
        for (int q = tid; q < no * NR; q += nt) {
            const int n = q / NR;
            T rv[3];
#pragma unroll
            for (int d = 0; d < 3; d++) rv[d] = r[(3 * n + d) * NR + kc];
            restrict3(rv, cm + 3 * n, nb + 3 * n, v0);
        }
        unsigned long long* pb0 = a.llp + (size_t)(e & 1) * kRep * a.G * SW;
        block_publish_multi<NR, 3>(v0, red, pb0, a.G, g, e);
        const bool ok = exchange_round_multi<T, NR>(pb0, a.G, 3 * NR, nullptr, w, no, no, gid, g, e, sp, wt);
        if (__syncthreads_or(!ok)) {
            status = ST_TIMEOUT;
        } else {
            coarse_apply_multi<T, NR>(Ai, a.G, rows, sp, 3 * NR, 0, cvb, 0);
            __syncthreads();
            for (int q = tid; q < nloc * NR; q += nt) {
                const int n = q / NR, sl = 3 * nslot[n];
                const double c3[3] = {cvb[sl * NR + kc], cvb[(sl + 1) * NR + kc], cvb[(sl + 2) * NR + kc]};
                prolong(n, c3);
            }
            __syncthreads();
        }
        e++;
    }

    CaseState cs{};
    cs.inv_gamma = 1.0;
    cs.inv_alpha = 1.0;
    cs.best_trn = INFINITY;
    cs.stop = -1;
    cs.true_rel = -1.0;
    cs.first = true;
    const double thr_abs = a.tol * a.tol;
    const unsigned cmask = (1u << NR) - 1u;
    int cb = 0;

    for (int it = 0; status == ST_OK; it++) {
        // ---- w = A u on owned rows, every case ----
        task_matvec_multi<NPE, T, T, NR>(u, yt, nta, ntm, tn, nta, kt, kstride);
        __syncthreads();
        clk.lap(0);
        // ---- gather, BC rows, dot products, publish w ----
        double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        unsigned long long* vb = a.llv + (size_t)(e & 1) * N3 * NR * 2;
        unsigned long long* pb = a.llp + (size_t)(e & 1) * kRep * a.G * SW;
        for (int q = tid; q < 3 * no * NR; q += nt) {
            const int k3 = q / NR, n = k3 / 3, d = k3 - 3 * n;
            const int tb = tptr[n + 1];
            T wk = T(0);
            for (int t = tptr[n]; t < tb; t++) wk += yt[((size_t)d * nta + t) * NR + kc];
            const bool c = cm[k3] != 0;
            const T uk = u[q], rk = r[q];
            if (c) wk = uk;
            w[q] = wk;
            v[0] += (double)rk * (double)uk;
            v[1] += (double)wk * (double)uk;
            v[2] += (double)rk * (double)rk;
            Tag<T>::put(vb + ((size_t)(3 * gid[n] + d) * NR + kc) * TW, wk, e);
            if (a.coarse && !c) {
                const T* bs = nb + 3 * n;
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
            block_publish_multi<NR, 6>(v, red, pb, a.G, g, e);
        } else {
            double v3[3] = {v[0], v[1], v[2]};
            block_publish_multi<NR, 3>(v3, red, pb, a.G, g, e);
        }
        clk.lap(2);
        {
            bool ok = exchange_round_multi<T, NR>(pb, a.G, KP * NR, vb, w, no, nloc, gid, g, e, sp, wt);
            if (a.test_stall && it == 0 && tid == 0) {
                // the two spare words after the partial-sum buffers: a tag no
                // block writes, so the wait must run out
                double never;
                ok = ok && poll<double>(a.llp + (size_t)2 * kRep * a.G * multi_slot_words<4>(), 0xffffffffu,
                                        never, wt);
            }
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            sum_partials<3 * NR>(sp, a.G, KP * NR, scal);
        }
        e++;
        clk.lap(4);
        // ---- decisions: lane k of warp 0 for case k ----
        __syncwarp();
        if (tid < 32) {
            int want = ACT_UPDATE;
            const bool me = lane < NR;
            const double gamma = scal[me ? lane : 0], delta = scal[me ? NR + lane : 0];
            const double rho = scal[me ? 2 * NR + lane : 0];
            if (me && !cs.done) {
                if (!isfinite(gamma) || !isfinite(delta) || !isfinite(rho)) {
                    cs.status = ST_NONFINITE;
                    cs.done = true;
                    cs.stop = STOP_BREAKDOWN;
                    if (g == 0) {
                        a.res[lane].nonfinite_it = it;
                        a.res[lane].nonfinite_vals[0] = gamma;
                        a.res[lane].nonfinite_vals[1] = delta;
                        a.res[lane].nonfinite_vals[2] = rho;
                    }
                } else if (cs.first && rho < 1e-60) {
                    cs.bnorm = sqrt(rho);
                    cs.stop = STOP_ZERO_RHS; cs.final_res = 0.0; cs.true_rel = 0.0; cs.done = true;
                } else {
                    if (cs.first) {
                        cs.bnorm = sqrt(rho);
                        cs.rn_ref = cs.bnorm;
                        cs.thr_rel = a.tol * cs.bnorm * (a.tol * cs.bnorm);
                        cs.thr_ru = a.reliable_delta * cs.rn_ref * (a.reliable_delta * cs.rn_ref);
                    } else {
                        const bool conv = (a.stop_rule == 0 && rho < thr_abs) || rho < cs.thr_rel;
                        if (MIXED && (conv || rho <= cs.thr_ru || cs.xupd - cs.xupd_ref >= a.reliable_interval))
                            want = ACT_RU;
                        else if (!MIXED && conv) {
                            cs.stop = STOP_CONVERGED; cs.final_res = sqrt(rho); cs.done = true;
                        }
                    }
                    if (!cs.done && want == ACT_UPDATE && cs.xupd >= a.maxit) {
                        cs.stop = STOP_MAX_ITER; cs.final_res = sqrt(rho); cs.done = true;
                    }
                }
            }
            const unsigned ru = __ballot_sync(0xffffffffu, me && !cs.done && want == ACT_RU) & cmask;
            const unsigned dn = __ballot_sync(0xffffffffu, me && cs.done) & cmask;
            const int act = ru ? ACT_RU : (dn == cmask ? ACT_STOP : ACT_UPDATE);
            if (me) {
                cs.asked = (ru >> lane) & 1u;
                double alpha = 0.0, beta = 0.0;
                if (act == ACT_UPDATE && !cs.done) {
                    beta = cs.first ? 0.0 : gamma * cs.inv_gamma;
                    const double pap = cs.first ? delta : delta - beta * gamma * cs.inv_alpha;
                    if (fabs(pap) < 1e-30) {
                        cs.stop = STOP_BREAKDOWN; cs.xupd++; cs.final_res = sqrt(rho); cs.done = true;
                        beta = 0.0;
                    } else {
                        alpha = gamma * recip(pap);
                        cs.inv_gamma = recip(gamma);
                        cs.inv_alpha = pap * cs.inv_gamma;
                        cs.first = false;
                        cs.xupd++;
                    }
                }
                scal[3 * NR + lane] = alpha;
                scal[4 * NR + lane] = beta;
            }
            if (lane == 0) {
                ctl[0] = act;
                ctl[2] = (int)ru;
            }
            clk.lap(6);
        }
        if (a.coarse) coarse_apply_multi<T, NR>(Ai, a.G, rows, sp, KP * NR, 3 * NR, qw, 1);
        __syncthreads();
        const int act = ctl[0];
        if (act == ACT_STOP) break;
        clk.lap(5);

        if (MIXED && act == ACT_RU) {
            // ---- FP64 residuals F - K x of every case; the cases that asked
            //      replace r with it ----
            const bool mine = ((unsigned)ctl[2] >> kc) & 1u;
            for (int q = tid; q < 3 * no * NR; q += nt) {
                const int k3 = q / NR;
                Tag<double>::put(a.llx + ((size_t)(3 * gid[k3 / 3] + k3 % 3) * NR + kc) * 2, x[q], xe);
            }
            bool ok = true;
            for (int q = tid; q < 3 * nloc * NR && ok; q += nt) {
                if (q < 3 * no * NR) { xl[q] = x[q]; continue; }
                const int k3 = q / NR;
                double xv;
                ok = poll<double>(a.llx + ((size_t)(3 * gid[k3 / 3] + k3 % 3) * NR + kc) * 2, xe, xv, wt);
                xl[q] = xv;
            }
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            xe++;
            task_matvec_multi<NPE, double, double, NR>(xl, ytd, ntm, ntm, tn, nta, a.kt64 + t0, (size_t)a.NT);
            __syncthreads();
            double vt[4] = {0.0, 0.0, 0.0, 0.0};
            unsigned long long* rb = a.llv + (size_t)(e & 1) * N3 * NR * 2;
            unsigned long long* qb = a.llp + (size_t)(e & 1) * kRep * a.G * SW;
            for (int q = tid; q < no * NR; q += nt) {
                const int n = q / NR, G3 = 3 * gid[n];
                double kx[3] = {0.0, 0.0, 0.0}, rtv[3];
                for (int t = tptr[n]; t < tptr[n + 1]; t++)
#pragma unroll
                    for (int d = 0; d < 3; d++) kx[d] += ytd[((size_t)d * ntm + t) * NR + kc];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int i = (3 * n + d) * NR + kc;
                    const double rt = cm[3 * n + d] ? -xl[i] : (double)a.F[kc * N3 + G3 + d] - kx[d];
                    vt[0] += rt * rt;
                    rtv[d] = rt;
                    if (mine) r[i] = (T)rt;
                    Tag<T>::put(rb + ((size_t)(G3 + d) * NR + kc) * TW, r[i], e);
                }
                if (a.coarse) restrict3(rtv, cm + 3 * n, nb + 3 * n, vt + 1);
            }
            int KR = 1;
            if (a.coarse) {
                block_publish_multi<NR, 4>(vt, red, qb, a.G, g, e);
                KR = 4;
            } else {
                double v1[1] = {vt[0]};
                block_publish_multi<NR, 1>(v1, red, qb, a.G, g, e);
            }
            ok = exchange_round_multi<T, NR>(qb, a.G, KR * NR, rb, r, no, nloc, gid, g, e, sp, wt);
            if (__syncthreads_or(!ok)) { status = ST_TIMEOUT; break; }
            sum_partials<NR>(sp, a.G, KR * NR, scal);
            if (a.coarse)
                coarse_apply_multi<T, NR>(Ai, a.G, rows, sp, KR * NR, NR, cvb + cb * RN, 0, (unsigned)ctl[2]);
            __syncthreads();
            e++;
            // u from r for every case: the FP64 task results may have used u's
            // space, and for a case that kept r and c this gives u's old bits
            for (int q = tid; q < nloc * NR; q += nt) {
                const int n = q / NR;
                T rv[3], uv[3];
#pragma unroll
                for (int d = 0; d < 3; d++) rv[d] = r[(3 * n + d) * NR + kc];
                block_jacobi3(B + 9 * n, rv, uv);
#pragma unroll
                for (int d = 0; d < 3; d++) u[(3 * n + d) * NR + kc] = uv[d];
                if (a.coarse && !cheb) {
                    const double* cv = cvb + cb * RN;
                    const int sl = 3 * nslot[n];
                    const double c3[3] = {cv[sl * NR + kc], cv[(sl + 1) * NR + kc], cv[(sl + 2) * NR + kc]};
                    prolong(n, c3);
                }
            }
            if (cheb) {
                __syncthreads();
                task_matvec_multi<NPE, T, T, NR>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0,
                                                 (size_t)a.NT);
                __syncthreads();
                for (int q = tid; q < nn1 * NR; q += nt) {
                    const int n = q / NR;
                    smooth(n);
                    if (a.coarse) {
                        const double* cv = cvb + cb * RN;
                        const int sl = 3 * nslot[n];
                        const double c3[3] = {cv[sl * NR + kc], cv[(sl + 1) * NR + kc], cv[(sl + 2) * NR + kc]};
                        prolong(n, c3);
                    }
                }
            }
            __syncwarp();
            if (tid < 32) {
                const bool me = lane < NR;
                if (me && !cs.done) {
                    const double trn = sqrt(scal[lane]);
                    if (cs.asked) {
                        cs.nru++;
                        cs.rn_ref = trn;
                        cs.thr_ru = a.reliable_delta * cs.rn_ref * (a.reliable_delta * cs.rn_ref);
                        cs.xupd_ref = cs.xupd;
                    }
                    if (!isfinite(trn)) {
                        cs.status = ST_NONFINITE; cs.stop = STOP_BREAKDOWN; cs.done = true;
                    } else if ((a.stop_rule == 0 && trn < a.tol) || trn / cs.bnorm < a.tol) {
                        cs.stop = STOP_CONVERGED; cs.final_res = trn; cs.true_rel = trn / cs.bnorm; cs.done = true;
                    } else if (!cs.asked) {
                        // a replacement for another case: this one's recurrences go on
                    } else if (cs.xupd >= a.maxit) {
                        cs.stop = STOP_MAX_ITER; cs.final_res = trn; cs.true_rel = trn / cs.bnorm; cs.done = true;
                    } else if (trn < 0.5 * cs.best_trn) {
                        cs.best_trn = trn;
                        cs.stall = 0;
                    } else if (++cs.stall >= 3) {
                        // three of its own replacements without halving the FP64
                        // residual: the FP32 inner iterations stopped helping
                        cs.stop = STOP_STAGNATED; cs.final_res = trn; cs.true_rel = trn / cs.bnorm; cs.done = true;
                    }
                }
                const unsigned dn = __ballot_sync(0xffffffffu, me && cs.done) & cmask;
                if (lane == 0) ctl[0] = dn == cmask ? ACT_STOP : ACT_UPDATE;
            }
            __syncthreads();
            if (ctl[0] == ACT_STOP) break;
            clk.lap(7);
            continue;
        }

        // ---- vector updates of every case (alpha = beta = 0 for a stopped one) ----
        const double alpha = scal[3 * NR + kc], beta = scal[4 * NR + kc];
        const T bt = (T)beta, at = (T)alpha;
        const double* cso = csb + cb * RN;
        const double* cvo = cvb + cb * RN;
        if (a.coarse)
            for (int i = tid; i < RN; i += nt) {
                const double c1 = __fma_rn(beta, cso[i], qw[i]);
                csb[(cb ^ 1) * RN + i] = c1;
                cvb[(cb ^ 1) * RN + i] = __fma_rn(-alpha, c1, cvo[i]);
            }
        auto c_new = [&](int n, double* c3) {
            const int sl = 3 * nslot[n];
#pragma unroll
            for (int m = 0; m < 3; m++) {
                const int i = (sl + m) * NR + kc;
                c3[m] = __fma_rn(-alpha, __fma_rn(beta, cso[i], qw[i]), cvo[i]);
            }
        };
        for (int q = tid; q < nloc * NR; q += nt) {
            const int n = q / NR;
            T rv[3], uv[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int i = (3 * n + d) * NR + kc;
                const T sk = w[i] + bt * s[i];
                s[i] = sk;
                if (cheb) {
                    if (n < no) {
                        const T pk = u[i] + bt * p[i];
                        p[i] = pk;
                        x[i] += alpha * (double)pk;
                    }
                } else {
                    const T pk = u[i] + bt * p[i];
                    p[i] = pk;
                    if (n < no) x[i] += alpha * (double)pk;
                }
                rv[d] = r[i] - at * sk;
                r[i] = rv[d];
            }
            block_jacobi3(B + 9 * n, rv, uv);
#pragma unroll
            for (int d = 0; d < 3; d++) u[(3 * n + d) * NR + kc] = uv[d];
            if (a.coarse && !cheb) {
                double c3[3];
                c_new(n, c3);
                prolong(n, c3);
            }
        }
        __syncthreads();
        clk.lap(7);
        if (cheb) {
            task_matvec_multi<NPE, T, T, NR>(u, yt, nta, nta, tn, nta, kt, kstride, ksplit, ktg + t0, (size_t)a.NT);
            __syncthreads();
            clk.lap(3);
            for (int q = tid; q < nn1 * NR; q += nt) {
                const int n = q / NR;
                smooth(n);
                if (a.coarse) {
                    double c3[3];
                    c_new(n, c3);
                    prolong(n, c3);
                }
            }
            __syncthreads();
            clk.lap(7);
        }
        if (a.coarse) cb ^= 1;
    }

    // ---- write x of every case; FP64 true residuals unless all known ----
    for (int q = tid; q < 3 * no * NR; q += nt) {
        const int k3 = q / NR;
        a.x[kc * N3 + 3 * gid[k3 / 3] + k3 % 3] = x[q];
    }
    if (tid < 32) {
        const unsigned need = __ballot_sync(0xffffffffu, lane < NR && cs.true_rel < 0.0) & cmask;
        if (lane == 0) ctl[1] = need ? 1 : 0;
    }
    __syncthreads();
    if (status == ST_OK && ctl[1]) {
        for (int q = tid; q < 3 * no * NR; q += nt) {
            const int k3 = q / NR;
            Tag<double>::put(a.llx + ((size_t)(3 * gid[k3 / 3] + k3 % 3) * NR + kc) * 2, x[q], xe);
        }
        bool ok = true;
        for (int q = tid; q < 3 * nloc * NR && ok; q += nt) {
            if (q < 3 * no * NR) { xl[q] = x[q]; continue; }
            const int k3 = q / NR;
            double xv;
            ok = poll<double>(a.llx + ((size_t)(3 * gid[k3 / 3] + k3 % 3) * NR + kc) * 2, xe, xv, wt);
            xl[q] = xv;
        }
        if (__syncthreads_or(!ok)) {
            status = ST_TIMEOUT;
        } else {
            if (MIXED || !a.ke_smem)
                task_matvec_multi<NPE, double, double, NR>(xl, ytd, ntm, ntm, tn, nta, a.kt64 + t0, (size_t)a.NT);
            else
                task_matvec_multi<NPE, double, double, NR>(xl, ytd, ntm, ntm, tn, nta, (const double*)kts, kstride);
            __syncthreads();
            double v2[2] = {0.0, 0.0};
            for (int q = tid; q < no * NR; q += nt) {
                const int n = q / NR, G3 = 3 * gid[n];
                double kx[3] = {0.0, 0.0, 0.0};
                for (int t = tptr[n]; t < tptr[n + 1]; t++)
#pragma unroll
                    for (int d = 0; d < 3; d++) kx[d] += ytd[((size_t)d * ntm + t) * NR + kc];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    const int i = (3 * n + d) * NR + kc;
                    const double f = cm[3 * n + d] ? 0.0 : (double)a.F[kc * N3 + G3 + d];
                    const double rt = cm[3 * n + d] ? -xl[i] : f - kx[d];
                    v2[0] += rt * rt;
                    v2[1] += f * f;
                }
            }
            unsigned long long* pb = a.llp + (size_t)(e & 1) * kRep * a.G * SW;
            block_publish_multi<NR, 2>(v2, red, pb, a.G, g, e);
            if (g == 0) {
                ok = exchange_round_multi<T, NR>(pb, a.G, 2 * NR, nullptr, w, no, no, gid, g, e, sp, wt);
                if (__syncthreads_or(!ok)) {
                    status = ST_TIMEOUT;
                } else {
                    sum_partials<2 * NR>(sp, a.G, 2 * NR, scal);
                    __syncthreads();
                    if (tid < NR && cs.true_rel < 0.0)
                        cs.true_rel = scal[NR + tid] > 0 ? sqrt(scal[tid] / scal[NR + tid]) : 0.0;
                }
            }
        }
    }
    if (g == 0 && tid < NR) {
        PcgResult& R = a.res[tid];
        R.status = status != ST_OK ? status : cs.status;
        R.iterations = cs.xupd;
        R.converged = (cs.stop == STOP_CONVERGED || cs.stop == STOP_ZERO_RHS) ? 1 : 0;
        R.stop_reason = cs.stop < 0 ? STOP_MAX_ITER : cs.stop;
        R.final_residual = cs.final_res;
        R.true_rel_residual = cs.true_rel < 0.0 ? 0.0 : cs.true_rel;
        R.b_norm = cs.bnorm;
        R.reliable_updates = cs.nru;
        R.reductions = (int)(e - 1 - a.tag0);
        R.last_tag = e > xe ? e : xe;
        for (int k = 0; k < 8; k++) R.phase_cycles[k] = clk.on ? clk.t[k] : 0;
    }
}

// NR load cases of one plate on the whole grid: part g = block g.  a.F and
// a.x hold NR vectors of 3 Nn back to back, a.res NR result records, and the
// exchange buffers are sized for NR cases.
template <int NPE, typename T, bool MIXED, int NR>
__global__ void __launch_bounds__(kMultiThreads, 1) pcg_multi_kernel(const __grid_constant__ PcgArgs a) {
    extern __shared__ __align__(16) unsigned char sm[];
    pcg_multi_body<NPE, T, MIXED, NR>(a, blockIdx.x, sm);
}

}  // namespace pg
