// C ABI of the plate solver (include/plategpu.h): context, plan cache,
// uploads, kernel launches.  No exception crosses the ABI; every failure
// becomes a pg_status plus a message for pg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <list>
#include <memory>
#include <mutex>
#include <atomic>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "coarse.cuh"
#include "internal.h"
#include "kernels.cuh"
#include "multi.cuh"
#include "plan.h"
#include "plategpu.h"

namespace {

thread_local std::string g_create_error;

struct Fail {
    int status;
    std::string msg;
};

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw Fail{e_ == cudaErrorMemoryAllocation ? PG_ENOMEM : PG_ECUDA,            \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};               \
    } while (0)

// Device array.  view() points it into memory owned elsewhere (a plan's
// arena), which it then does not free.
template <typename T>
struct DevBuf {
    using value_type = T;
    T* p = nullptr;
    size_t n = 0;
    bool own = true;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) CK(cudaMalloc(&p, count * sizeof(T)));
    }
    void upload(const T* h, size_t count, cudaStream_t st) {
        alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void view(T* ptr, size_t count) {
        release();
        p = ptr;
        n = count;
        own = false;
    }
    void release() {
        if (p && own) cudaFree(p);
        p = nullptr;
        n = 0;
        own = true;
    }
    ~DevBuf() { release(); }
};

// Typed arrays carved out of one device allocation, each 256-byte aligned:
// one cudaMalloc instead of one per array (each a driver call that maps
// pages, which the first solve of a new mesh pays many times over).  add()
// records an array (with the host data to copy into it, or none);
// commit() allocates `store`, points the arrays into it and queues the
// copies on `st`.
struct Arena {
    size_t total = 0;
    std::vector<std::function<void(unsigned char*, cudaStream_t)>> bind;
    template <typename B>
    void add(B& buf, size_t count, const void* host) {
        using T = typename B::value_type;
        const size_t off = total;
        total += (count * sizeof(T) + 255) & ~size_t(255);
        B* b = &buf;
        bind.push_back([b, off, count, host](unsigned char* base, cudaStream_t st) {
            b->view(reinterpret_cast<T*>(base + off), count);
            if (host && count) CK(cudaMemcpyAsync(b->p, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
        });
    }
    void commit(DevBuf<unsigned char>& store, cudaStream_t st) {
        store.alloc(total);
        for (auto& f : bind) f(store.p, st);
    }
};

struct Plan {
    int G = 0;
    pg::HostPlan hp;
    // host copies of the problem's arrays: read by the coarse-space set-up,
    // and compared with a new problem's to find its plan in the cache
    std::vector<float> h_nodes;
    std::vector<uint32_t> h_elements;
    std::vector<uint8_t> h_cons;
    std::vector<float> h_elem_t;
    uint32_t h_color_count = 0;
    std::vector<uint32_t> h_color_off, h_by_color;  // the caller's colouring
    pg_problem prob_view{};
    double E = 0, nu = 0, t = 0;
    bool has_elem_t = false;
    DevBuf<int> node_off, nown, nodes, task_off, tp_off, tptr, task_elem, inc_ptr, inc_idx, n1;
    double lambda_max = 0;  // of D^-1 K, for the polynomial smoother (0 = not estimated)
    bool setup_done = false;  // element matrices, block inverses and task blocks queued
    // exchange buffers: tags up to tag0 may sit in them (valid when ll_ready)
    unsigned tag0 = 0;
    bool ll_ready = false;
    // last launch shape that passed the residency check
    const void* ok_fn = nullptr;
    int ok_threads = 0, ok_smem = 0;
    DevBuf<uint16_t> task_nodes;
    DevBuf<uint8_t> task_pos;
    DevBuf<float> mesh_nodes, elem_t, F;
    DevBuf<uint32_t> mesh_elements, cob_off, cob_list;
    DevBuf<uint8_t> cons;
    DevBuf<double> ke64, kt64, binv64, x;
    DevBuf<float> ke32, kt32, binv32;
    DevBuf<unsigned long long> llv, llx, llp;
    DevBuf<int> cagg_off, node_slot, ainv_off;
    DevBuf<double> node_basis, ainv64;
    DevBuf<float> ainv32;
    DevBuf<int> abort_flag;
    DevBuf<unsigned long long> trace;
    DevBuf<pg::PcgResult> res;
    // one allocation holding the arrays above that build_plan creates, one
    // for the coarse-space arrays
    DevBuf<unsigned char> arena, coarse_arena;
    // load cases solved together (NR cases per launch): their loads,
    // solutions, exchange buffers and result records
    int m_nr = 0;
    unsigned m_tag0 = 0;
    bool m_ready = false;
    const void* m_ok_fn = nullptr;
    int m_ok_smem = 0;
    DevBuf<float> mF;
    DevBuf<double> mx;
    DevBuf<unsigned long long> mllv, mllx, mllp;
    DevBuf<pg::PcgResult> mres;
    // FP64 correction after a stagnated mixed solve: the mixed x, K x and
    // the FP32 residual
    DevBuf<double> xw, kx, nrm, pw;
    DevBuf<float> rf;
    // global-memory flexible PCG of a plate too large for the persistent
    // kernel's shared memory (created on first use)
    pgi::GlobalPcg* gpcg = nullptr;
    ~Plan() {
        if (gpcg) pgi::global_pcg_destroy(gpcg);
    }
};

}  // namespace

struct pg_plan {
    pg_ctx* ctx = nullptr;
    std::unique_ptr<Plan> plan;
};

// A batch of independent plates: one plan per plate, partitioned for the
// size of the team of blocks that solves it, and the team schedule (one
// launch per phase).
struct BatchPhaseDev {
    int grid = 0, kind = 4;
    DevBuf<int> block_team, team_base, team_class, class_off, class_queue, log_off;
    DevBuf<int> class_next;               // zeroed before each launch
    DevBuf<unsigned long long> claims;    // zeroed before each launch
};
struct pg_batch {
    pg_ctx* ctx = nullptr;
    int rings = 1;
    std::vector<std::unique_ptr<Plan>> plans;
    pg::BatchSchedule sched;
    std::vector<std::unique_ptr<BatchPhaseDev>> phases;
    DevBuf<int> abort_flag, claim_failures;
    DevBuf<pg::PcgArgs> args;
    DevBuf<pg::PcgResult> res;
    DevBuf<unsigned long long> times;
    int ok_smem = 0, ok_precision = 0;
    std::vector<std::vector<float>> hF;   // each plate's current load (for the FP64 fallback)
    std::unique_ptr<pg_batch> fb;         // FP64 batch of the plates whose mixed solve stagnated
    std::vector<int> fb_ids;              // its plates
    // the phase launches captured as one CUDA graph (per precision and
    // shared-memory size); graph_failed: capture not possible, launch directly
    cudaGraphExec_t graph = nullptr;
    int graph_precision = 0, graph_smem = 0;
    unsigned long long graph_timeout_ns = 0;
    bool graph_failed = false;
    ~pg_batch() {
        if (graph) cudaGraphExecDestroy(graph);
    }
};

struct pg_ctx {
    int device = 0;
    int sms = 0;
    int max_smem = 0;
    double clock_khz = 1.0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::mutex mu;
    std::string err;
    std::list<std::unique_ptr<Plan>> plans;  // most recently used first
    std::vector<const void*> smem_opt_in;    // kernels given the full shared-memory opt-in
    float* hF = nullptr;                     // pinned staging
    double* hx = nullptr;
    size_t hcap = 0;
};

namespace {

constexpr size_t kMaxPlans = 4;

void ensure_staging(pg_ctx* c, size_t n) {
    if (n <= c->hcap) return;
    if (c->hF) cudaFreeHost(c->hF);
    if (c->hx) cudaFreeHost(c->hx);
    c->hF = nullptr;
    c->hx = nullptr;
    c->hcap = 0;
    CK(cudaMallocHost(&c->hF, n * sizeof(float)));
    CK(cudaMallocHost(&c->hx, n * sizeof(double)));
    c->hcap = n;
}

int auto_ctas(const pg_ctx* c, int Nn) {
    int G = (Nn + 127) / 128;
    return std::max(1, std::min(G, c->sms));
}

// ke_mode: Ke task blocks in shared memory for 0 = no task, 1 = the owned
// nodes' tasks, 2 = every task (ring-1 tasks too, with a 2-ring halo).
pg::SmemLayout make_layout(const pg::HostPlan& hp, bool mixed, int ke_mode, bool coarse,
                           bool ainv_smem) {
    const size_t T = mixed ? 4 : 8, nd = 3 * hp.npe;
    const size_t nloc = hp.max_nloc, nown = hp.max_nown, ntask = hp.max_ntask;
    const size_t ntask_own = hp.max_ntask_own, n1 = std::max(hp.max_n1, hp.max_nown);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const int o = (int)off;
        off = (off + bytes + 15) & ~(size_t)15;
        return o;
    };
    pg::SmemLayout L{};
    L.x = take(3 * nown * 8);
    L.xl = take(mixed ? 3 * nloc * 8 : 0);
    L.red = take(32 * 8 * 8);  // [warps][8]
    L.scal = take(8 * 8);
    L.sp = take((size_t)6 * hp.G * 8);
    L.qw = take(coarse ? (size_t)3 * hp.max_kagg * 8 : 0);
    L.cs = take(coarse ? (size_t)2 * 3 * hp.max_kagg * 8 : 0);
    L.cv = take(coarse ? (size_t)2 * 3 * hp.max_kagg * 8 : 0);
    L.ctl = take(4 * 4);
    L.clk = take(8 * 8);
    L.r = take(3 * nloc * T);
    L.p = take(3 * nloc * T);
    L.s = take(3 * nloc * T);
    L.B = take(9 * nloc * T);
    // yt, w, u back to back: the mixed-precision FP64 residual's task
    // results (ytd) reuse them when they fit, since none of the three is
    // live during a residual replacement or the final residual
    L.yt = take(3 * ntask * T);
    L.w = take(3 * nloc * T);
    L.u = take(3 * nloc * T);
    if (mixed)
        L.ytd = 3 * ntask_own * 8 <= off - (size_t)L.yt ? L.yt : take(3 * ntask_own * 8);
    L.kt = take(ke_mode == 2 ? 3 * nd * ntask * T : ke_mode == 1 ? 3 * nd * ntask_own * T : 0);
    L.nb = take(coarse ? 3 * nloc * T : 0);
    L.ainv = take(coarse && ainv_smem ? (size_t)3 * hp.max_kagg * hp.C * T : 0);
    L.nslot = take(coarse ? nloc * 4 : 0);
    L.gid = take(nloc * 4);
    L.tptr = take((n1 + 1) * 4);
    L.tnode = take(hp.npe * ntask * 2);
    L.cm = take(3 * nloc);
    L.total = (int)off;
    return L;
}

// Shared-memory layout of a launch of NR load cases: every per-DOF vector
// and the task results hold NR values per entry; the partial sums 6 per case.
pg::SmemLayout make_layout_multi(const pg::HostPlan& hp, bool mixed, int ke_mode, bool coarse,
                                 bool ainv_smem, int NR) {
    const size_t T = mixed ? 4 : 8, nd = 3 * hp.npe, R = NR;
    const size_t nloc = hp.max_nloc, nown = hp.max_nown, ntask = hp.max_ntask;
    const size_t ntask_own = hp.max_ntask_own, n1 = std::max(hp.max_n1, hp.max_nown);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const int o = (int)off;
        off = (off + bytes + 15) & ~(size_t)15;
        return o;
    };
    pg::SmemLayout L{};
    L.x = take(3 * nown * 8 * R);
    L.xl = take(mixed ? 3 * nloc * 8 * R : 0);
    L.red = take(32 * 6 * R * 8);  // [warps][6 NR]
    L.scal = take(5 * R * 8);      // dots, alpha, beta per case
    L.sp = take((size_t)6 * R * hp.G * 8);
    L.qw = take(coarse ? 3 * (size_t)hp.max_kagg * 8 * R : 0);
    L.cs = take(coarse ? 2 * 3 * (size_t)hp.max_kagg * 8 * R : 0);
    L.cv = take(coarse ? 2 * 3 * (size_t)hp.max_kagg * 8 * R : 0);
    L.ctl = take(4 * 4);
    L.clk = take(8 * 8);
    L.r = take(3 * nloc * T * R);
    L.p = take(3 * nloc * T * R);
    L.s = take(3 * nloc * T * R);
    L.B = take(9 * nloc * T);
    // yt, w, u back to back: the FP64 residual's task results (ytd) reuse
    // them when they fit (u is rebuilt from r after every replacement)
    L.yt = take(3 * ntask * T * R);
    L.w = take(3 * nloc * T * R);
    L.u = take(3 * nloc * T * R);
    if (mixed)
        L.ytd = 3 * ntask_own * 8 * R <= off - (size_t)L.yt ? L.yt : take(3 * ntask_own * 8 * R);
    L.kt = take(ke_mode == 2 ? 3 * nd * ntask * T : ke_mode == 1 ? 3 * nd * ntask_own * T : 0);
    L.nb = take(coarse ? 3 * nloc * T : 0);
    L.ainv = take(coarse && ainv_smem ? (size_t)3 * hp.max_kagg * hp.C * T : 0);
    L.nslot = take(coarse ? nloc * 4 : 0);
    L.gid = take(nloc * 4);
    L.tptr = take((n1 + 1) * 4);
    L.tnode = take(hp.npe * ntask * 2);
    L.cm = take(3 * nloc);
    L.total = (int)off;
    return L;
}

std::unique_ptr<Plan> build_plan(pg_ctx* c, const pg_problem& p, int G, int rings) {
    auto pl = std::make_unique<Plan>();
    std::string e = pg::build_structure(p, pl->hp);
    if (e.empty()) e = pg::build_partition(p, G, rings, pl->hp);
    if (!e.empty()) throw Fail{PG_EINVAL, e};
    pl->G = pl->hp.G;
    pl->h_nodes.assign(p.nodes, p.nodes + 2 * (size_t)p.node_count);
    pl->h_elements.assign(p.elements, p.elements + (size_t)p.nodes_per_element * p.element_count);
    pl->h_cons.assign(p.constrained, p.constrained + 3 * (size_t)p.node_count);
    pl->prob_view = p;
    pl->prob_view.nodes = pl->h_nodes.data();
    pl->prob_view.elements = pl->h_elements.data();
    pl->prob_view.constrained = pl->h_cons.data();
    pl->prob_view.F = nullptr;
    pl->prob_view.color_count = 0;  // a plan rebuilt from the view recolours greedily
    pl->prob_view.color_offsets = nullptr;
    pl->prob_view.elements_by_color = nullptr;
    if (p.elem_t) pl->h_elem_t.assign(p.elem_t, p.elem_t + (size_t)p.element_count);
    pl->prob_view.elem_t = p.elem_t ? pl->h_elem_t.data() : nullptr;
    pl->h_color_count = p.color_count;
    if (p.color_count) {
        pl->h_color_off.assign(p.color_offsets, p.color_offsets + p.color_count + 1);
        pl->h_by_color.assign(p.elements_by_color, p.elements_by_color + p.element_count);
    }
    pl->E = p.E;
    pl->nu = p.nu;
    pl->t = p.t;
    const pg::HostPlan& hp = pl->hp;
    cudaStream_t st = c->stream;
    const size_t Nn = p.node_count, Ne = p.element_count, npe = p.nodes_per_element;
    const size_t kk = 9 * npe * npe;
    const size_t NT = hp.task_elem.size();
    // every device array of the plan in one allocation
    Arena ar;
    auto carve = [&](auto& buf, size_t count, const void* host) { ar.add(buf, count, host); };
    carve(pl->node_off, hp.node_off.size(), hp.node_off.data());
    carve(pl->nown, hp.nown.size(), hp.nown.data());
    carve(pl->nodes, hp.nodes.size(), hp.nodes.data());
    carve(pl->task_off, hp.task_off.size(), hp.task_off.data());
    carve(pl->tp_off, hp.tp_off.size(), hp.tp_off.data());
    carve(pl->tptr, hp.tptr.size(), hp.tptr.data());
    carve(pl->n1, hp.n1.size(), hp.n1.data());
    carve(pl->task_elem, hp.task_elem.size(), hp.task_elem.data());
    carve(pl->task_pos, hp.task_pos.size(), hp.task_pos.data());
    carve(pl->task_nodes, hp.task_nodes.size(), hp.task_nodes.data());
    carve(pl->inc_ptr, hp.inc_ptr.size(), hp.inc_ptr.data());
    carve(pl->inc_idx, hp.inc_idx.size(), hp.inc_idx.data());
    carve(pl->mesh_nodes, 2 * Nn, p.nodes);
    carve(pl->mesh_elements, npe * Ne, p.elements);
    carve(pl->cob_off, hp.color_offsets.size(), hp.color_offsets.data());
    carve(pl->cob_list, hp.elements_by_color.size(), hp.elements_by_color.data());
    carve(pl->cons, 3 * Nn, p.constrained);
    pl->has_elem_t = p.elem_t != nullptr;
    if (p.elem_t) carve(pl->elem_t, Ne, p.elem_t);
    carve(pl->F, 3 * Nn, nullptr);
    carve(pl->ke64, std::max<size_t>(1, Ne * kk), nullptr);
    carve(pl->ke32, std::max<size_t>(1, Ne * kk), nullptr);
    carve(pl->kt64, std::max<size_t>(1, NT * 9 * npe), nullptr);
    carve(pl->kt32, std::max<size_t>(1, NT * 9 * npe), nullptr);
    carve(pl->binv64, 9 * Nn, nullptr);
    carve(pl->binv32, 9 * Nn, nullptr);
    carve(pl->x, 3 * Nn, nullptr);
    carve(pl->llv, 12 * Nn, nullptr);
    carve(pl->llx, 6 * Nn, nullptr);
    carve(pl->llp, 32 * (size_t)pg::kRep * pl->G + 2, nullptr);
    carve(pl->abort_flag, 1, nullptr);
    carve(pl->trace, 4 * (size_t)pl->G, nullptr);
    carve(pl->res, 1, nullptr);
    ar.commit(pl->arena, st);
    // synchronous: uploads read the host plan arrays
    CK(cudaStreamSynchronize(st));
    return pl;
}

// Whether p is the problem plan pl was made from: mesh, colouring,
// constraints and material compared in full (the load is not part of a
// plan).  Exact, and faster than hashing the arrays (memcmp stops at the
// first difference and otherwise streams at memory speed).
bool same_problem(const Plan& pl, const pg_problem& p) {
    const pg_problem& q = pl.prob_view;
    if (q.node_count != p.node_count || q.element_count != p.element_count ||
        q.nodes_per_element != p.nodes_per_element || pl.h_color_count != p.color_count || q.E != p.E ||
        q.nu != p.nu || q.t != p.t || (q.elem_t != nullptr) != (p.elem_t != nullptr))
        return false;
    auto same = [](const void* a, const void* b, size_t bytes) {
        return bytes == 0 || std::memcmp(a, b, bytes) == 0;
    };
    const size_t Nn = p.node_count, Ne = p.element_count;
    return same(pl.h_cons.data(), p.constrained, 3 * Nn) &&
           same(pl.h_nodes.data(), p.nodes, 2 * Nn * sizeof(float)) &&
           same(pl.h_elements.data(), p.elements, (size_t)p.nodes_per_element * Ne * sizeof(uint32_t)) &&
           (!p.color_count ||
            (same(pl.h_color_off.data(), p.color_offsets, (p.color_count + 1) * sizeof(uint32_t)) &&
             same(pl.h_by_color.data(), p.elements_by_color, Ne * sizeof(uint32_t)))) &&
           (!p.elem_t || same(pl.h_elem_t.data(), p.elem_t, Ne * sizeof(float)));
}

Plan* get_plan(pg_ctx* c, const pg_problem& p, int G, int rings, bool* cached) {
    for (auto it = c->plans.begin(); it != c->plans.end(); ++it) {
        if ((*it)->G == G && (*it)->hp.rings == rings && same_problem(**it, p)) {
            c->plans.splice(c->plans.begin(), c->plans, it);
            *cached = true;
            return c->plans.front().get();
        }
    }
    *cached = false;
    auto pl = build_plan(c, p, G, rings);
    c->plans.push_front(std::move(pl));
    while (c->plans.size() > kMaxPlans) c->plans.pop_back();
    return c->plans.front().get();
}

// Element matrices, block-Jacobi inverses and task blocks: pure functions
// of the plan's own copies of the mesh, material and constraints, so they
// are computed once per plan (queued on the context stream; pg_set_stream
// drains the old stream before switching).
void run_setup(pg_ctx* c, Plan* pl) {
    if (pl->setup_done) return;
    pl->setup_done = true;
    const pg::HostPlan& hp = pl->hp;
    const int Ne = hp.Ne, Nn = hp.Nn;
    const float* et = pl->has_elem_t ? pl->elem_t.p : nullptr;
    if (Ne > 0 && hp.npe == 4)
        pg::ke_kernel<4><<<(Ne + 127) / 128, 128, 0, c->stream>>>(
            Ne, pl->mesh_nodes.p, pl->mesh_elements.p, pl->E, pl->nu, pl->t, et, pl->ke64.p, pl->ke32.p);
    else if (Ne > 0)
        pg::ke_kernel<3><<<(Ne + 127) / 128, 128, 0, c->stream>>>(
            Ne, pl->mesh_nodes.p, pl->mesh_elements.p, pl->E, pl->nu, pl->t, et, pl->ke64.p, pl->ke32.p);
    CK(cudaGetLastError());
    if (Nn > 0)
        pg::binv_kernel<<<(Nn + 127) / 128, 128, 0, c->stream>>>(
            Nn, hp.npe, pl->inc_ptr.p, pl->inc_idx.p, pl->ke64.p, pl->cons.p, pl->binv64.p,
            pl->binv32.p);
    CK(cudaGetLastError());
    const int NT = (int)hp.task_elem.size();
    if (NT > 0 && hp.npe == 4)
        pg::task_ke_kernel<4><<<(NT + 127) / 128, 128, 0, c->stream>>>(
            NT, pl->task_elem.p, pl->task_pos.p, pl->ke64.p, pl->kt64.p, pl->kt32.p);
    else if (NT > 0)
        pg::task_ke_kernel<3><<<(NT + 127) / 128, 128, 0, c->stream>>>(
            NT, pl->task_elem.p, pl->task_pos.p, pl->ke64.p, pl->kt64.p, pl->kt32.p);
    CK(cudaGetLastError());
}

// y = K x on the device (colour by colour, then the identity rows of the
// constrained DOFs), queued on the context stream.  The plan's set-up must
// have run.
void queue_apply_k(pg_ctx* c, Plan* pl, const double* x, double* y) {
    const pg::HostPlan& hp = pl->hp;
    const size_t n = 3 * (size_t)hp.Nn;
    CK(cudaMemsetAsync(y, 0, n * sizeof(double), c->stream));
    for (int col = 0; col < hp.colors; col++) {
        const int off = (int)hp.color_offsets[col], cnt = (int)hp.color_offsets[col + 1] - off;
        if (cnt > 0)
            pg::applyk_color_kernel<<<(cnt + 127) / 128, 128, 0, c->stream>>>(
                cnt, pl->cob_list.p + off, hp.npe, pl->mesh_elements.p, pl->ke64.p, x, y);
        CK(cudaGetLastError());
    }
    pg::bc_copy_kernel<<<((int)n + 255) / 256, 256, 0, c->stream>>>((int)n, pl->cons.p, x, y);
    CK(cudaGetLastError());
}

// lambda_max(D^-1 K) by `iters` power steps on the device from the start
// vector 1 + 0.5 sin(0.7 i) (0 on constrained DOFs): |z_iters| / |z_(iters-1)|
// with z_(k+1) = D^-1 K z_k.  The iterates are left unnormalised; their
// growth, at most about 9^iters for the plate operators, stays far inside
// FP64's range.  queue_power_steps queues the steps (z_iters ends in pl->xw
// for even iters, else pl->pw; z_(iters-1) in the other), lambda_from_power
// reads them back once the stream has run them and sums the two norms on
// the host, in order.
void queue_power_steps(pg_ctx* c, Plan* pl, int iters) {
    const pg::HostPlan& hp = pl->hp;
    const size_t n = 3 * (size_t)hp.Nn;
    if (n == 0) return;
    run_setup(c, pl);
    if (pl->xw.n != n) pl->xw.alloc(n);
    if (pl->kx.n != n) pl->kx.alloc(n);
    if (pl->pw.n != n) pl->pw.alloc(n);
    cudaStream_t st = c->stream;
    double* a = pl->xw.p;
    double* b = pl->pw.p;
    pg::power_start_kernel<<<((int)n + 255) / 256, 256, 0, st>>>((int)n, pl->cons.p, a);
    CK(cudaGetLastError());
    for (int it = 0; it < iters; it++) {
        if (hp.npe == 4)
            pg::power_step_kernel<4><<<(hp.Nn + 255) / 256, 256, 0, st>>>(
                hp.Nn, pl->inc_ptr.p, pl->inc_idx.p, pl->mesh_elements.p, pl->ke64.p, pl->cons.p, pl->binv64.p, a, b);
        else
            pg::power_step_kernel<3><<<(hp.Nn + 255) / 256, 256, 0, st>>>(
                hp.Nn, pl->inc_ptr.p, pl->inc_idx.p, pl->mesh_elements.p, pl->ke64.p, pl->cons.p, pl->binv64.p, a, b);
        CK(cudaGetLastError());
        std::swap(a, b);
    }
}

double lambda_from_power(pg_ctx* c, Plan* pl, int iters) {
    const size_t n = 3 * (size_t)pl->hp.Nn;
    if (n == 0 || iters < 1) return 1.0;
    const double* last = iters % 2 == 0 ? pl->xw.p : pl->pw.p;
    const double* prev = iters % 2 == 0 ? pl->pw.p : pl->xw.p;
    std::vector<double> za(n), zb(n);
    CK(cudaMemcpyAsync(za.data(), last, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(zb.data(), prev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double na = 0.0, nb = 0.0;
    for (size_t i = 0; i < n; i++) {
        na += za[i] * za[i];
        nb += zb[i] * zb[i];
    }
    const double lam = nb > 0 ? std::sqrt(na / nb) : 0.0;
    return std::isfinite(lam) && lam > 0 ? lam : (double)pl->hp.npe;
}

double device_lambda_max(pg_ctx* c, Plan* pl, int iters) {
    queue_power_steps(c, pl, iters);
    return lambda_from_power(c, pl, iters);
}

void fill_options(const pg_options* in, pg_options* o) {
    pg_options_default(o);
    if (!in) return;
    size_t n = std::min<size_t>(in->struct_size ? in->struct_size : sizeof(pg_options), sizeof(pg_options));
    std::memcpy(o, in, n);
    o->struct_size = sizeof(pg_options);
    if (!(o->tolerance >= 0) || !std::isfinite(o->tolerance)) throw Fail{PG_EINVAL, "tolerance must be finite and >= 0"};
    if (o->max_iterations < 0) throw Fail{PG_EINVAL, "max_iterations must be >= 0"};
    if (o->precision != PG_PREC_FP64 && o->precision != PG_PREC_MIXED)
        throw Fail{PG_EINVAL, "unknown precision"};
    if (o->stop_rule != PG_STOP_REFERENCE && o->stop_rule != PG_STOP_RELATIVE)
        throw Fail{PG_EINVAL, "unknown stop_rule"};
    if (o->threads < 0 || o->threads > pg::kMaxThreads || (o->threads % 32) != 0)
        throw Fail{PG_EINVAL, "threads must be a multiple of 32 in [32, 576] (0 = automatic)"};
    if (o->ctas < 0) throw Fail{PG_EINVAL, "ctas must be >= 0"};
    if (o->batch_part_nodes < 0 || o->batch_part_nodes > 100000)
        throw Fail{PG_EINVAL, "batch_part_nodes must be in [0, 100000]"};
    if (!(o->wait_timeout_ms >= 0) || !std::isfinite(o->wait_timeout_ms) || o->wait_timeout_ms > 600000.0)
        throw Fail{PG_EINVAL, "wait_timeout_ms must be finite and in [0, 600000]"};
    if (o->preconditioner != PG_PRECOND_BLOCK_JACOBI && o->preconditioner != PG_PRECOND_TWO_LEVEL)
        throw Fail{PG_EINVAL, "unknown preconditioner"};
    if (o->smoother != PG_SMOOTHER_BLOCK_JACOBI && o->smoother != PG_SMOOTHER_CHEBYSHEV)
        throw Fail{PG_EINVAL, "unknown smoother"};
}

// Ghost halo a solve with these options needs: 2 element layers for the
// polynomial smoother, else 1.
int halo_rings(const pg_options& o) { return o.smoother == PG_SMOOTHER_CHEBYSHEV ? 2 : 1; }

// Coarse data of the two-level preconditioner, built once per plan.  One
// plate: the aggregate lists and basis data on the host (build_coarse_meta),
// A_c = P^T K P, its factorisation and inverse, and each part's A_c^-1 rows
// on the device (coarse.cuh), from the element matrices already there.
// Batches build the dense part on host threads (prepare_many, build_coarse).
void upload_coarse(pg_ctx* c, Plan* pl);
void carve_coarse(Arena& ar, Plan* pl, size_t n, const double* a64, const float* a32);

void ensure_coarse(pg_ctx* c, Plan* pl) {
    pg::HostPlan& hp = pl->hp;
    if (hp.coarse) return;
    run_setup(c, pl);
    std::string e = pg::build_coarse_meta(pl->prob_view, hp);
    if (!e.empty()) throw Fail{PG_EINVAL, e};
    cudaStream_t st = c->stream;
    const int C = hp.C;
    const size_t CC = (size_t)C * C;
    const int rows = (int)hp.ainv_src.size();
    // the set-up's scratch arrays in one allocation, freed on return; A_c,
    // L, Lt and A_c^-1 ([C][C] each, consecutive) in `mats`: the first three
    // start zeroed, every entry of A_c^-1 is written by coarse_inverse_kernel
    DevBuf<unsigned char> scratch;
    DevBuf<int> owner, src, keep, dropped;
    DevBuf<double> geom, mats;
    {
        Arena ar;
        ar.add(owner, hp.coarse_owner.size(), hp.coarse_owner.data());
        ar.add(geom, hp.coarse_geom.size(), hp.coarse_geom.data());
        ar.add(src, hp.ainv_src.size(), hp.ainv_src.data());
        ar.add(mats, 4 * CC, nullptr);
        ar.add(keep, (size_t)C, nullptr);
        ar.add(dropped, 1, nullptr);
        ar.commit(scratch, st);
    }
    {
        Arena ar;
        carve_coarse(ar, pl, (size_t)rows * C, nullptr, nullptr);
        ar.commit(pl->coarse_arena, st);
    }
    double* const Ac = mats.p;
    double* const L = mats.p + CC;
    double* const Lt = mats.p + 2 * CC;
    double* const Ainv = mats.p + 3 * CC;
    CK(cudaMemsetAsync(mats.p, 0, 3 * CC * sizeof(double), st));
    if (hp.Ne > 0) {
        if (hp.npe == 4)
            pg::coarse_assemble_kernel<4><<<(hp.Ne + 127) / 128, 128, 0, st>>>(
                hp.Ne, C, pl->mesh_nodes.p, pl->mesh_elements.p, pl->cons.p, owner.p, geom.p, pl->ke64.p, Ac);
        else
            pg::coarse_assemble_kernel<3><<<(hp.Ne + 127) / 128, 128, 0, st>>>(
                hp.Ne, C, pl->mesh_nodes.p, pl->mesh_elements.p, pl->cons.p, owner.p, geom.p, pl->ke64.p, Ac);
        CK(cudaGetLastError());
    }
    // the blocked factorisation when its panels fit in shared memory
    // (1 KB left for the kernel's static shared memory)
    const size_t smem_cap = (size_t)c->max_smem - 1024;
    const bool blocked = pg::coarse_factor_blocked_smem(C) <= smem_cap;
    const size_t fsm = blocked ? pg::coarse_factor_blocked_smem(C) : pg::coarse_factor_smem(C);
    if (fsm > smem_cap) throw Fail{PG_EUNSUPPORTED, "coarse space too large for its factorisation"};
    const void* ffn = blocked ? (const void*)pg::coarse_factor_kernel : (const void*)pg::coarse_factor_tiles_kernel;
    if (fsm > 48 * 1024) CK(cudaFuncSetAttribute(ffn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
    {
        const double* acp = Ac;
        double *lp = L, *ltp = Lt;
        int *kp = keep.p, *dp = dropped.p;
        void* fargs[] = {(void*)&C, (void*)&acp, (void*)&lp, (void*)&ltp, (void*)&kp, (void*)&dp};
        CK(cudaLaunchKernel(ffn, dim3(1), dim3(pg::kCoarseThreads), fargs, fsm, st));
    }
    CK(cudaGetLastError());
    // A_c^-1 = L^-T L^-1: one block per 32 x 32 tile of the lower triangle
    const int ntile = (C + 31) / 32;
    pg::coarse_inverse_kernel<<<ntile * (ntile + 1) / 2, pg::kCoarseThreads, 0, st>>>(C, Lt, Ainv);
    CK(cudaGetLastError());
    if (rows > 0) {
        const long tot = (long)rows * C;
        pg::coarse_rows_kernel<<<(int)std::min<long>((tot + 255) / 256, 4096), 256, 0, st>>>(
            rows, C, src.p, Ainv, pl->ainv64.p, pl->ainv32.p);
        CK(cudaGetLastError());
    }
    int nd = 0;
    CK(cudaMemcpyAsync(&nd, dropped.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));  // nd; the scratch is freed on return
    hp.dropped_modes = nd;
    hp.coarse = true;
}

// The plan's device copies of its aggregate lists and node basis data and
// of its A_c^-1 rows (n entries in FP64 and FP32, copied from a64 / a32
// when given, else left for coarse_rows_kernel).
void carve_coarse(Arena& ar, Plan* pl, size_t n, const double* a64, const float* a32) {
    const pg::HostPlan& hp = pl->hp;
    ar.add(pl->ainv64, n, a64);
    ar.add(pl->ainv32, n, a32);
    ar.add(pl->cagg_off, hp.cagg_off.size(), hp.cagg_off.data());
    ar.add(pl->node_slot, hp.node_slot.size(), hp.node_slot.data());
    ar.add(pl->node_basis, hp.node_basis.size(), hp.node_basis.data());
    ar.add(pl->ainv_off, hp.ainv_off.size(), hp.ainv_off.data());
}

// Device copies of a plan's coarse data built on the host (build_coarse).
void upload_coarse(pg_ctx* c, Plan* pl) {
    const pg::HostPlan& hp = pl->hp;
    std::vector<float> a32(hp.ainv.begin(), hp.ainv.end());
    Arena ar;
    carve_coarse(ar, pl, hp.ainv.size(), hp.ainv.data(), a32.data());
    ar.commit(pl->coarse_arena, c->stream);
    CK(cudaStreamSynchronize(c->stream));  // a32 is read by the copy
}

// Largest eigenvalue of D^-1 K for the polynomial smoother, estimated once
// per plan by power steps on the device.
void ensure_smoother(pg_ctx* c, Plan* pl) {
    if (pl->lambda_max > 0) return;
    pl->lambda_max = device_lambda_max(c, pl, 30);
}

// Coefficients of u = a t - b D^-1 K t (t = D^-1 r): two steps of the
// Chebyshev iteration for D^-1 K on [lo, hi], hi = 1.1 lambda_max,
// lo = hi / 20.  The residual polynomial is T2((theta - x) / delta) /
// T2(theta / delta) with theta, delta the centre and half-width; the
// preconditioner polynomial a - b x is positive on (0, hi + lo).
void chebyshev2(double lambda_max, double* a, double* b) {
    const double hi = 1.1 * lambda_max, lo = hi / 20.0;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    const double rho0 = 1.0 / sigma, rho1 = 1.0 / (2.0 * sigma - rho0);
    *a = (1.0 + rho1 * rho0) / theta + 2.0 * rho1 / delta;
    *b = 2.0 * rho1 / (delta * theta);
}

// Queues setup + persistent PCG on the context stream, then waits for the
// result record (one small readback).  F must already be in pl->F.
// Coarse data and the smoother's eigenvalue, built once per plan on first use.
// info (optional) receives the host wall time of the coarse space and of
// the eigenvalue estimate (0 when the plan already had them).
void prepare_plan_data(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* info = nullptr) {
    if (o.smoother == PG_SMOOTHER_CHEBYSHEV && pl->hp.rings != 2)
        throw Fail{PG_EINVAL, "the Chebyshev smoother needs a plan made with it (2-ring halo)"};
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t0) {
        return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    };
    auto t0 = clk::now();
    if (o.preconditioner == PG_PRECOND_TWO_LEVEL && !pl->hp.coarse) {
        ensure_coarse(c, pl);
        if (info) info->coarse_ms = ms_since(t0);
    }
    t0 = clk::now();
    if (o.smoother == PG_SMOOTHER_CHEBYSHEV && !(pl->lambda_max > 0)) {
        ensure_smoother(c, pl);
        if (info) info->eigen_ms = ms_since(t0);
    }
}

// prepare_plan_data for many plans (a batch): the eigenvalue estimates run on
// the device for all plates before one wait; for the coarse matrices the
// element matrices come down in chunks of plates, the host work runs on
// worker threads, and the results go back up.
void prepare_many(pg_ctx* c, const std::vector<Plan*>& pls, const pg_options& o) {
    const bool coarse = o.preconditioner == PG_PRECOND_TWO_LEVEL;
    const bool cheb = o.smoother == PG_SMOOTHER_CHEBYSHEV;
    std::vector<Plan*> todo, lam_todo;
    for (Plan* pl : pls) {
        if (coarse && !pl->hp.coarse) todo.push_back(pl);
        // plates on a 1-ring halo run with block Jacobi (plate_options)
        if (cheb && pl->hp.rings == 2 && !(pl->lambda_max > 0)) lam_todo.push_back(pl);
    }
    // eigenvalue estimates: every plate's power steps queued back to back
    for (Plan* pl : lam_todo) queue_power_steps(c, pl, 30);
    for (Plan* pl : lam_todo) pl->lambda_max = lambda_from_power(c, pl, 30);
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    for (size_t i = 0; i < todo.size();) {
        size_t j = i, elems = 0;
        while (j < todo.size() && (j == i || elems + (size_t)todo[j]->hp.Ne <= 1500000)) elems += todo[j++]->hp.Ne;
        const size_t m = j - i;
        std::vector<std::vector<double>> ke(m);
        for (size_t k = 0; k < m; k++) {
            Plan* pl = todo[i + k];
            run_setup(c, pl);
            const size_t kk = 9 * (size_t)pl->hp.npe * pl->hp.npe;
            ke[k].resize(std::max<size_t>(1, (size_t)pl->hp.Ne * kk));
            if (pl->hp.Ne > 0)
                CK(cudaMemcpyAsync(ke[k].data(), pl->ke64.p, (size_t)pl->hp.Ne * kk * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
        }
        CK(cudaStreamSynchronize(c->stream));
        std::vector<std::string> err(m);
        std::atomic<size_t> next{0};
        auto work = [&]() {
            for (size_t k; (k = next.fetch_add(1)) < m;) {
                Plan* pl = todo[i + k];
                try {
                    err[k] = pg::build_coarse(pl->prob_view, ke[k], pl->hp);
                } catch (...) {
                    err[k] = "host set-up of the batch failed";
                }
            }
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < std::min<size_t>(hw, m); t++) th.emplace_back(work);
        work();
        for (auto& t : th) t.join();
        for (size_t k = 0; k < m; k++) {
            if (!err[k].empty()) throw Fail{PG_EINVAL, err[k]};
            Plan* pl = todo[i + k];
            if (pl->hp.coarse && pl->ainv64.n == 0) upload_coarse(c, pl);
        }
        i = j;
    }
}

// Shared-memory layout of a launch: keep in shared memory what fits, in this
// order of preference: every task's Ke blocks (only differs from the owned
// tasks' with a 2-ring halo) and the A_c^-1 rows; the owned tasks' blocks
// and A_c^-1; then the larger of the owned tasks' blocks and A_c^-1; then
// neither (read from L2).
pg::SmemLayout choose_layout(pg_ctx* c, const pg::HostPlan& hp, const pg_options& o, int* ke_mode,
                             bool* ainv_smem) {
    const bool mixed = o.precision == PG_PREC_MIXED, coarse = o.preconditioner == PG_PRECOND_TWO_LEVEL;
    const int full = hp.rings == 2 ? 2 : 1;
    const bool ke_first = 3 * 3 * hp.npe * (size_t)hp.max_ntask_own >= (size_t)3 * hp.max_kagg * hp.C;
    const int cand[6][2] = {{full, 1}, {1, 1}, {ke_first ? full : 0, ke_first ? 0 : 1},
                            {ke_first ? 1 : 0, ke_first ? 0 : 1}, {0, 1}, {0, 0}};
    pg::SmemLayout L{};
    for (auto& cd : cand) {
        *ke_mode = cd[0];
        *ainv_smem = coarse && cd[1];
        L = make_layout(hp, mixed, *ke_mode, coarse, *ainv_smem);
        if (L.total <= c->max_smem) break;
    }
    if (L.total > c->max_smem)
        throw Fail{PG_EUNSUPPORTED, "partition too large for shared memory: use more ctas"};
    return L;
}

// Clears what a launch of pl needs cleared: its result record, and its
// exchange buffers on the plan's first launch, after a failed one, or when
// the round tags come near 0xffffffff (the test hook's tag); otherwise the
// tags simply continue from the last launch.
void reset_for_launch(pg_ctx* c, Plan* pl, pg::PcgResult* res) {
    if (!pl->ll_ready || pl->tag0 > 0xf0000000u) {
        CK(cudaMemsetAsync(pl->llv.p, 0, pl->llv.n * sizeof(unsigned long long), c->stream));
        CK(cudaMemsetAsync(pl->llx.p, 0, pl->llx.n * sizeof(unsigned long long), c->stream));
        CK(cudaMemsetAsync(pl->llp.p, 0, pl->llp.n * sizeof(unsigned long long), c->stream));
        pl->tag0 = 0;
    }
    pl->ll_ready = false;  // until this launch's result record is back
    CK(cudaMemsetAsync(res, 0, sizeof(pg::PcgResult), c->stream));
}

pg::PcgArgs fill_args(Plan* pl, const pg_options& o, const pg::SmemLayout& L, int ke_mode,
                      bool ainv_smem, int* abort_flag, pg::PcgResult* res) {
    const pg::HostPlan& hp = pl->hp;
    const bool coarse = o.preconditioner == PG_PRECOND_TWO_LEVEL;
    const bool cheb = o.smoother == PG_SMOOTHER_CHEBYSHEV;
    pg::PcgArgs a{};
    a.G = pl->G;
    a.NT = (int)hp.task_elem.size();
    a.Nn = hp.Nn;
    a.npe = hp.npe;
    a.node_off = pl->node_off.p;
    a.nown = pl->nown.p;
    a.nodes = pl->nodes.p;
    a.task_off = pl->task_off.p;
    a.tp_off = pl->tp_off.p;
    a.tptr = pl->tptr.p;
    a.task_nodes = pl->task_nodes.p;
    a.kt64 = pl->kt64.p;
    a.kt32 = pl->kt32.p;
    a.binv64 = pl->binv64.p;
    a.binv32 = pl->binv32.p;
    a.cons = pl->cons.p;
    a.F = pl->F.p;
    a.x = pl->x.p;
    a.llv = pl->llv.p;
    a.llx = pl->llx.p;
    a.llp = pl->llp.p;
    a.abort_flag = abort_flag;
    a.res = res;
    a.tol = o.tolerance;
    a.tag0 = pl->tag0;
    a.maxit = o.max_iterations;
    a.stop_rule = o.stop_rule;
    a.timeout_ns = (unsigned long long)(o.wait_timeout_ms * 1e6);
    a.ke_smem = ke_mode;
    a.timing = o.phase_timing ? 1 : 0;
    a.test_stall = o.test_stall ? 1 : 0;
    a.coarse = coarse ? 1 : 0;
    a.C = coarse ? hp.C : 0;
    a.cagg_off = pl->cagg_off.p;
    a.node_slot = pl->node_slot.p;
    a.node_basis = pl->node_basis.p;
    a.ainv_off = pl->ainv_off.p;
    a.ainv64 = pl->ainv64.p;
    a.ainv32 = pl->ainv32.p;
    a.ainv_smem = ainv_smem ? 1 : 0;
    a.smoother = cheb ? 1 : 0;
    a.n1 = pl->n1.p;
    if (cheb) chebyshev2(pl->lambda_max, &a.cheb_a, &a.cheb_b);
    a.trace_it = o.trace_iteration > 0 ? o.trace_iteration : -1;
    a.trace = pl->trace.p;
    // automatic: a replacement at least every 200 updates, so a mixed solve
    // whose FP32 residual stalls along with the true one is still checked
    a.reliable_interval = o.reliable_interval > 0 ? o.reliable_interval : 200;
    a.reliable_delta = o.reliable_delta > 0 ? o.reliable_delta : 0.1;
    a.L = L;
    return a;
}

// After the result record is back: tags continue next launch if this one ended cleanly.
void finish_launch(Plan* pl, const pg::PcgResult& r) {
    if (r.status == pg::ST_OK && r.wait_failures == 0) {
        pl->tag0 = r.last_tag;
        pl->ll_ready = true;
    }
}

void fill_info(pg_info* info, const pg::PcgResult& r, const Plan* pl, const pg_options& o, int threads,
               int shared_bytes) {
    const pg::HostPlan& hp = pl->hp;
    info->iterations = r.iterations;
    info->converged = r.converged;
    info->stop_reason = r.stop_reason;
    info->final_residual = r.final_residual;
    info->true_rel_residual = r.true_rel_residual;
    info->b_norm = r.b_norm;
    info->ctas = pl->G;
    info->threads = threads;
    info->reliable_updates = r.reliable_updates;
    info->reductions = r.reductions;
    info->shared_bytes = shared_bytes;
    info->coarse_dim = o.preconditioner == PG_PRECOND_TWO_LEVEL ? hp.C - hp.dropped_modes : 0;
    info->smoother_lambda_max = o.smoother == PG_SMOOTHER_CHEBYSHEV ? pl->lambda_max : 0.0;
}

void throw_on_failure(const pg::PcgResult& r) {
    if (r.wait_failures > 0 || r.status == PG_ETIMEOUT)
        throw Fail{PG_ETIMEOUT, "a wait for another block exceeded wait_timeout_ms"};
    if (r.status == PG_ENONFINITE) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "non-finite value in the PCG iteration (reduction %d: gamma=%g delta=%g rho=%g)",
                      r.nonfinite_it, r.nonfinite_vals[0], r.nonfinite_vals[1], r.nonfinite_vals[2]);
        throw Fail{PG_ENONFINITE, buf};
    }
}

// Gives kernel fn the full shared-memory opt-in once per context.
void opt_in_smem(pg_ctx* c, const void* fn) {
    if (std::find(c->smem_opt_in.begin(), c->smem_opt_in.end(), fn) == c->smem_opt_in.end()) {
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, c->max_smem));
        c->smem_opt_in.push_back(fn);
    }
}

// Queues set-up (first solve of the plan) and the persistent PCG launch on
// the context stream, then waits for the result record (one readback).
// x_dst (optional) receives the solution by a copy of `kind` queued right
// behind the kernel, so the call waits for the device once.
void run_solve(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* info, void* x_dst = nullptr,
               cudaMemcpyKind kind = cudaMemcpyDeviceToDevice) {
    const pg::HostPlan& hp = pl->hp;
    const bool mixed = o.precision == PG_PREC_MIXED;
    int threads = o.threads;
    if (!threads) {
        // one thread per task of the largest part, within the launch bound:
        // up to 512 threads the kernel has 128 registers (576: 96), which
        // measured faster for FP32 inner iterations and for FP64 block
        // Jacobi; FP64 with the Chebyshev smoother keeps 576 threads (its
        // split task passes: fewer of them)
        const bool wide = !mixed && o.smoother == PG_SMOOTHER_CHEBYSHEV;
        threads = std::min(wide ? pg::kMaxThreads : pg::kLeanThreads, std::max(128, (hp.max_ntask + 31) / 32 * 32));
    }
    const bool lean = threads <= pg::kLeanThreads;
    prepare_plan_data(c, pl, o, info);
    int ke_mode = 0;
    bool ainv_smem = false;
    const pg::SmemLayout L = choose_layout(c, hp, o, &ke_mode, &ainv_smem);

    CK(cudaEventRecord(c->ev[0], c->stream));
    run_setup(c, pl);
    CK(cudaEventRecord(c->ev[1], c->stream));
    reset_for_launch(c, pl, pl->res.p);
    CK(cudaMemsetAsync(pl->abort_flag.p, 0, sizeof(int), c->stream));
    pg::PcgArgs a = fill_args(pl, o, L, ke_mode, ainv_smem, pl->abort_flag.p, pl->res.p);
    if (a.trace_it > 0)
        CK(cudaMemsetAsync(pl->trace.p, 0, pl->trace.n * sizeof(unsigned long long), c->stream));

    const void* fn;
    constexpr int LT = pg::kLeanThreads, MT = pg::kMaxThreads;
    if (hp.npe == 4)
        fn = mixed ? (lean ? (const void*)pg::pcg_kernel<4, float, true, LT> : (const void*)pg::pcg_kernel<4, float, true, MT>)
                   : (lean ? (const void*)pg::pcg_kernel<4, double, false, LT>
                           : (const void*)pg::pcg_kernel<4, double, false, MT>);
    else
        fn = mixed ? (lean ? (const void*)pg::pcg_kernel<3, float, true, LT> : (const void*)pg::pcg_kernel<3, float, true, MT>)
                   : (lean ? (const void*)pg::pcg_kernel<3, double, false, LT>
                           : (const void*)pg::pcg_kernel<3, double, false, MT>);
    opt_in_smem(c, fn);
    if (pl->ok_fn != fn || pl->ok_threads != threads || pl->ok_smem != L.total) {
        int nb = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, L.total));
        if (nb < 1 || nb * c->sms < pl->G)
            throw Fail{PG_EUNSUPPORTED, "persistent grid does not fit on the device"};
        pl->ok_fn = fn;
        pl->ok_threads = threads;
        pl->ok_smem = L.total;
    }
    void* args[] = {&a};
    CK(cudaLaunchCooperativeKernel(fn, dim3(pl->G), dim3(threads), args, L.total, c->stream));
    CK(cudaEventRecord(c->ev[2], c->stream));
    pg::PcgResult r{};
    if (x_dst)
        CK(cudaMemcpyAsync(x_dst, pl->x.p, 3 * (size_t)hp.Nn * sizeof(double), kind, c->stream));
    CK(cudaMemcpyAsync(&r, pl->res.p, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    finish_launch(pl, r);
    float ms_setup = 0, ms_solve = 0;
    CK(cudaEventElapsedTime(&ms_setup, c->ev[0], c->ev[1]));
    CK(cudaEventElapsedTime(&ms_solve, c->ev[1], c->ev[2]));
    if (info) {
        fill_info(info, r, pl, o, threads, L.total);
        info->setup_ms = ms_setup;
        info->solve_ms = ms_solve;
        for (int k = 0; k < 8; k++) info->phase_us[k] = r.phase_cycles[k] / (c->clock_khz * 1e-3);
        if (a.trace_it > 0) {
            std::vector<unsigned long long> tr(pl->trace.n);
            CK(cudaMemcpy(tr.data(), pl->trace.p, tr.size() * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost));
            unsigned long long s0 = ~0ull, s1 = 0, p0 = ~0ull, p1 = 0, x0 = ~0ull, x1 = 0, e1 = 0;
            for (int g = 0; g < pl->G; g++) {
                s0 = std::min(s0, tr[4 * g]); s1 = std::max(s1, tr[4 * g]);
                p0 = std::min(p0, tr[4 * g + 1]); p1 = std::max(p1, tr[4 * g + 1]);
                x0 = std::min(x0, tr[4 * g + 2]); x1 = std::max(x1, tr[4 * g + 2]);
                e1 = std::max(e1, tr[4 * g + 3]);
            }
            if (s0 > 0) {
                info->trace_ns[0] = (double)(s1 - s0);  // start spread
                info->trace_ns[1] = (double)(p1 - p0);  // publish spread
                info->trace_ns[2] = (double)(p1 - s0);  // first start -> last publish
                info->trace_ns[3] = (double)(x0 - p1);  // last publish -> first block done
                info->trace_ns[4] = (double)(x1 - x0);  // exchange-done spread
                info->trace_ns[5] = (double)(e1 - s0);  // whole iteration (first start -> last end)
            }
        }
    }
    throw_on_failure(r);
}

// run_solve, and when a mixed solve stagnated (with o.fallback) the same
// solve again in FP64 on the same plan; info then describes the FP64 solve,
// with fallback = 1 and solve_ms covering both.
// Queues ||F - K x||^2 and ||F||^2 of plan pl into pl->nrm (uses pl->kx).
void queue_true_residual(pg_ctx* c, Plan* pl, const double* x, const float* F) {
    const int n = 3 * pl->hp.Nn;
    if (pl->kx.n != (size_t)n) pl->kx.alloc(n);
    if (pl->nrm.n != 2) pl->nrm.alloc(2);
    queue_apply_k(c, pl, x, pl->kx.p);
    CK(cudaMemsetAsync(pl->nrm.p, 0, 2 * sizeof(double), c->stream));
    const int blocks = std::max(1, std::min(4 * c->sms, (n + 255) / 256));
    pg::residual_norms_kernel<<<blocks, 256, 0, c->stream>>>(n, pl->cons.p, F, pl->kx.p, pl->nrm.p);
    CK(cudaGetLastError());
}

// Stop of an FP64 correction K d = F - K x_m: the caller's rule on x_m + d
// (||r|| < tol or ||r|| / ||F|| < tol; or the relative test alone) as a
// relative tolerance on the correction's load, whose norm is r0.
double correction_tolerance(const pg_options& o, double bnorm, double r0) {
    const double target = o.stop_rule == PG_STOP_REFERENCE ? std::max(o.tolerance, o.tolerance * bnorm)
                                                           : o.tolerance * bnorm;
    return r0 > 0 ? std::min(0.5, target / r0) : o.tolerance;
}

// After a mixed solve of pl stagnated (pl->x holds its x_m, pl->F the
// load): solves K d = F - K x_m in FP64, its load the FP32-rounded residual
// and its stop scaled to the residual x_m already reached, then x = x_m + d
// into x_dst.  mi: the mixed solve's record in (its final residual is the
// FP64 true residual of x_m), the result's out.
void fp64_correction(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* mi, void* x_dst,
                     cudaMemcpyKind kind) {
    const size_t n = 3 * (size_t)pl->hp.Nn;
    const int ni = (int)n;
    const double bnorm = mi->b_norm, r0 = mi->final_residual;
    cudaStream_t st = c->stream;
    if (pl->xw.n != n) pl->xw.alloc(n);
    if (pl->kx.n != n) pl->kx.alloc(n);
    if (pl->rf.n != n) pl->rf.alloc(n);
    // the load kept in rf; the correction's load into F (what run_solve reads)
    CK(cudaMemcpyAsync(pl->rf.p, pl->F.p, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(pl->xw.p, pl->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    queue_apply_k(c, pl, pl->xw.p, pl->kx.p);
    pg::residual_f32_kernel<<<(ni + 255) / 256, 256, 0, st>>>(ni, pl->cons.p, pl->rf.p, pl->kx.p, pl->F.p);
    CK(cudaGetLastError());
    pg_options o64 = o;
    o64.precision = PG_PREC_FP64;
    o64.stop_rule = PG_STOP_RELATIVE;
    o64.tolerance = correction_tolerance(o, bnorm, r0);
    pg_info fi{};
    run_solve(c, pl, o64, &fi, nullptr, kind);
    pg::add_kernel<<<(ni + 255) / 256, 256, 0, st>>>(ni, pl->xw.p, pl->x.p);
    CK(cudaGetLastError());
    queue_true_residual(c, pl, pl->x.p, pl->rf.p);
    double nrm[2] = {0.0, 0.0};
    CK(cudaMemcpyAsync(nrm, pl->nrm.p, sizeof nrm, cudaMemcpyDeviceToHost, st));
    if (x_dst) CK(cudaMemcpyAsync(x_dst, pl->x.p, n * sizeof(double), kind, st));
    CK(cudaStreamSynchronize(st));
    const double mixed_ms = mi->setup_ms + mi->solve_ms;
    *mi = fi;
    mi->true_rel_residual = nrm[1] > 0 ? std::sqrt(nrm[0] / nrm[1]) : 0.0;
    mi->b_norm = bnorm;
    mi->fallback = 1;
    mi->solve_ms += mixed_ms;
}

pgi::OperatorView operator_view(Plan* pl) {
    const pg::HostPlan& hp = pl->hp;
    pgi::OperatorView v;
    v.Nn = hp.Nn;
    v.Ne = hp.Ne;
    v.npe = hp.npe;
    v.inc_ptr = pl->inc_ptr.p;
    v.inc_idx = pl->inc_idx.p;
    v.elements = pl->mesh_elements.p;
    v.ke32 = pl->ke32.p;
    v.ke64 = pl->ke64.p;
    v.binv32 = pl->binv32.p;
    v.binv64 = pl->binv64.p;
    v.cons = pl->cons.p;
    return v;
}

// Whether the smallest layout of the persistent kernel (element blocks and
// coarse rows in L2) fits one block's shared memory for this plan's parts.
bool persistent_fits(const pg_ctx* c, const Plan* pl, const pg_options& o) {
    const pg::SmemLayout L = make_layout(pl->hp, o.precision == PG_PREC_MIXED, 0, false, false);
    return L.total <= c->max_smem;
}

// A plate whose parts do not fit shared memory even with one part per SM:
// flexible PCG over global memory (FP32 vectors in L2/HBM, FP64 x, dot
// products and true-residual stop), block Jacobi, or damped block-Jacobi
// smoothing steps when a faster preconditioner was asked for.  F is in
// pl->F.
void global_solve(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* info, void* x_dst, cudaMemcpyKind kind) {
    run_setup(c, pl);
    if (!pl->gpcg) {
        if (!(pl->lambda_max > 0)) pl->lambda_max = device_lambda_max(c, pl, 30);
        std::string err;
        pl->gpcg = pgi::global_pcg_create(c, operator_view(pl), pl->lambda_max, &err);
        if (!pl->gpcg) throw Fail{PG_ECUDA, err};
    }
    if (!x_dst) {
        if (pl->x.n != 3 * (size_t)pl->hp.Nn) pl->x.alloc(3 * (size_t)pl->hp.Nn);
        x_dst = pl->x.p;
        kind = cudaMemcpyDeviceToDevice;
    }
    const int mode = (o.preconditioner == PG_PRECOND_TWO_LEVEL || o.smoother == PG_SMOOTHER_CHEBYSHEV) ? 2 : 0;
    std::string err;
    pg_info local{};
    pg_info* fi = info ? info : &local;
    const int st = pgi::global_pcg_solve(pl->gpcg, o, mode, pl->F.p, x_dst, kind == cudaMemcpyDeviceToHost, fi, &err);
    if (st != PG_OK) throw Fail{st, err};
    fi->ctas = pl->G;
    fi->global_path = 1;
}

void solve_with_fallback(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* info, void* x_dst = nullptr,
                         cudaMemcpyKind kind = cudaMemcpyDeviceToDevice) {
    pg_info local{};
    pg_info* fi = info ? info : &local;
    if (!persistent_fits(c, pl, o)) {
        global_solve(c, pl, o, fi, x_dst, kind);
        return;
    }
    run_solve(c, pl, o, fi, x_dst, kind);
    if (o.precision != PG_PREC_MIXED || !o.fallback || fi->stop_reason != PG_STOP_STAGNATED) return;
    fp64_correction(c, pl, o, fi, x_dst, kind);
}

// Layout of an NR-case launch: the first of the single solve's preferences
// that fits; false when none does (the plate's parts are then solved with
// fewer cases per launch).
bool choose_layout_multi(pg_ctx* c, const pg::HostPlan& hp, const pg_options& o, int NR, int* ke_mode,
                         bool* ainv_smem, pg::SmemLayout* out) {
    const bool mixed = o.precision == PG_PREC_MIXED, coarse = o.preconditioner == PG_PRECOND_TWO_LEVEL;
    const int full = hp.rings == 2 ? 2 : 1;
    const bool ke_first = 3 * 3 * hp.npe * (size_t)hp.max_ntask_own >= (size_t)3 * hp.max_kagg * hp.C;
    const int cand[6][2] = {{full, 1}, {1, 1}, {ke_first ? full : 0, ke_first ? 0 : 1},
                            {ke_first ? 1 : 0, ke_first ? 0 : 1}, {0, 1}, {0, 0}};
    for (auto& cd : cand) {
        *ke_mode = cd[0];
        *ainv_smem = coarse && cd[1];
        *out = make_layout_multi(hp, mixed, *ke_mode, coarse, *ainv_smem, NR);
        if (out->total <= c->max_smem) return true;
    }
    return false;
}

const void* multi_kernel(int npe, bool mixed, int NR) {
    if (npe == 4) {
        if (NR == 2) return mixed ? (const void*)pg::pcg_multi_kernel<4, float, true, 2>
                                  : (const void*)pg::pcg_multi_kernel<4, double, false, 2>;
        return mixed ? (const void*)pg::pcg_multi_kernel<4, float, true, 4>
                     : (const void*)pg::pcg_multi_kernel<4, double, false, 4>;
    }
    if (NR == 2) return mixed ? (const void*)pg::pcg_multi_kernel<3, float, true, 2>
                              : (const void*)pg::pcg_multi_kernel<3, double, false, 2>;
    return mixed ? (const void*)pg::pcg_multi_kernel<3, float, true, 4>
                 : (const void*)pg::pcg_multi_kernel<3, double, false, 4>;
}

// count <= NR load cases of plan pl in one launch of the NR-case kernel
// (cases count..NR-1 get a zero load and stop at once).  F[k] / x[k] are
// host vectors of 3 Nn; infos (optional) gets one record per case.  Cases
// whose mixed solve stagnated are solved again, one by one, in FP64.
void run_solve_multi(pg_ctx* c, Plan* pl, const pg_options& o, int NR, int count, const float* const* F,
                     double* const* x, pg_info* infos) {
    const pg::HostPlan& hp = pl->hp;
    const bool mixed = o.precision == PG_PREC_MIXED;
    const size_t n = 3 * (size_t)hp.Nn;
    prepare_plan_data(c, pl, o);
    int ke_mode = 0;
    bool ainv_smem = false;
    pg::SmemLayout L{};
    if (!choose_layout_multi(c, hp, o, NR, &ke_mode, &ainv_smem, &L))
        throw Fail{PG_EUNSUPPORTED, "load-case partition too large for shared memory"};
    cudaStream_t st = c->stream;
    if (pl->m_nr != NR) {
        pl->mF.alloc(n * NR);
        pl->mx.alloc(n * NR);
        pl->mllv.alloc(2 * n * NR * 2);
        pl->mllx.alloc(n * NR * 2);
        pl->mllp.alloc(2 * (size_t)pg::kRep * pl->G * pg::multi_slot_words<4>() + 2);
        pl->mres.alloc(NR);
        pl->m_nr = NR;
        pl->m_ready = false;
    }
    ensure_staging(c, n * NR);
    for (int k = 0; k < NR; k++) {
        if (k < count)
            std::memcpy(c->hF + k * n, F[k], n * sizeof(float));
        else
            std::memset(c->hF + k * n, 0, n * sizeof(float));
    }
    CK(cudaEventRecord(c->ev[0], st));
    run_setup(c, pl);
    CK(cudaMemcpyAsync(pl->mF.p, c->hF, n * NR * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(c->ev[1], st));
    if (!pl->m_ready || pl->m_tag0 > 0xf0000000u) {
        CK(cudaMemsetAsync(pl->mllv.p, 0, pl->mllv.n * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(pl->mllx.p, 0, pl->mllx.n * sizeof(unsigned long long), st));
        CK(cudaMemsetAsync(pl->mllp.p, 0, pl->mllp.n * sizeof(unsigned long long), st));
        pl->m_tag0 = 0;
    }
    pl->m_ready = false;
    CK(cudaMemsetAsync(pl->mres.p, 0, NR * sizeof(pg::PcgResult), st));
    CK(cudaMemsetAsync(pl->abort_flag.p, 0, sizeof(int), st));
    pg::PcgArgs a = fill_args(pl, o, L, ke_mode, ainv_smem, pl->abort_flag.p, pl->mres.p);
    a.F = pl->mF.p;
    a.x = pl->mx.p;
    a.llv = pl->mllv.p;
    a.llx = pl->mllx.p;
    a.llp = pl->mllp.p;
    a.tag0 = pl->m_tag0;
    a.trace_it = -1;
    const void* fn = multi_kernel(hp.npe, mixed, NR);
    opt_in_smem(c, fn);
    if (pl->m_ok_fn != fn || pl->m_ok_smem != L.total) {
        int nb = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, pg::kMultiThreads, L.total));
        if (nb < 1 || nb * c->sms < pl->G)
            throw Fail{PG_EUNSUPPORTED, "load-case grid does not fit on the device"};
        pl->m_ok_fn = fn;
        pl->m_ok_smem = L.total;
    }
    void* args[] = {&a};
    CK(cudaLaunchCooperativeKernel(fn, dim3(pl->G), dim3(pg::kMultiThreads), args, L.total, st));
    CK(cudaEventRecord(c->ev[2], st));
    std::vector<pg::PcgResult> r(NR);
    if (x) CK(cudaMemcpyAsync(c->hx, pl->mx.p, n * count * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(r.data(), pl->mres.p, NR * sizeof(pg::PcgResult), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool clean = r[0].wait_failures == 0;
    unsigned last = 0;
    for (int k = 0; k < NR; k++) {
        clean = clean && r[k].status == pg::ST_OK;
        last = std::max(last, r[k].last_tag);
    }
    if (clean) {
        pl->m_tag0 = last;
        pl->m_ready = true;
    }
    float ms_setup = 0, ms_solve = 0;
    CK(cudaEventElapsedTime(&ms_setup, c->ev[0], c->ev[1]));
    CK(cudaEventElapsedTime(&ms_solve, c->ev[1], c->ev[2]));
    if (x)
        for (int k = 0; k < count; k++) std::memcpy(x[k], c->hx + k * n, n * sizeof(double));
    for (int k = 0; k < count; k++) {
        if (infos) {
            std::memset(&infos[k], 0, sizeof(pg_info));
            fill_info(&infos[k], r[k], pl, o, pg::kMultiThreads, L.total);
            infos[k].status = r[k].status;
            infos[k].setup_ms = ms_setup;
            infos[k].solve_ms = ms_solve;
            infos[k].plan_cached = 1;
            for (int q = 0; q < 8; q++) infos[k].phase_us[q] = r[0].phase_cycles[q] / (c->clock_khz * 1e-3);
        }
    }
    if (r[0].wait_failures > 0) throw_on_failure(r[0]);
    for (int k = 0; k < count; k++) throw_on_failure(r[k]);
    if (!mixed || !o.fallback) return;
    for (int k = 0; k < count; k++) {
        if (r[k].stop_reason != PG_STOP_STAGNATED) continue;
        // the case's x_m and load into the plan's one-load buffers, then the
        // FP64 correction as for a one-load solve
        CK(cudaMemcpyAsync(pl->x.p, pl->mx.p + k * n, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(pl->F.p, F[k], n * sizeof(float), cudaMemcpyHostToDevice, st));
        pg_info fi{};
        fill_info(&fi, r[k], pl, o, pg::kMultiThreads, L.total);
        fi.solve_ms = ms_solve;
        fp64_correction(c, pl, o, &fi, x ? (void*)x[k] : nullptr, cudaMemcpyDeviceToHost);
        if (infos) {
            infos[k] = fi;
            infos[k].plan_cached = 1;
        }
    }
}

template <typename F>
int guarded(pg_ctx* c, pg_info* info, F&& body) {
    if (!c) return PG_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    auto t0 = std::chrono::steady_clock::now();
    int st = PG_OK;
    try {
        CK(cudaSetDevice(c->device));
        body();
    } catch (const Fail& f) {
        c->err = f.msg;
        st = f.status;
    } catch (const std::bad_alloc&) {
        c->err = "host allocation failed";
        st = PG_ENOMEM;
    } catch (...) {
        c->err = "internal error";
        st = PG_ECUDA;
    }
    if (info) {
        info->status = st;
        info->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

void check_problem(const pg_problem* p, bool need_rhs) {
    if (!p) throw Fail{PG_EINVAL, "problem is NULL"};
    std::string e = pg::validate_problem(*p, need_rhs);
    if (!e.empty()) throw Fail{PG_EINVAL, e};
}

void zero_info(pg_info* info) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
}

}  // namespace

namespace {

// Owned nodes per block that the shared-memory layout holds (vectors, block
// inverses, task results; the Ke blocks then stay in L2): a first guess,
// checked against each plate's actual layout by build_batch.  DKT nodes
// carry about 6 element tasks instead of 4.
int batch_capacity(const pg_options& o, int rings, int npe) {
    const bool mixed = o.precision == PG_PREC_MIXED;
    // about 85% of what the layout holds for a 257 x 257-node plate's parts
    static const int cap[2][2][2] = {{{450, 300}, {400, 250}},   // FP64: Q4, DKT x rings 1, 2
                                     {{640, 500}, {560, 380}}};  // mixed
    return cap[mixed ? 1 : 0][npe == 3 ? 1 : 0][rings == 2 ? 1 : 0];
}

// The options a plate of a batch runs with: the batch's, but the
// block-Jacobi smoother where the plate's plan has a 1-ring halo (a plate
// whose 2-ring layout for the Chebyshev smoother does not fit in shared
// memory even on the whole device).
pg_options plate_options(const pg_options& o, const Plan* pl) {
    pg_options oi = o;
    if (pl->hp.rings != 2) oi.smoother = PG_SMOOTHER_BLOCK_JACOBI;
    return oi;
}

std::unique_ptr<pg_batch> build_batch(pg_ctx* c, const pg_problem* probs, int count,
                                      const pg_options& o) {
    auto b = std::make_unique<pg_batch>();
    b->ctx = c;
    b->rings = halo_rings(o);
    std::vector<int> nodes(count);
    for (int i = 0; i < count; i++) {
        check_problem(&probs[i], true);
        if (probs[i].node_count == 0) throw Fail{PG_EINVAL, "a plate of the batch has no nodes"};
        const size_t n = 3 * (size_t)probs[i].node_count;
        for (size_t k = 0; k < n; k++)
            if (!std::isfinite(probs[i].F[k])) throw Fail{PG_ENONFINITE, "F contains NaN or Inf"};
        nodes[i] = (int)probs[i].node_count;
    }
    // schedule, then check every plate's layout at its team size; lower the
    // capacity of the plates whose parts do not fit and reschedule
    std::vector<int> caps(count), kinds(count), rings(count, b->rings);
    for (int i = 0; i < count; i++) kinds[i] = (int)probs[i].nodes_per_element;
    for (int i = 0; i < count; i++) {
        caps[i] = batch_capacity(o, rings[i], (int)probs[i].nodes_per_element);
        // a plate too large for the whole device at the first guess gets the
        // whole device anyway; its layout (element blocks and A_c^-1 rows then
        // possibly in L2, as in a one-plate solve) is checked below
        caps[i] = std::max(caps[i], (nodes[i] + c->sms - 1) / c->sms);
    }
    for (int attempt = 0;; attempt++) {
        std::string e = pg::schedule_batch(nodes, caps, kinds, c->sms, b->sched, o.batch_part_nodes);
        if (!e.empty() && attempt > 0)
            throw Fail{PG_EUNSUPPORTED, "a plate of the batch does not fit in shared memory even on the whole "
                                        "device with these options"};
        if (!e.empty()) throw Fail{PG_EUNSUPPORTED, e};
        b->plans.clear();
        bool fits = true;
        for (int i = 0; i < count; i++) {
            const int G = b->sched.plate_size[i];
            b->plans.push_back(build_plan(c, probs[i], G, rings[i]));
            int ke_mode = 0;
            bool ainv = false;
            try {
                choose_layout(c, b->plans.back()->hp, plate_options(o, b->plans.back().get()), &ke_mode, &ainv);
            } catch (const Fail&) {
                fits = false;
                if (rings[i] == 2 && G == c->sms) {
                    // the 2-ring halo does not fit even on the whole device:
                    // this plate runs with a 1-ring halo and block Jacobi
                    rings[i] = 1;
                    caps[i] = std::max(batch_capacity(o, 1, (int)probs[i].nodes_per_element),
                                       (nodes[i] + c->sms - 1) / c->sms);
                } else {
                    // the next attempt gets at least twice as many blocks (a cap
                    // below n/G), past the largest power of two the whole device,
                    // and never less than the whole device's share, so a plate
                    // that keeps failing reaches the whole-device attempt (and,
                    // with a 2-ring halo, the 1-ring fallback above)
                    const int floor_cap = (nodes[i] + c->sms - 1) / c->sms;
                    const int below = std::max(1, (nodes[i] - 1) / std::max(1, G));
                    caps[i] = std::max(floor_cap, std::min(caps[i] * 3 / 4, below));
                }
            }
        }
        if (fits) break;
        if (attempt == 11) throw Fail{PG_EUNSUPPORTED, "batch plates too large for shared memory"};
    }
    cudaStream_t st = c->stream;
    for (const pg::BatchPhase& P : b->sched.phases) {
        auto d = std::make_unique<BatchPhaseDev>();
        std::vector<int> bt(P.grid);
        for (size_t t = 0; t < P.team_size.size(); t++)
            for (int k = 0; k < P.team_size[t]; k++) bt[P.team_base[t] + k] = (int)t;
        d->grid = P.grid;
        d->kind = P.kind;
        d->block_team.upload(bt.data(), bt.size(), st);
        d->team_base.upload(P.team_base.data(), P.team_base.size(), st);
        d->team_class.upload(P.team_class.data(), P.team_class.size(), st);
        d->class_off.upload(P.class_off.data(), P.class_off.size(), st);
        d->class_queue.upload(P.class_queue.data(), P.class_queue.size(), st);
        d->log_off.upload(P.log_off.data(), P.log_off.size(), st);
        d->class_next.alloc(std::max<size_t>(1, P.class_off.size() - 1));
        d->claims.alloc(std::max(1, P.log_off.back()));
        CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
        b->phases.push_back(std::move(d));
    }
    b->abort_flag.alloc(1);
    b->claim_failures.alloc(1);
    b->args.alloc(count);
    b->res.alloc(count);
    b->times.alloc(2 * (size_t)count);
    b->hF.resize(count);
    for (int i = 0; i < count; i++) {
        b->hF[i].assign(probs[i].F, probs[i].F + 3 * (size_t)probs[i].node_count);
        CK(cudaMemcpyAsync(b->plans[i]->F.p, b->hF[i].data(), b->hF[i].size() * sizeof(float),
                           cudaMemcpyHostToDevice, st));
    }
    CK(cudaStreamSynchronize(st));
    return b;
}

void run_batch(pg_batch* b, const pg_options& o, const float* const* F, double* const* x_out,
               pg_info* infos, pg_batch_info* bi, const double* tols = nullptr);

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)pos, hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

// tols (optional): a stop tolerance per plate in place of o.tolerance.
void run_batch(pg_batch* b, const pg_options& o, const float* const* F, double* const* x_out,
               pg_info* infos, pg_batch_info* bi, const double* tols) {
    pg_ctx* c = b->ctx;
    const int count = (int)b->plans.size();
    if (halo_rings(o) != b->rings)
        throw Fail{PG_EINVAL, "the batch was made for another smoother (ghost halo width)"};
    cudaStream_t st = c->stream;
    if (F)
        for (int i = 0; i < count; i++) {
            if (!F[i]) continue;
            const size_t n = 3 * (size_t)b->plans[i]->hp.Nn;
            for (size_t k = 0; k < n; k++)
                if (!std::isfinite(F[i][k])) throw Fail{PG_ENONFINITE, "F contains NaN or Inf"};
            b->hF[i].assign(F[i], F[i] + n);
            CK(cudaMemcpyAsync(b->plans[i]->F.p, b->hF[i].data(), n * sizeof(float), cudaMemcpyHostToDevice,
                               st));
        }
    {
        std::vector<Plan*> pls;
        for (auto& pl : b->plans) pls.push_back(pl.get());
        prepare_many(c, pls, o);
    }
    CK(cudaEventRecord(c->ev[0], st));
    for (auto& pl : b->plans) run_setup(c, pl.get());
    CK(cudaEventRecord(c->ev[1], st));
    std::vector<pg::PcgArgs> a(count);
    int smem = 0;
    for (int i = 0; i < count; i++) {
        Plan* pl = b->plans[i].get();
        const pg_options oi = plate_options(o, pl);
        int ke_mode = 0;
        bool ainv = false;
        const pg::SmemLayout L = choose_layout(c, pl->hp, oi, &ke_mode, &ainv);
        reset_for_launch(c, pl, b->res.p + i);
        pg::PcgArgs ai = fill_args(pl, oi, L, ke_mode, ainv, b->abort_flag.p, b->res.p + i);
        ai.timing = 0;
        ai.test_stall = 0;
        ai.trace_it = -1;
        if (tols) ai.tol = tols[i];
        a[i] = ai;
        smem = std::max(smem, L.total);
    }
    CK(cudaMemcpyAsync(b->args.p, a.data(), count * sizeof(pg::PcgArgs), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(b->abort_flag.p, 0, sizeof(int), st));
    CK(cudaMemsetAsync(b->claim_failures.p, 0, sizeof(int), st));
    CK(cudaMemsetAsync(b->times.p, 0, b->times.n * sizeof(unsigned long long), st));
    const unsigned long long claim_timeout_ns = (unsigned long long)(o.wait_timeout_ms * 1e6);
    const bool mixed = o.precision == PG_PREC_MIXED;
    auto kernel_of = [&](int kind) {
        if (kind == 4)
            return mixed ? (const void*)pg::pcg_batch_kernel<4, float, true>
                         : (const void*)pg::pcg_batch_kernel<4, double, false>;
        return mixed ? (const void*)pg::pcg_batch_kernel<3, float, true>
                     : (const void*)pg::pcg_batch_kernel<3, double, false>;
    };
    int grid_max = 0;
    for (auto& ph : b->phases) grid_max = std::max(grid_max, ph->grid);
    if (b->ok_precision != (mixed ? 1 : 2) || b->ok_smem != smem) {
        for (int kind : {3, 4}) {
            const void* fk = kernel_of(kind);
            opt_in_smem(c, fk);
            int nb = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fk, pg::kBatchThreads, smem));
            if (nb < 1 || nb * c->sms < grid_max)
                throw Fail{PG_EUNSUPPORTED, "batch grid does not fit on the device"};
        }
        b->ok_precision = mixed ? 1 : 2;  // residency checked for this precision and size
        b->ok_smem = smem;
    }
    // one persistent launch per phase, back to back (each after zeroing its
    // queue counters and claim slots), captured once per batch (and
    // precision / shared-memory size / time limit) into a CUDA graph
    auto launch_phases = [&](cudaStream_t s) -> cudaError_t {
        for (auto& ph : b->phases) {
            const void* fn = kernel_of(ph->kind);
            cudaError_t e = cudaMemsetAsync(ph->class_next.p, 0, ph->class_next.n * sizeof(int), s);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(ph->claims.p, 0, ph->claims.n * sizeof(unsigned long long), s);
            if (e != cudaSuccess) return e;
            pg::BatchArgs ba{b->args.p,          ph->block_team.p,
                             ph->team_base.p,    ph->team_class.p,
                             ph->class_off.p,    ph->class_queue.p,
                             ph->log_off.p,      ph->class_next.p,
                             ph->claims.p,       b->times.p,
                             b->abort_flag.p,    b->claim_failures.p,
                             claim_timeout_ns};
            void* args[] = {&ba};
            e = cudaLaunchCooperativeKernel(fn, dim3(ph->grid), dim3(pg::kBatchThreads), args, smem, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    const int prec_key = mixed ? 1 : 2;
    if (!b->graph_failed && (!b->graph || b->graph_precision != prec_key || b->graph_smem != smem ||
                             b->graph_timeout_ns != claim_timeout_ns)) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t el = launch_phases(st);
            e = cudaStreamEndCapture(st, &g);
            if (el != cudaSuccess) e = el;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b->graph = nullptr;
            b->graph_failed = true;
        }
        b->graph_precision = prec_key;
        b->graph_smem = smem;
        b->graph_timeout_ns = claim_timeout_ns;
    }
    if (b->graph)
        CK(cudaGraphLaunch(b->graph, st));
    else
        CK(launch_phases(st));
    CK(cudaEventRecord(c->ev[2], st));
    if (x_out)
        for (int i = 0; i < count; i++)
            if (x_out[i])
                CK(cudaMemcpyAsync(x_out[i], b->plans[i]->x.p, 3 * (size_t)b->plans[i]->hp.Nn * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
    std::vector<pg::PcgResult> r(count);
    std::vector<unsigned long long> tm(2 * (size_t)count);
    CK(cudaMemcpyAsync(r.data(), b->res.p, count * sizeof(pg::PcgResult), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(tm.data(), b->times.p, tm.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    int claim_failures = 0;
    CK(cudaMemcpyAsync(&claim_failures, b->claim_failures.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (claim_failures)
        throw Fail{PG_ETIMEOUT, "a batch team's wait for its next plate ran out of time"};
    float ms_setup = 0, ms_solve = 0;
    CK(cudaEventElapsedTime(&ms_setup, c->ev[0], c->ev[1]));
    CK(cudaEventElapsedTime(&ms_solve, c->ev[1], c->ev[2]));
    std::vector<double> plate_ms(count);
    int converged = 0;
    for (int i = 0; i < count; i++) {
        finish_launch(b->plans[i].get(), r[i]);
        plate_ms[i] = tm[2 * i + 1] > tm[2 * i] ? (double)(tm[2 * i + 1] - tm[2 * i]) * 1e-6 : 0.0;
        converged += r[i].converged ? 1 : 0;
        if (infos) {
            std::memset(&infos[i], 0, sizeof(pg_info));
            fill_info(&infos[i], r[i], b->plans[i].get(), plate_options(o, b->plans[i].get()),
                      pg::kBatchThreads, a[i].L.total);
            infos[i].status = r[i].status;
            infos[i].solve_ms = plate_ms[i];
            infos[i].plan_cached = 1;
        }
    }
    if (bi) {
        bi->count = count;
        int teams = 0;
        for (const pg::BatchPhase& P : b->sched.phases) teams += (int)P.team_size.size();
        bi->teams = teams;
        bi->grid = grid_max;
        bi->phases = (int32_t)b->sched.phases.size();
        bi->converged = converged;
        bi->setup_ms = ms_setup;
        bi->solve_ms = ms_solve;
        bi->plate_ms_p50 = percentile(plate_ms, 0.50);
        bi->plate_ms_p99 = percentile(plate_ms, 0.99);
        bi->plate_ms_max = percentile(plate_ms, 1.0);
        bi->solves_per_s = ms_solve > 0 ? count / (ms_solve * 1e-3) : 0.0;
        bi->shared_bytes = smem;
        bi->graph = b->graph != nullptr;
    }
    for (int i = 0; i < count; i++) throw_on_failure(r[i]);
    // plates whose mixed solve stagnated: an FP64 correction K d = F - K x_m
    // for each, solved as a batch of their own (planned for FP64
    // shared-memory capacity, kept while the same plates stagnate), each with
    // its stop scaled to the residual its x_m reached; then x = x_m + d
    if (o.precision != PG_PREC_MIXED || !o.fallback) return;
    std::vector<int> failed;
    for (int i = 0; i < count; i++)
        if (r[i].stop_reason == PG_STOP_STAGNATED) failed.push_back(i);
    if (bi) bi->fallbacks = (int32_t)failed.size();
    if (failed.empty()) return;
    pg_options o64 = o;
    o64.precision = PG_PREC_FP64;
    o64.stop_rule = PG_STOP_RELATIVE;
    const int nf = (int)failed.size();
    std::vector<std::vector<float>> rh(nf);
    std::vector<const float*> Ff(nf);
    std::vector<double> tols_f(nf);
    for (int k = 0; k < nf; k++) {
        Plan* pl = b->plans[failed[k]].get();
        const size_t n = 3 * (size_t)pl->hp.Nn;
        const int ni = (int)n;
        if (pl->kx.n != n) pl->kx.alloc(n);
        if (pl->rf.n != n) pl->rf.alloc(n);
        queue_apply_k(c, pl, pl->x.p, pl->kx.p);
        pg::residual_f32_kernel<<<(ni + 255) / 256, 256, 0, st>>>(ni, pl->cons.p, pl->F.p, pl->kx.p, pl->rf.p);
        CK(cudaGetLastError());
        rh[k].resize(n);
        CK(cudaMemcpyAsync(rh[k].data(), pl->rf.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
        Ff[k] = rh[k].data();
        tols_f[k] = correction_tolerance(o, r[failed[k]].b_norm, r[failed[k]].final_residual);
    }
    CK(cudaStreamSynchronize(st));
    if (!b->fb || b->fb_ids != failed) {
        std::vector<pg_problem> fp(nf);
        for (int k = 0; k < nf; k++) {
            fp[k] = b->plans[failed[k]]->prob_view;
            fp[k].F = Ff[k];
        }
        b->fb.reset();
        b->fb = build_batch(c, fp.data(), nf, o64);
        b->fb_ids = failed;
    }
    std::vector<std::vector<double>> d(nf);
    std::vector<double*> xf(nf, nullptr);
    for (int k = 0; k < nf; k++) {
        d[k].resize(3 * (size_t)b->plans[failed[k]]->hp.Nn);
        xf[k] = d[k].data();
    }
    std::vector<pg_info> inf(nf);
    pg_batch_info fbi{};
    run_batch(b->fb.get(), o64, Ff.data(), xf.data(), inf.data(), &fbi, tols_f.data());
    // x = x_m + d on each plate's plan, and the true residual of that x
    std::vector<double> nrm(2 * (size_t)nf, 0.0);
    for (int k = 0; k < nf; k++) {
        const int i = failed[k];
        Plan* pl = b->plans[i].get();
        const size_t n = d[k].size();
        const int ni = (int)n;
        if (pl->xw.n != n) pl->xw.alloc(n);
        CK(cudaMemcpyAsync(pl->xw.p, d[k].data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        pg::add_kernel<<<(ni + 255) / 256, 256, 0, st>>>(ni, pl->xw.p, pl->x.p);
        CK(cudaGetLastError());
        queue_true_residual(c, pl, pl->x.p, pl->F.p);
        CK(cudaMemcpyAsync(nrm.data() + 2 * k, pl->nrm.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (x_out && x_out[i])
            CK(cudaMemcpyAsync(x_out[i], pl->x.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));  // d[k] and the pageable x_out[i] are host memory
    }
    for (int k = 0; k < nf; k++) {
        const int i = failed[k];
        if (infos) {
            const double mixed_ms = infos[i].solve_ms, bn = r[i].b_norm;
            infos[i] = inf[k];
            infos[i].true_rel_residual = nrm[2 * k + 1] > 0 ? std::sqrt(nrm[2 * k] / nrm[2 * k + 1]) : 0.0;
            infos[i].b_norm = bn;
            infos[i].fallback = 1;
            infos[i].solve_ms += mixed_ms;
        }
        if (inf[k].converged) converged++;
    }
    if (bi) {
        bi->converged = converged;
        bi->solve_ms += fbi.setup_ms + fbi.solve_ms;
        bi->solves_per_s = bi->solve_ms > 0 ? count / (bi->solve_ms * 1e-3) : 0.0;
    }
}

// Queues the two moment kernels of plan pl: x_dev [3 Nn] -> M_dev [3][Nn].
void run_moments(pg_ctx* c, Plan* pl, const double* x_dev, double* M_dev) {
    const pg::HostPlan& hp = pl->hp;
    if (hp.Ne == 0 || hp.Nn == 0) return;
    DevBuf<double4> em;
    em.alloc(hp.Ne);
    const double D = (pl->E * std::pow(pl->t, 3.0)) / (12.0 * (1.0 - std::pow(pl->nu, 2.0)));
    if (hp.npe == 4)
        pg::elem_moments_kernel<4><<<(hp.Ne + 127) / 128, 128, 0, c->stream>>>(
            hp.Ne, pl->mesh_nodes.p, pl->mesh_elements.p, D, pl->nu, x_dev, em.p);
    else
        pg::elem_moments_kernel<3><<<(hp.Ne + 127) / 128, 128, 0, c->stream>>>(
            hp.Ne, pl->mesh_nodes.p, pl->mesh_elements.p, D, pl->nu, x_dev, em.p);
    CK(cudaGetLastError());
    pg::node_moments_kernel<<<(hp.Nn + 127) / 128, 128, 0, c->stream>>>(hp.Nn, pl->inc_ptr.p, pl->inc_idx.p,
                                                                       em.p, M_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));  // em is released on return
}

}  // namespace

namespace pgi {

std::mutex& ctx_mutex(pg_ctx* c) { return c->mu; }
int ctx_device(const pg_ctx* c) { return c->device; }
int ctx_sms(const pg_ctx* c) { return c->sms; }
cudaStream_t ctx_stream(const pg_ctx* c) { return c->stream; }
void ctx_set_error(pg_ctx* c, const std::string& msg) { c->err = msg; }
pg_ctx* plan_ctx(const pg_plan* h) { return h ? h->ctx : nullptr; }

std::string plan_operator(pg_plan* h, OperatorView* out) {
    try {
        Plan* pl = h->plan.get();
        run_setup(h->ctx, pl);
        *out = operator_view(pl);
        return std::string();
    } catch (const Fail& f) {
        return f.msg;
    }
}

double plan_lambda_max(pg_plan* h) {
    Plan* pl = h->plan.get();
    try {
        if (!(pl->lambda_max > 0)) pl->lambda_max = device_lambda_max(h->ctx, pl, 30);
    } catch (const Fail&) {
        return 2.0;
    }
    return pl->lambda_max;
}

}  // namespace pgi

extern "C" {

void pg_options_default(pg_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(pg_options);
    o->tolerance = 1e-6;
    o->max_iterations = 1000;
    o->precision = PG_PREC_FP64;
    o->stop_rule = PG_STOP_REFERENCE;
    o->wait_timeout_ms = 1000.0;
    o->fallback = 1;
}

int pg_is_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < n; d++) {
        cudaDeviceProp pr;
        if (cudaGetDeviceProperties(&pr, d) == cudaSuccess && pr.major == 10) return 1;
    }
    return 0;
}

int pg_create(int device, pg_ctx** out) {
    if (!out) return PG_EINVAL;
    *out = nullptr;
    auto c = std::make_unique<pg_ctx>();
    c->device = device;
    try {
        int n = 0;
        CK(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Fail{PG_EINVAL, "no such CUDA device"};
        CK(cudaSetDevice(device));
        cudaDeviceProp pr;
        CK(cudaGetDeviceProperties(&pr, device));
        if (pr.major != 10)
            throw Fail{PG_ECUDA, "this build targets sm_100a (B200); device is sm_" +
                                     std::to_string(pr.major) + std::to_string(pr.minor)};
        if (!pr.cooperativeLaunch) throw Fail{PG_ECUDA, "device lacks cooperative launch"};
        c->sms = pr.multiProcessorCount;
        c->max_smem = (int)pr.sharedMemPerBlockOptin;
        int khz = 0;
        CK(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device));
        c->clock_khz = khz > 0 ? khz : 1.0;
        CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
        c->stream = c->own_stream;
        for (auto& e : c->ev) CK(cudaEventCreate(&e));
    } catch (const Fail& f) {
        g_create_error = f.msg;
        cudaGetLastError();
        return f.status;
    }
    *out = c.release();
    return PG_OK;
}

void pg_destroy(pg_ctx* c) {
    if (!c) return;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        if (c->stream) cudaStreamSynchronize(c->stream);
        c->plans.clear();
        for (auto& e : c->ev)
            if (e) cudaEventDestroy(e);
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        if (c->hF) cudaFreeHost(c->hF);
        if (c->hx) cudaFreeHost(c->hx);
    }
    delete c;
}

const char* pg_last_error(const pg_ctx* c) {
    return c ? c->err.c_str() : g_create_error.c_str();
}

int pg_clear_cache(pg_ctx* c) {
    return guarded(c, nullptr, [&] {
        CK(cudaStreamSynchronize(c->stream));
        c->plans.clear();
    });
}

int pg_set_stream(pg_ctx* c, void* stream) {
    return guarded(c, nullptr, [&] {
        CK(cudaStreamSynchronize(c->stream));
        c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    });
}

int pg_solve(pg_ctx* c, const pg_problem* p, const pg_options* opt, double* x_out, pg_info* info) {
    zero_info(info);
    return guarded(c, info, [&] {
        check_problem(p, true);
        pg_options o;
        fill_options(opt, &o);
        const size_t n = 3 * (size_t)p->node_count;
        if (n && !x_out) throw Fail{PG_EINVAL, "x_out is NULL"};
        for (size_t i = 0; i < n; i++)
            if (!std::isfinite(p->F[i])) throw Fail{PG_ENONFINITE, "F contains NaN or Inf"};
        if (n == 0) {
            if (info) { info->converged = 1; info->stop_reason = PG_STOP_ZERO_RHS; }
            return;
        }
        const int G = o.ctas ? std::min(o.ctas, (int)p->node_count) : auto_ctas(c, (int)p->node_count);
        bool cached = false;
        const auto tp = std::chrono::steady_clock::now();
        Plan* pl = get_plan(c, *p, G, halo_rings(o), &cached);
        const double plan_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count();
        ensure_staging(c, n);
        std::memcpy(c->hF, p->F, n * sizeof(float));
        CK(cudaMemcpyAsync(pl->F.p, c->hF, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        solve_with_fallback(c, pl, o, info, c->hx, cudaMemcpyDeviceToHost);
        std::memcpy(x_out, c->hx, n * sizeof(double));
        if (info) {
            info->plan_cached = cached ? 1 : 0;
            info->plan_ms = cached ? 0.0 : plan_ms;
        }
    });
}

int pg_solve_load_cases(pg_ctx* c, const pg_problem* p, int count, const float* F, const pg_options* opt,
                        int cases_per_launch, double* x_out, pg_info* infos) {
    if (infos && count > 0) std::memset(infos, 0, (size_t)count * sizeof(pg_info));
    return guarded(c, nullptr, [&] {
        check_problem(p, false);
        if (count < 1 || !F) throw Fail{PG_EINVAL, "need count >= 1 load cases and F"};
        if (cases_per_launch != 0 && cases_per_launch != 1 && cases_per_launch != 2 && cases_per_launch != 4)
            throw Fail{PG_EINVAL, "cases_per_launch must be 0 (automatic), 1, 2 or 4"};
        pg_options o;
        fill_options(opt, &o);
        const size_t n = 3 * (size_t)p->node_count;
        if (n && !x_out) throw Fail{PG_EINVAL, "x_out is NULL"};
        for (size_t i = 0; i < n * count; i++)
            if (!std::isfinite(F[i])) throw Fail{PG_ENONFINITE, "F contains NaN or Inf"};
        if (n == 0) {
            if (infos)
                for (int k = 0; k < count; k++) { infos[k].converged = 1; infos[k].stop_reason = PG_STOP_ZERO_RHS; }
            return;
        }
        const int G = o.ctas ? std::min(o.ctas, (int)p->node_count) : auto_ctas(c, (int)p->node_count);
        bool cached = false;
        Plan* pl = get_plan(c, *p, G, halo_rings(o), &cached);
        prepare_plan_data(c, pl, o);
        // group width: automatic = the widest whose layout keeps the Ke
        // blocks in shared memory, else the widest that fits.  Ke blocks read
        // from L2 by every block twice per iteration cost more than a wider
        // group saves (60k-DOF plate, mixed two-level Chebyshev: four cases
        // per launch with Ke in L2 1.64 ms per case, two with Ke in shared
        // memory 1.35, one 1.71)
        auto fits = [&](int NR, int* km = nullptr) {
            int m = 0;
            bool ai = false;
            pg::SmemLayout L{};
            const bool ok = choose_layout_multi(c, pl->hp, o, NR, &m, &ai, &L);
            if (km) *km = m;
            return ok;
        };
        int W = cases_per_launch;
        if (W == 0) {
            int km4 = 0, km2 = 0;
            const bool f4 = fits(4, &km4), f2 = fits(2, &km2);
            W = (f4 && km4 > 0) ? 4 : (f2 && km2 > 0) ? 2 : f4 ? 4 : f2 ? 2 : 1;
        }
        else if (W > 1 && !fits(W)) throw Fail{PG_EUNSUPPORTED, "load-case partition too large for shared memory"};
        for (int k0 = 0; k0 < count;) {
            const int m = std::min(W, count - k0);
            std::vector<const float*> Fk(m);
            std::vector<double*> xk(m);
            for (int k = 0; k < m; k++) {
                Fk[k] = F + (size_t)(k0 + k) * n;
                xk[k] = x_out + (size_t)(k0 + k) * n;
            }
            pg_info* ik = infos ? infos + k0 : nullptr;
            if (m == 1) {
                ensure_staging(c, n);
                std::memcpy(c->hF, Fk[0], n * sizeof(float));
                CK(cudaMemcpyAsync(pl->F.p, c->hF, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
                solve_with_fallback(c, pl, o, ik, c->hx, cudaMemcpyDeviceToHost);
                std::memcpy(xk[0], c->hx, n * sizeof(double));
            } else {
                run_solve_multi(c, pl, o, (m == 2 && (W == 2 || fits(2))) ? 2 : W, m, Fk.data(), xk.data(), ik);
            }
            if (ik)
                for (int k = 0; k < m; k++) ik[k].plan_cached = (cached || k0 > 0) ? 1 : 0;
            k0 += m;
        }
    });
}

int pg_plan_create(pg_ctx* c, const pg_problem* p, const pg_options* opt, pg_plan** out) {
    if (out) *out = nullptr;
    return guarded(c, nullptr, [&] {
        if (!out) throw Fail{PG_EINVAL, "out is NULL"};
        check_problem(p, false);
        if (p->node_count == 0) throw Fail{PG_EINVAL, "empty mesh: nothing to plan"};
        pg_options o;
        fill_options(opt, &o);
        const int G = o.ctas ? std::min(o.ctas, (int)p->node_count) : auto_ctas(c, (int)p->node_count);
        auto h = std::make_unique<pg_plan>();
        h->ctx = c;
        h->plan = build_plan(c, *p, G, halo_rings(o));
        *out = h.release();
    });
}

int pg_plan_solve_device(pg_plan* h, const pg_options* opt, const float* F_dev, double* x_dev,
                         pg_info* info) {
    zero_info(info);
    if (!h) return PG_EINVAL;
    pg_ctx* c = h->ctx;
    return guarded(c, info, [&] {
        pg_options o;
        fill_options(opt, &o);
        if (!F_dev || !x_dev) throw Fail{PG_EINVAL, "F_dev / x_dev is NULL"};
        Plan* pl = h->plan.get();
        const size_t n = 3 * (size_t)pl->hp.Nn;
        CK(cudaMemcpyAsync(pl->F.p, F_dev, n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
        solve_with_fallback(c, pl, o, info, x_dev, cudaMemcpyDeviceToDevice);
        if (info) info->plan_cached = 1;
    });
}

void pg_plan_destroy(pg_plan* h) {
    if (!h) return;
    {
        std::lock_guard<std::mutex> lk(h->ctx->mu);
        cudaSetDevice(h->ctx->device);
        cudaStreamSynchronize(h->ctx->stream);
        h->plan.reset();
    }
    delete h;
}

int pg_apply_k(pg_ctx* c, const pg_problem* p, const double* x, double* y) {
    return guarded(c, nullptr, [&] {
        check_problem(p, false);
        const size_t n = 3 * (size_t)p->node_count;
        if (n == 0) return;
        if (!x || !y) throw Fail{PG_EINVAL, "x / y is NULL"};
        bool cached = false;
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), 1, &cached);
        run_setup(c, pl);
        DevBuf<double> dx, dy;
        dx.upload(x, n, c->stream);
        dy.alloc(n);
        queue_apply_k(c, pl, dx.p, dy.p);
        CK(cudaMemcpyAsync(y, dy.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int pg_block_jacobi(pg_ctx* c, const pg_problem* p, double* binv_out) {
    return guarded(c, nullptr, [&] {
        check_problem(p, false);
        if (p->node_count == 0) return;
        if (!binv_out) throw Fail{PG_EINVAL, "binv_out is NULL"};
        bool cached = false;
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), 1, &cached);
        run_setup(c, pl);
        CK(cudaMemcpyAsync(binv_out, pl->binv64.p, 9 * sizeof(double) * p->node_count,
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int pg_element_stiffness(pg_ctx* c, const pg_problem* p, double* ke_out) {
    return guarded(c, nullptr, [&] {
        check_problem(p, false);
        if (p->element_count == 0 || p->node_count == 0) return;
        if (!ke_out) throw Fail{PG_EINVAL, "ke_out is NULL"};
        bool cached = false;
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), 1, &cached);
        run_setup(c, pl);
        const size_t kk = 9 * (size_t)p->nodes_per_element * p->nodes_per_element;
        CK(cudaMemcpyAsync(ke_out, pl->ke64.p, kk * sizeof(double) * p->element_count,
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int pg_plan_inspect(const pg_problem* p, int ctas, int32_t* stats, char* msg, size_t msg_len) {
    return pg_plan_inspect_halo(p, ctas, 1, stats, msg, msg_len);
}

int pg_plan_inspect_halo(const pg_problem* p, int ctas, int rings, int32_t* stats, char* msg,
                         size_t msg_len) {
    auto put = [&](const std::string& m) {
        if (msg && msg_len) {
            std::strncpy(msg, m.c_str(), msg_len - 1);
            msg[msg_len - 1] = 0;
        }
    };
    if (!p || !stats) { put("problem / stats_out is NULL"); return PG_EINVAL; }
    try {
        std::string e = pg::validate_problem(*p, false);
        if (!e.empty()) { put(e); return PG_EINVAL; }
        pg::HostPlan hp;
        e = pg::build_structure(*p, hp);
        if (rings != 1 && rings != 2) e = "rings must be 1 or 2";
        if (e.empty()) e = pg::build_partition(*p, ctas > 0 ? ctas : 1, rings, hp);
        if (!e.empty()) { put(e); return PG_EINVAL; }
        const int Nn = hp.Nn, npe = hp.npe, C = hp.colors;
        int bad = 0;
        std::vector<int> owner(Nn, -1);
        long ghosts = 0;
        for (int g = 0; g < hp.G; g++) {
            const int n0 = hp.node_off[g], no = hp.nown[g], nl = hp.node_off[g + 1] - n0;
            ghosts += nl - no;
            for (int k = 0; k < no; k++) {
                if (owner[hp.nodes[n0 + k]] >= 0) bad++;
                owner[hp.nodes[n0 + k]] = g;
            }
            // tasks of node k < n1 (owned, and ring 1 with rings = 2): exactly
            // its incidences, in order, the node itself first
            const int t0 = hp.task_off[g], m1 = hp.n1[g];
            const int* tp = hp.tptr.data() + hp.tp_off[g];
            if (m1 < no || m1 > nl || (rings == 1 && m1 != no)) bad++;
            if (hp.tp_off[g + 1] - hp.tp_off[g] != m1 + 1 || tp[0] != 0 ||
                tp[m1] != hp.task_off[g + 1] - t0)
                bad++;
            std::vector<char> used(nl, 0);
            for (int k = 0; k < m1; k++) {
                const int n = hp.nodes[n0 + k];
                used[k] = 1;
                if (tp[k + 1] - tp[k] != hp.inc_ptr[n + 1] - hp.inc_ptr[n]) { bad++; continue; }
                for (int i = 0; i < tp[k + 1] - tp[k]; i++) {
                    const int t = t0 + tp[k] + i, inc = hp.inc_idx[hp.inc_ptr[n] + i];
                    const int e = inc / 4, pos = inc % 4;
                    if (hp.task_elem[t] != e || hp.task_pos[t] != pos) bad++;
                    for (int j = 0; j < npe; j++) {
                        const int ln = hp.task_nodes[(size_t)t * npe + j];
                        if (ln >= nl || hp.nodes[n0 + ln] != (int)p->elements[(size_t)e * npe + (pos + j) % npe])
                            bad++;
                        else
                            used[ln] = 1;
                    }
                    if (hp.task_nodes[(size_t)t * npe] != k) bad++;
                }
            }
            for (int k = no; k < nl; k++)  // ghosts: referenced, and not owned here
                if (!used[k]) bad++;
        }
        for (int n = 0; n < Nn; n++)
            if (owner[n] < 0) bad++;
        for (int g = 0; g < hp.G; g++)
            for (int k = hp.nown[g]; k < hp.node_off[g + 1] - hp.node_off[g]; k++)
                if (owner[hp.nodes[hp.node_off[g] + k]] == g) bad++;
        // colour validity of the colouring in use
        std::vector<int> col(hp.Ne, -1), stamp(C, -1);
        for (int c = 0; c < C; c++)
            for (uint32_t q = hp.color_offsets[c]; q < hp.color_offsets[c + 1]; q++) col[hp.elements_by_color[q]] = c;
        for (int n = 0; n < Nn; n++)
            for (int q = hp.inc_ptr[n]; q < hp.inc_ptr[n + 1]; q++) {
                const int c = col[hp.inc_idx[q] / 4];
                if (stamp[c] == n) bad++;
                stamp[c] = n;
            }
        stats[0] = hp.G;
        stats[1] = C;
        stats[2] = hp.recolored ? 1 : 0;
        stats[3] = hp.max_nloc;
        stats[4] = hp.max_nown;
        stats[5] = hp.max_ntask;
        stats[6] = (int32_t)ghosts;
        stats[7] = bad;
        put(bad ? "plan invariants violated" : "");
        return PG_OK;
    } catch (const std::bad_alloc&) {
        put("host allocation failed");
        return PG_ENOMEM;
    } catch (...) {
        put("internal error");
        return PG_ECUDA;
    }
}

int pg_batch_create(pg_ctx* c, const pg_problem* probs, int count, const pg_options* opt,
                    pg_batch** out) {
    if (out) *out = nullptr;
    return guarded(c, nullptr, [&] {
        if (!out) throw Fail{PG_EINVAL, "out is NULL"};
        if (!probs || count < 1) throw Fail{PG_EINVAL, "the batch needs at least one problem"};
        pg_options o;
        fill_options(opt, &o);
        *out = build_batch(c, probs, count, o).release();
    });
}

int pg_batch_solve(pg_batch* b, const pg_options* opt, const float* const* F, double* const* x_out,
                   pg_info* infos, pg_batch_info* bi) {
    if (bi) std::memset(bi, 0, sizeof(*bi));
    if (!b) return PG_EINVAL;
    pg_ctx* c = b->ctx;
    auto t0 = std::chrono::steady_clock::now();
    const int st = guarded(c, nullptr, [&] {
        pg_options o;
        fill_options(opt, &o);
        run_batch(b, o, F, x_out, infos, bi);
    });
    if (bi) {
        bi->status = st;
        bi->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

void pg_batch_destroy(pg_batch* b) {
    if (!b) return;
    {
        std::lock_guard<std::mutex> lk(b->ctx->mu);
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
        b->fb.reset();
        b->plans.clear();
        b->phases.clear();
        b->abort_flag.release();
        b->args.release();
        b->res.release();
        b->times.release();
    }
    delete b;
}

int pg_solve_batch(pg_ctx* c, const pg_problem* probs, int count, const pg_options* opt,
                   double* const* x_out, pg_info* infos, pg_batch_info* bi) {
    if (bi) std::memset(bi, 0, sizeof(*bi));
    pg_batch* b = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    int st = pg_batch_create(c, probs, count, opt, &b);
    if (st == PG_OK) st = pg_batch_solve(b, opt, nullptr, x_out, infos, bi);
    pg_batch_destroy(b);
    if (bi) {
        bi->status = st;
        bi->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return st;
}

int pg_batch_schedule(const uint32_t* node_counts, int count, int sms, int cap, int32_t* plate_phase,
                      int32_t* plate_size, int32_t* plate_team, int32_t* phase_grid,
                      int32_t* phases_out) {
    if (!node_counts || count < 1 || !plate_phase || !plate_size || !plate_team || !phase_grid ||
        !phases_out)
        return PG_EINVAL;
    try {
        std::vector<int> nodes(node_counts, node_counts + count);
        pg::BatchSchedule S;
        if (!pg::schedule_batch(nodes, std::vector<int>(count, cap), std::vector<int>(count, 4), sms, S).empty())
            return PG_EUNSUPPORTED;
        for (int i = 0; i < count; i++) {
            plate_phase[i] = S.plate_phase[i];
            plate_size[i] = S.plate_size[i];
            plate_team[i] = S.plate_team[i];
        }
        for (size_t k = 0; k < S.phases.size(); k++) phase_grid[k] = S.phases[k].grid;
        *phases_out = (int32_t)S.phases.size();
        return PG_OK;
    } catch (...) {
        return PG_ENOMEM;
    }
}

int pg_partition_nodes(const float* nodes, uint32_t node_count, int ctas, int32_t* part_of) {
    if (node_count == 0) return PG_OK;
    if (!nodes || !part_of || ctas < 1 || node_count > (uint32_t)INT32_MAX) return PG_EINVAL;
    for (size_t i = 0; i < 2 * (size_t)node_count; i++)
        if (!std::isfinite(nodes[i])) return PG_EINVAL;
    try {
        const int Nn = (int)node_count;
        std::vector<int> part;
        pg::strip_partition(nodes, Nn, std::min(ctas, Nn), part);
        for (int n = 0; n < Nn; n++) part_of[n] = part[n];
        return PG_OK;
    } catch (...) {
        return PG_ENOMEM;
    }
}

int pg_moments(pg_ctx* c, const pg_problem* p, const double* x, double* Mx, double* My,
                          double* Mxy) {
    return guarded(c, nullptr, [&] {
        check_problem(p, false);
        const size_t Nn = p->node_count;
        if (Nn == 0) return;
        if (!x || !Mx || !My || !Mxy) throw Fail{PG_EINVAL, "x / Mx / My / Mxy is NULL"};
        bool cached = false;
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)Nn), 1, &cached);
        DevBuf<double> dx, dm;
        dx.upload(x, 3 * Nn, c->stream);
        dm.alloc(3 * Nn);
        run_moments(c, pl, dx.p, dm.p);
        std::vector<double> h(3 * Nn);
        CK(cudaMemcpy(h.data(), dm.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        std::memcpy(Mx, h.data(), Nn * sizeof(double));
        std::memcpy(My, h.data() + Nn, Nn * sizeof(double));
        std::memcpy(Mxy, h.data() + 2 * Nn, Nn * sizeof(double));
    });
}

int pg_plan_moments_device(pg_plan* h, const double* x_dev, double* M_dev) {
    if (!h) return PG_EINVAL;
    return guarded(h->ctx, nullptr, [&] {
        if (!x_dev || !M_dev) throw Fail{PG_EINVAL, "x_dev / M_dev is NULL"};
        run_moments(h->ctx, h->plan.get(), x_dev, M_dev);
    });
}

}  // extern "C"
