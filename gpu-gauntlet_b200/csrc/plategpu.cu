// C ABI of the plate solver (include/plategpu.h): context, plan cache,
// uploads, kernel launches.  No exception crosses the ABI; every failure
// becomes a pg_status plus a message for pg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
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

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) CK(cudaMalloc(&p, count * sizeof(T)));
    }
    void upload(const T* h, size_t count, cudaStream_t st) {
        alloc(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

struct Plan {
    uint64_t key = 0;
    int G = 0;
    pg::HostPlan hp;
    double E = 0, nu = 0, t = 0;
    bool has_elem_t = false;
    DevBuf<int> node_off, nown, nodes, elem_off, color_off, elems, lnode, inc_ptr, inc_idx;
    DevBuf<float> mesh_nodes, elem_t, F;
    DevBuf<uint32_t> mesh_elements, cob_off, cob_list;
    DevBuf<uint8_t> cons;
    DevBuf<double> ke64, binv64, x, xch64, partials;
    DevBuf<float> ke32, binv32, xch32;
    DevBuf<unsigned int> bar;
    DevBuf<int> abort_flag;
    DevBuf<pg::PcgResult> res;
};

}  // namespace

struct pg_plan {
    pg_ctx* ctx = nullptr;
    std::unique_ptr<Plan> plan;
};

struct pg_ctx {
    int device = 0;
    int sms = 0;
    int max_smem = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::mutex mu;
    std::string err;
    std::list<std::unique_ptr<Plan>> plans;  // most recently used first
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

size_t smem_bytes(const pg::HostPlan& hp, bool ke_smem) {
    const int nd = 3 * hp.npe, ns = nd * (nd + 1) / 2;
    size_t dbl = 15 * (size_t)hp.max_nloc + 3 * (size_t)hp.max_nown + 9 * (size_t)hp.max_nloc + 32 * 4 +
                 8 + (ke_smem ? (size_t)hp.max_nel * ns : 0);
    size_t ints = (size_t)hp.npe * hp.max_nel + (hp.colors + 1) + 4;
    size_t bytes = 3 * (size_t)hp.max_nloc;
    return dbl * 8 + ints * 4 + bytes + 16;
}

std::unique_ptr<Plan> build_plan(pg_ctx* c, const pg_problem& p, int G) {
    auto pl = std::make_unique<Plan>();
    std::string e = pg::build_structure(p, pl->hp);
    if (e.empty()) e = pg::build_partition(p, G, pl->hp);
    if (!e.empty()) throw Fail{PG_EINVAL, e};
    pl->G = pl->hp.G;
    pl->E = p.E;
    pl->nu = p.nu;
    pl->t = p.t;
    const pg::HostPlan& hp = pl->hp;
    cudaStream_t st = c->stream;
    const size_t Nn = p.node_count, Ne = p.element_count, npe = p.nodes_per_element;
    const size_t kk = 9 * npe * npe;
    pl->node_off.upload(hp.node_off.data(), hp.node_off.size(), st);
    pl->nown.upload(hp.nown.data(), hp.nown.size(), st);
    pl->nodes.upload(hp.nodes.data(), hp.nodes.size(), st);
    pl->elem_off.upload(hp.elem_off.data(), hp.elem_off.size(), st);
    pl->color_off.upload(hp.color_off.data(), hp.color_off.size(), st);
    pl->elems.upload(hp.elems.data(), hp.elems.size(), st);
    pl->lnode.upload(hp.lnode.data(), hp.lnode.size(), st);
    pl->inc_ptr.upload(hp.inc_ptr.data(), hp.inc_ptr.size(), st);
    pl->inc_idx.upload(hp.inc_idx.data(), hp.inc_idx.size(), st);
    pl->mesh_nodes.upload(p.nodes, 2 * Nn, st);
    pl->mesh_elements.upload(p.elements, npe * Ne, st);
    pl->cob_off.upload(hp.color_offsets.data(), hp.color_offsets.size(), st);
    pl->cob_list.upload(hp.elements_by_color.data(), hp.elements_by_color.size(), st);
    pl->cons.upload(p.constrained, 3 * Nn, st);
    pl->has_elem_t = p.elem_t != nullptr;
    if (p.elem_t) pl->elem_t.upload(p.elem_t, Ne, st);
    pl->F.alloc(3 * Nn);
    pl->ke64.alloc(std::max<size_t>(1, Ne * kk));
    pl->ke32.alloc(std::max<size_t>(1, Ne * kk));
    pl->binv64.alloc(9 * Nn);
    pl->binv32.alloc(9 * Nn);
    pl->x.alloc(3 * Nn);
    pl->xch64.alloc(6 * Nn);
    pl->xch32.alloc(6 * Nn);
    pl->partials.alloc(8 * (size_t)pl->G);
    pl->bar.alloc(1);
    pl->abort_flag.alloc(1);
    pl->res.alloc(1);
    // synchronous: uploads read the host plan arrays
    CK(cudaStreamSynchronize(st));
    return pl;
}

Plan* get_plan(pg_ctx* c, const pg_problem& p, int G, bool* cached) {
    const uint64_t key = pg::problem_hash(p);
    for (auto it = c->plans.begin(); it != c->plans.end(); ++it) {
        if ((*it)->key == key && (*it)->G == G) {
            c->plans.splice(c->plans.begin(), c->plans, it);
            *cached = true;
            return c->plans.front().get();
        }
    }
    *cached = false;
    auto pl = build_plan(c, p, G);
    pl->key = key;
    c->plans.push_front(std::move(pl));
    while (c->plans.size() > kMaxPlans) c->plans.pop_back();
    return c->plans.front().get();
}

void run_setup(pg_ctx* c, Plan* pl) {
    const pg::HostPlan& hp = pl->hp;
    const int Ne = hp.Ne, Nn = hp.Nn;
    if (Ne > 0)
        pg::ke_kernel<<<(Ne + 127) / 128, 128, 0, c->stream>>>(
            Ne, hp.npe, pl->mesh_nodes.p, pl->mesh_elements.p, pl->E, pl->nu, pl->t,
            pl->has_elem_t ? pl->elem_t.p : nullptr, pl->ke64.p, pl->ke32.p);
    CK(cudaGetLastError());
    if (Nn > 0)
        pg::binv_kernel<<<(Nn + 127) / 128, 128, 0, c->stream>>>(
            Nn, hp.npe, pl->inc_ptr.p, pl->inc_idx.p, pl->ke64.p, pl->cons.p, pl->binv64.p,
            pl->binv32.p);
    CK(cudaGetLastError());
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
    if (o->threads < 0 || o->threads > 512 || (o->threads % 32) != 0)
        throw Fail{PG_EINVAL, "threads must be a multiple of 32 in [32, 512] (0 = automatic)"};
    if (o->ctas < 0) throw Fail{PG_EINVAL, "ctas must be >= 0"};
    if (!(o->wait_timeout_ms >= 0)) throw Fail{PG_EINVAL, "wait_timeout_ms must be >= 0"};
}

// Queues setup + persistent PCG on the context stream, then waits for the
// result record (one small readback).  F must already be in pl->F.
void run_solve(pg_ctx* c, Plan* pl, const pg_options& o, pg_info* info) {
    const pg::HostPlan& hp = pl->hp;
    if (o.precision == PG_PREC_MIXED) throw Fail{PG_EUNSUPPORTED, "mixed precision is not built yet"};
    const int threads = o.threads ? o.threads : 512;
    bool ke_smem = true;
    size_t sm = smem_bytes(hp, true);
    if (sm > (size_t)c->max_smem) {
        ke_smem = false;
        sm = smem_bytes(hp, false);
    }
    if (sm > (size_t)c->max_smem)
        throw Fail{PG_EUNSUPPORTED, "partition too large for shared memory: use more ctas"};
    if (pl->G > c->sms) throw Fail{PG_EINVAL, "ctas exceeds the number of SMs"};

    CK(cudaEventRecord(c->ev[0], c->stream));
    run_setup(c, pl);
    CK(cudaEventRecord(c->ev[1], c->stream));
    CK(cudaMemsetAsync(pl->bar.p, 0, sizeof(unsigned int), c->stream));
    CK(cudaMemsetAsync(pl->abort_flag.p, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(pl->res.p, 0, sizeof(pg::PcgResult), c->stream));

    pg::PcgArgs a{};
    a.G = pl->G;
    a.npe = hp.npe;
    a.C = hp.colors;
    a.Nn = hp.Nn;
    a.node_off = pl->node_off.p;
    a.nown = pl->nown.p;
    a.nodes = pl->nodes.p;
    a.elem_off = pl->elem_off.p;
    a.color_off = pl->color_off.p;
    a.elems = pl->elems.p;
    a.lnode = pl->lnode.p;
    a.ke64 = pl->ke64.p;
    a.ke32 = pl->ke32.p;
    a.binv64 = pl->binv64.p;
    a.binv32 = pl->binv32.p;
    a.cons = pl->cons.p;
    a.F = pl->F.p;
    a.x = pl->x.p;
    a.xch64 = pl->xch64.p;
    a.xch32 = pl->xch32.p;
    a.partials = pl->partials.p;
    a.bar = pl->bar.p;
    a.abort_flag = pl->abort_flag.p;
    a.res = pl->res.p;
    a.tol = o.tolerance;
    a.maxit = o.max_iterations;
    a.stop_rule = o.stop_rule;
    a.timeout_ns = (unsigned long long)(o.wait_timeout_ms * 1e6);
    a.ke_smem = ke_smem ? 1 : 0;
    a.sm_nloc = hp.max_nloc;
    a.sm_nown = hp.max_nown;
    a.sm_nel = hp.max_nel;
    a.reliable_interval = o.reliable_interval;
    a.reliable_delta = o.reliable_delta;

    const void* fn = hp.npe == 4 ? (const void*)pg::pcg_fp64_kernel<4> : (const void*)pg::pcg_fp64_kernel<3>;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, sm));
    if (nb < 1 || nb * c->sms < pl->G)
        throw Fail{PG_EUNSUPPORTED, "persistent grid does not fit on the device"};
    void* args[] = {&a};
    CK(cudaLaunchCooperativeKernel(fn, dim3(pl->G), dim3(threads), args, sm, c->stream));
    CK(cudaEventRecord(c->ev[2], c->stream));
    pg::PcgResult r{};
    CK(cudaMemcpyAsync(&r, pl->res.p, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float ms_setup = 0, ms_solve = 0;
    CK(cudaEventElapsedTime(&ms_setup, c->ev[0], c->ev[1]));
    CK(cudaEventElapsedTime(&ms_solve, c->ev[1], c->ev[2]));
    if (info) {
        info->iterations = r.iterations;
        info->converged = r.converged;
        info->stop_reason = r.stop_reason;
        info->final_residual = r.final_residual;
        info->true_rel_residual = r.true_rel_residual;
        info->b_norm = r.b_norm;
        info->setup_ms = ms_setup;
        info->solve_ms = ms_solve;
        info->ctas = pl->G;
        info->threads = threads;
        info->reliable_updates = r.reliable_updates;
    }
    if (r.wait_failures > 0 || r.status == PG_ETIMEOUT)
        throw Fail{PG_ETIMEOUT, "a grid-wide wait exceeded wait_timeout_ms"};
    if (r.status == PG_ENONFINITE) throw Fail{PG_ENONFINITE, "non-finite value in the PCG iteration"};
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
        Plan* pl = get_plan(c, *p, G, &cached);
        ensure_staging(c, n);
        std::memcpy(c->hF, p->F, n * sizeof(float));
        CK(cudaMemcpyAsync(pl->F.p, c->hF, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        run_solve(c, pl, o, info);
        CK(cudaMemcpyAsync(c->hx, pl->x.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        std::memcpy(x_out, c->hx, n * sizeof(double));
        if (info) info->plan_cached = cached ? 1 : 0;
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
        h->plan = build_plan(c, *p, G);
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
        run_solve(c, pl, o, info);
        CK(cudaMemcpyAsync(x_dev, pl->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
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
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), &cached);
        run_setup(c, pl);
        DevBuf<double> dx, dy;
        dx.upload(x, n, c->stream);
        dy.alloc(n);
        CK(cudaMemsetAsync(dy.p, 0, n * sizeof(double), c->stream));
        const pg::HostPlan& hp = pl->hp;
        for (int col = 0; col < hp.colors; col++) {
            const int off = (int)hp.color_offsets[col], cnt = (int)hp.color_offsets[col + 1] - off;
            if (cnt > 0)
                pg::applyk_color_kernel<<<(cnt + 127) / 128, 128, 0, c->stream>>>(
                    cnt, pl->cob_list.p + off, hp.npe, pl->mesh_elements.p, pl->ke64.p, dx.p, dy.p);
            CK(cudaGetLastError());
        }
        pg::bc_copy_kernel<<<((int)n + 255) / 256, 256, 0, c->stream>>>((int)n, pl->cons.p, dx.p, dy.p);
        CK(cudaGetLastError());
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
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), &cached);
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
        Plan* pl = get_plan(c, *p, auto_ctas(c, (int)p->node_count), &cached);
        run_setup(c, pl);
        const size_t kk = 9 * (size_t)p->nodes_per_element * p->nodes_per_element;
        CK(cudaMemcpyAsync(ke_out, pl->ke64.p, kk * sizeof(double) * p->element_count,
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int pg_plan_inspect(const pg_problem* p, int ctas, int32_t* stats, char* msg, size_t msg_len) {
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
        if (e.empty()) e = pg::build_partition(*p, ctas > 0 ? ctas : 1, hp);
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
            // elements: exactly those touching an owned node, colour-sorted
            std::vector<char> in_part(hp.Ne, 0);
            for (int q = hp.elem_off[g]; q < hp.elem_off[g + 1]; q++) in_part[hp.elems[q]] = 1;
            for (int k = 0; k < no; k++) {
                const int n = hp.nodes[n0 + k];
                for (int q = hp.inc_ptr[n]; q < hp.inc_ptr[n + 1]; q++)
                    if (!in_part[hp.inc_idx[q] / 4]) bad++;
            }
            for (int c = 0; c < C; c++) {
                for (int q = hp.color_off[(size_t)g * (C + 1) + c]; q < hp.color_off[(size_t)g * (C + 1) + c + 1]; q++) {
                    const int e = hp.elems[q];
                    bool touches = false;
                    for (int k = 0; k < npe; k++) {
                        const int ln = hp.lnode[(size_t)q * npe + k];
                        if (ln < 0 || ln >= nl || hp.nodes[n0 + ln] != (int)p->elements[(size_t)e * npe + k]) bad++;
                        if (ln >= 0 && ln < no) touches = true;
                    }
                    if (!touches) bad++;
                    bool found = false;
                    for (uint32_t q2 = hp.color_offsets[c]; q2 < hp.color_offsets[c + 1] && !found; q2++)
                        found = hp.elements_by_color[q2] == (uint32_t)e;
                    if (!found) bad++;
                }
            }
        }
        for (int n = 0; n < Nn; n++)
            if (owner[n] < 0) bad++;
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
        stats[5] = hp.max_nel;
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

}  // extern "C"
