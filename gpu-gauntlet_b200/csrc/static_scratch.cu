// pg_apply_k_static: y = K x with no device allocation.
//
// Some callers cannot call cudaMalloc: code whose device memory is owned by
// another allocator that hands out no untracked blocks (a framework's
// caching allocator or a fixed memory budget), and code that must not
// allocate once it is running (a real-time loop, a driver callback).  This
// entry point serves them: the caller passes device buffers for every input
// and output, and the one piece of scratch the operator needs -- the element
// stiffness matrices -- lives in a file-scope static device array of fixed
// size that the CUDA runtime creates when the library is loaded (every GPU
// that loads the library holds it until the process exits).
//
// The kernels are variants of ke_kernel / applyk_color_kernel /
// bc_copy_kernel of the regular pg_apply_k path: the same element formulas
// and the same colour-by-colour scatter, reading and writing the static
// scratch instead of a plan buffer.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "element.cuh"
#include "plategpu.h"

namespace {

// Scratch capacity: 2^20 doubles (8 MiB), room for the element matrices of
// 7,281 Q4 or 12,945 DKT elements.  Every element matrix a call reads is
// written earlier in the same call, so nothing needs clearing between calls.
constexpr size_t kScratchDoubles = size_t(1) << 20;
static __device__ __align__(256) double g_ke_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

template <int NPE>
__global__ void ke_static_kernel(int Ne, const float* __restrict__ nodes,
                                 const uint32_t* __restrict__ elements, double E, double nu,
                                 double t, const float* __restrict__ elem_t,
                                 double* __restrict__ ke) {
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
    double K[KK];
    if constexpr (NPE == 4)
        pg::q4_ke(c, E, nu, te, K);
    else
        pg::dkt_ke(c, E, nu, te, K);
    for (int i = 0; i < KK; i++) ke[(size_t)e * KK + i] = K[i];
}

// One colour of y += K x; elements of one colour share no node.
template <int NPE>
__global__ void applyk_static_kernel(int cnt, const uint32_t* __restrict__ list,
                                     const uint32_t* __restrict__ elements,
                                     const double* __restrict__ ke, const double* __restrict__ x,
                                     double* __restrict__ y) {
    constexpr int ND = 3 * NPE;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const uint32_t e = list[i];
    int dof[ND];
    double xl[ND];
#pragma unroll
    for (int k = 0; k < NPE; k++)
#pragma unroll
        for (int d = 0; d < 3; d++) {
            dof[3 * k + d] = (int)elements[(size_t)e * NPE + k] * 3 + d;
            xl[3 * k + d] = x[dof[3 * k + d]];
        }
    const double* K = ke + (size_t)e * ND * ND;
    for (int r = 0; r < ND; r++) {
        double s = 0;
#pragma unroll
        for (int c = 0; c < ND; c++) s += K[r * ND + c] * xl[c];
        y[dof[r]] += s;
    }
}

__global__ void bc_static_kernel(int n, const uint8_t* __restrict__ cons,
                                 const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && cons[i]) y[i] = x[i];
}

int fail(int st, char* msg, size_t len, const char* text) {
    if (msg && len) {
        std::strncpy(msg, text, len - 1);
        msg[len - 1] = 0;
    }
    return st;
}

// Device address of the static scratch on the current device, looked up
// once per device (cudaGetSymbolAddress must run with that device current).
// The cached address belongs to the device's current context: after a
// cudaDeviceReset the module is loaded again and the array may move, so
// this entry point must not be used across a device reset.
cudaError_t scratch_address(int dev, double** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ke_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = (double*)p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

template <int NPE>
int run(const pg_problem* p, const double* x, double* y, cudaStream_t st, double* ke, char* msg,
        size_t len) {
    const int Ne = (int)p->element_count, n = 3 * (int)p->node_count;
    cudaError_t e = cudaMemsetAsync(y, 0, (size_t)n * sizeof(double), st);
    if (e == cudaSuccess && Ne > 0)
        ke_static_kernel<NPE><<<(Ne + 127) / 128, 128, 0, st>>>(Ne, p->nodes, p->elements, p->E,
                                                                 p->nu, p->t, p->elem_t, ke);
    for (uint32_t c = 0; e == cudaSuccess && c < p->color_count; c++) {
        e = cudaGetLastError();
        const int off = (int)p->color_offsets[c], cnt = (int)(p->color_offsets[c + 1] - off);
        if (e == cudaSuccess && cnt > 0)
            applyk_static_kernel<NPE><<<(cnt + 127) / 128, 128, 0, st>>>(
                cnt, p->elements_by_color + off, p->elements, ke, x, y);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess)
        bc_static_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, p->constrained, x, y);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PG_ECUDA, msg, len, cudaGetErrorString(e));
    return PG_OK;
}

}  // namespace

extern "C" int pg_apply_k_static(const pg_problem* p, const double* x, double* y, void* stream,
                                 char* msg, size_t msg_len) {
    if (msg && msg_len) msg[0] = 0;
    if (!p) return fail(PG_EINVAL, msg, msg_len, "problem is NULL");
    if (p->nodes_per_element != 3 && p->nodes_per_element != 4)
        return fail(PG_EINVAL, msg, msg_len, "nodes_per_element must be 3 (DKT) or 4 (Q4)");
    const size_t kk = 9 * (size_t)p->nodes_per_element * p->nodes_per_element;
    if ((size_t)p->element_count * kk > kScratchDoubles) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "element_count %u exceeds the static scratch (at most %zu %s elements)",
                      p->element_count, kScratchDoubles / kk,
                      p->nodes_per_element == 4 ? "Q4" : "DKT");
        return fail(PG_EINVAL, msg, msg_len, buf);
    }
    if (p->node_count == 0) return PG_OK;
    if (!x || !y || !p->nodes || !p->constrained)
        return fail(PG_EINVAL, msg, msg_len, "x, y, nodes or constrained is NULL");
    if (p->element_count > 0 &&
        (!p->elements || !p->color_offsets || !p->elements_by_color || p->color_count == 0))
        return fail(PG_EINVAL, msg, msg_len, "elements or colouring arrays are NULL");
    if (p->element_count > 0) {
        // the offsets are on the host: check all of them before the kernels
        // index elements_by_color with them
        if (p->color_offsets[0] != 0 || p->color_offsets[p->color_count] != p->element_count)
            return fail(PG_EINVAL, msg, msg_len, "color_offsets must start at 0 and end at element_count");
        for (uint32_t c = 0; c < p->color_count; c++)
            if (p->color_offsets[c] > p->color_offsets[c + 1])
                return fail(PG_EINVAL, msg, msg_len, "color_offsets must not decrease");
    }
    {
        // y is cleared before K x is accumulated into it, so x and y must not
        // overlap (an in-place call would return K 0)
        const size_t bytes = 3 * (size_t)p->node_count * sizeof(double);
        const uintptr_t xa = (uintptr_t)x, ya = (uintptr_t)y;
        if (xa < ya + bytes && ya < xa + bytes)
            return fail(PG_EINVAL, msg, msg_len, "x and y must not overlap");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(PG_ECUDA, msg, msg_len, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(PG_EUNSUPPORTED, msg, msg_len, "device index too large");
    double* ke = nullptr;
    e = scratch_address(dev, &ke);
    if (e != cudaSuccess) return fail(PG_ECUDA, msg, msg_len, cudaGetErrorString(e));
    cudaStream_t st = (cudaStream_t)stream;
    return p->nodes_per_element == 4 ? run<4>(p, x, y, st, ke, msg, msg_len)
                                     : run<3>(p, x, y, st, ke, msg, msg_len);
}
