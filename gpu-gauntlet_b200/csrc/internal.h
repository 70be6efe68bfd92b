// Library-internal interface between plategpu.cu (contexts, plans, the
// persistent PCG) and learned.cu (the learned two-level preconditioner):
// the learned solver reads a plan's device-resident operator through this
// view instead of the plan's private layout.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "plategpu.h"

namespace pgi {

// A plan's operator on the device, valid while the plan lives (its set-up
// -- element matrices, block-Jacobi inverses -- has been queued on the
// context stream).
struct OperatorView {
    int Nn = 0, Ne = 0, npe = 0;
    const int* inc_ptr = nullptr;   // [Nn+1] node -> incident elements
    const int* inc_idx = nullptr;   // element * 4 + local node position
    const uint32_t* elements = nullptr;  // [npe * Ne]
    const float* ke32 = nullptr;    // [Ne][(3 npe)^2] element matrices
    const double* ke64 = nullptr;
    const float* binv32 = nullptr;  // [Nn][9] block-Jacobi inverses (computed in FP64)
    const double* binv64 = nullptr;
    const uint8_t* cons = nullptr;  // [3 Nn] constrained DOFs
};

std::mutex& ctx_mutex(pg_ctx* c);
int ctx_device(const pg_ctx* c);
int ctx_sms(const pg_ctx* c);
cudaStream_t ctx_stream(const pg_ctx* c);
void ctx_set_error(pg_ctx* c, const std::string& msg);
pg_ctx* plan_ctx(const pg_plan* h);
// Queues the plan's set-up if it has not run and returns its operator;
// the caller holds the context's mutex.  Returns an empty message on
// success.
std::string plan_operator(pg_plan* h, OperatorView* out);
// lambda_max(D^-1 K) of the plan's operator (30 power steps on the device,
// cached in the plan); the caller holds the context's mutex.
double plan_lambda_max(pg_plan* h);

// Flexible PCG on global memory (learned.cu): the solve of a plate whose
// partition does not fit the persistent kernel's shared memory.  FP32
// vectors, FP64 x, dot products and true-residual stop; mode 0 block
// Jacobi, mode 2 damped block-Jacobi smoothing steps (damping from
// lambda_max).  The caller holds the context's mutex and has set the
// device.  Failures return a pg_status and a message.
struct GlobalPcg;
GlobalPcg* global_pcg_create(pg_ctx* c, const OperatorView& ov, double lambda_max, std::string* err);
void global_pcg_destroy(GlobalPcg* g);
int global_pcg_solve(GlobalPcg* g, const pg_options& o, int mode, const float* F_dev, void* x_dst, bool x_host,
                     pg_info* info, std::string* err);

}  // namespace pgi
