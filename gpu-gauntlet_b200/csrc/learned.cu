// Learned two-level preconditioner: a U-Net coarse correction inside
// flexible PCG, trained on the GPU by this library's own kernels.
//
// The reference (cseifert512/gpu-gauntlet) preconditions its PCG with the
// 3 x 3 block Jacobi only (src/lib/plate/gpu/shaders/index.ts:214-262,
// applied once per iteration of runGPUPCG, src/lib/plate/gpu/solver.ts:
// 190-553).  This file adds, at that point of the iteration, a two-level
// preconditioner for plates on a structured node grid:
//
//   t  = S r                          damped block-Jacobi pre-smoothing,
//                                     S = omega D^-1
//   r1 = r - K t                      residual after smoothing
//   y  = N(r1)                        network correction (coarse level)
//   c  = y.r1 / y.K y                 energy-optimal step along y
//   z  = t + c y + S (r1 - c K y)     post-smoothing
//
// N maps the residual, laid out as a 3-channel image over the node grid
// (w, theta_x, theta_y per node), to an approximation of K^-1 r1.  It is a
// 4-level U-Net (unet.cuh) without biases, so N(c r) = c N(r) for c > 0 and
// its correction scales with the residual.  Whenever the correction cannot
// reduce the energy norm of the error (y.r1 <= 0) that iteration uses
// z = D^-1 r (plain block Jacobi), and after `fallback_after` such
// iterations in a row the rest of the solve is plain block-Jacobi PCG.  Because N is
// nonlinear the outer iteration is flexible PCG with the Polak-Ribiere
// beta = z_k+1 . (r_k+1 - r_k) / (z_k . r_k) and alpha = p.r / p.Kp.
//
// Precision: r, z, p, K p and the network in FP32 / BF16 (FP32
// accumulation); x, every dot product and the alpha/beta recurrences in
// FP64; the block inverses are computed in FP64; every `replace_every`
// iterations, and before the solve may stop, the residual is recomputed as
// r = F - K x in FP64 and the stop test is made on that true residual.
//
// Execution: the whole solve is one CUDA graph launch: a conditional WHILE
// node whose body is one iteration (about 30 kernels), ended from the
// device by cudaGraphSetConditional once the true residual meets the
// tolerance (or the iteration limit, a breakdown or a non-finite value).
// Training is a second graph whose WHILE body is one Adam step (batch
// gather, forward, energy-norm loss through the library's own K.p,
// backward, Adam), so an epoch is one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "internal.h"
#include "plategpu.h"
#include "unet.cuh"

using pgn::bf16;

namespace {

struct LFail {
    int status;
    std::string msg;
};

#define LCK(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw LFail{e_ == cudaErrorMemoryAllocation ? PG_ENOMEM : PG_ECUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_)};              \
    } while (0)

template <typename T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        n = count;
        if (count) LCK(cudaMalloc(&p, count * sizeof(T)));
    }
    void zero(cudaStream_t st) {
        if (n) LCK(cudaMemsetAsync(p, 0, n * sizeof(T), st));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~Buf() { release(); }
};

// ---------------------------------------------------------------------------
// network description (matches oracle/unet_oracle.py LAYERS)
// ---------------------------------------------------------------------------

struct LayerSpec {
    int cin, cout;  // real channel counts
};
constexpr LayerSpec kSpec[pgn::kLayers] = {
    {3, 16},   {16, 16},  {16, 32},  {32, 32},  {32, 64},  {64, 64},  {64, 128}, {128, 128},
    {192, 64}, {64, 64},  {96, 32},  {32, 32},  {48, 16},  {16, 16},  {16, 3}};
enum { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B, OUTL };

int pad16(int c) { return (c + 15) / 16 * 16; }

pgn::LayerTable make_table() {
    pgn::LayerTable T{};
    long off = 0, off_f = 0, off_d = 0;
    for (int k = 0; k < pgn::kLayers; k++) {
        const int ci = pad16(kSpec[k].cin), co = pad16(kSpec[k].cout);
        T.l[k] = {ci, co, off, off_f, off_d};
        off += 9L * ci * co;
        off_f += 9L * ci * co;
        off_d += 9L * ci * co;
    }
    T.total = off;
    return T;
}

long real_param_count() {
    long s = 0;
    for (const LayerSpec& l : kSpec) s += 9L * l.cin * l.cout;
    return s;
}

// Activations (and, for training, their gradients) of one batch size.
struct Workspace {
    int B = 0;
    bool grads = false;
    Buf<bf16> in, e0a, cat0, d0a, d0, p1, e1a, cat1, d1a, d1, p2, e2a, cat2, d2a, d2, p3, e3a, e3;
    Buf<float> out;  // [B][H][W][4], channels 0..2
    Buf<bf16> gout, g_d0, g_d0a, dcat0, g_d1, g_d1a, dcat1, g_d2, g_d2a, dcat2, g_e3, g_e3a, dp3, g_e2,
        g_e2a, dp2, g_e1, g_e1a, dp1, g_e0, g_e0a, din;
};

}  // namespace

struct pg_net {
    pg_ctx* ctx = nullptr;
    int H = 0, W = 0;
    int version = 0;  // bumped when the scales change (solve graphs bake them in)
    pgn::LayerTable T{};
    Buf<float> w, m, v, g;  // FP32 master weights, Adam moments, gradients (padded layout)
    Buf<bf16> wf, wd;       // BF16 forward / input-gradient copies
    Buf<int> step;          // Adam steps taken (device)
    float scale[6] = {1, 1, 1, 1, 1, 1};  // input scales (3) and output scales (3)
    std::map<int, std::unique_ptr<Workspace>> ws;
};

namespace {

// ---------------------------------------------------------------------------
// launches
// ---------------------------------------------------------------------------

// Output channels per block: the largest of 64, 48, 32, 16 that divides
// the layer's rows and keeps the halo and all nine taps' weights within
// 160 KB of shared memory.
int pick_cot(int rows, int cin) {
    for (int c : {64, 48, 32, 16})
        if (rows % c == 0 && pgn::conv_smem_bytes(cin, c) <= 160 * 1024) return c;
    return 16;
}

// Launches kernel<<<grid, block, smem, st>>>(args...), with programmatic
// stream serialisation when pdl is set (the kernel then starts while its
// predecessor finishes and waits in pdl_wait before reading its results).
template <typename... K, typename... A>
void launch(bool pdl, void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
    if (!pdl) {
        kernel<<<grid, block, smem, st>>>(std::forward<A>(args)...);
        LCK(cudaGetLastError());
        return;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    LCK(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

template <int CIN, int COT, int MODE>
void conv_launch(const pgn::ConvArgs& a, int rows, cudaStream_t st, bool pdl) {
    const int smem = pgn::conv_smem_bytes(CIN, COT);
    const void* fn = (const void*)pgn::conv3x3_kernel<CIN, COT, MODE>;
    LCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((a.W + 7) / 8, ((a.H + 7) / 8) * a.B, rows / COT);
    launch(pdl, pgn::conv3x3_kernel<CIN, COT, MODE>, grid, dim3(pgn::kConvThreads), smem, st, a);
}

// Dispatches the (input channels, output tile, epilogue) combinations the
// network uses.
void conv(int mode, int cin, int rows, const pgn::ConvArgs& a, cudaStream_t st, bool pdl = false) {
    const int cot = pick_cot(rows, cin);
#define PG_CONV(C, T, M)                                   \
    if (cin == C && cot == T && mode == M) {               \
        conv_launch<C, T, M>(a, rows, st, pdl);            \
        return;                                            \
    }
    using namespace pgn;
    PG_CONV(16, 16, OUT_BF16_RELU) PG_CONV(16, 32, OUT_BF16_RELU) PG_CONV(32, 32, OUT_BF16_RELU)
    PG_CONV(32, 64, OUT_BF16_RELU) PG_CONV(64, 64, OUT_BF16_RELU) PG_CONV(128, 32, OUT_BF16_RELU)
    PG_CONV(192, 32, OUT_BF16_RELU) PG_CONV(96, 32, OUT_BF16_RELU) PG_CONV(48, 16, OUT_BF16_RELU)
    PG_CONV(16, 16, OUT_F32)
    PG_CONV(16, 16, OUT_BF16_MASKED) PG_CONV(16, 48, OUT_BF16_MASKED) PG_CONV(32, 32, OUT_BF16_MASKED)
    PG_CONV(32, 48, OUT_BF16_MASKED) PG_CONV(64, 64, OUT_BF16_MASKED) PG_CONV(128, 32, OUT_BF16_MASKED)
    PG_CONV(128, 32, OUT_BF16) PG_CONV(64, 32, OUT_BF16) PG_CONV(32, 16, OUT_BF16) PG_CONV(16, 16, OUT_BF16)
#undef PG_CONV
    throw LFail{PG_EUNSUPPORTED, "no convolution kernel for cin " + std::to_string(cin) + ", tile " +
                                     std::to_string(cot) + ", mode " + std::to_string(mode)};
}

pgn::ConvArgs cargs(int B, int H, int W, const bf16* in, int in_cs, const bf16* w, int w_rows, void* out,
                    int out_cs, int out_coff, int cout_real, const int* skip) {
    pgn::ConvArgs a{};
    a.B = B;
    a.H = H;
    a.W = W;
    a.in = in;
    a.in_cs = in_cs;
    a.w = w;
    a.w_rows = w_rows;
    a.out = out;
    a.out_cs = out_cs;
    a.out_coff = out_coff;
    a.cout_real = cout_real;
    a.skip = skip;
    return a;
}

// The encoder's second convolution of a level also writes the pooled
// input of the next level (2 x 2 average in its epilogue).
pgn::ConvArgs pooled(pgn::ConvArgs a, bf16* pool_out, int pool_cs) {
    a.pool_out = pool_out;
    a.pool_cs = pool_cs;
    return a;
}

int ew_grid(long items) { return (int)std::min<long>((items + 255) / 256, 148L * 16); }

// The workspace of batch size B, created on first use; gradient buffers
// are added to an existing workspace when first needed, so the activation
// buffers a captured graph points to never move.
Workspace* workspace(pg_net* n, int B, bool grads) {
    auto it = n->ws.find(B);
    Workspace* w = nullptr;
    cudaStream_t st = pgi::ctx_stream(n->ctx);
    const size_t P0 = (size_t)B * n->H * n->W, P1 = P0 / 4, P2 = P1 / 4, P3 = P2 / 4;
    if (it != n->ws.end()) {
        w = it->second.get();
        if (w->grads || !grads) return w;
    } else {
        auto nw = std::make_unique<Workspace>();
        w = nw.get();
        n->ws[B] = std::move(nw);
        w->B = B;
        w->in.alloc(P0 * 16);
        w->e0a.alloc(P0 * 16);
        w->cat0.alloc(P0 * 48);
        w->d0a.alloc(P0 * 16);
        w->d0.alloc(P0 * 16);
        w->out.alloc(P0 * 4);
        w->p1.alloc(P1 * 16);
        w->e1a.alloc(P1 * 32);
        w->cat1.alloc(P1 * 96);
        w->d1a.alloc(P1 * 32);
        w->d1.alloc(P1 * 32);
        w->p2.alloc(P2 * 32);
        w->e2a.alloc(P2 * 64);
        w->cat2.alloc(P2 * 192);
        w->d2a.alloc(P2 * 64);
        w->d2.alloc(P2 * 64);
        w->p3.alloc(P3 * 64);
        w->e3a.alloc(P3 * 128);
        w->e3.alloc(P3 * 128);
        w->in.zero(st);  // channels 3..15 and pixels without a node stay 0
        w->out.zero(st);
    }
    if (grads) {
        w->grads = true;
        w->gout.alloc(P0 * 16);
        w->gout.zero(st);  // channels 3..15 and pixels without a node stay 0
        w->g_d0.alloc(P0 * 16);
        w->g_d0a.alloc(P0 * 16);
        w->dcat0.alloc(P0 * 48);
        w->g_d1.alloc(P1 * 32);
        w->g_d1a.alloc(P1 * 32);
        w->dcat1.alloc(P1 * 96);
        w->g_d2.alloc(P2 * 64);
        w->g_d2a.alloc(P2 * 64);
        w->dcat2.alloc(P2 * 192);
        w->g_e3.alloc(P3 * 128);
        w->g_e3a.alloc(P3 * 128);
        w->dp3.alloc(P3 * 64);
        w->g_e2.alloc(P2 * 64);
        w->g_e2a.alloc(P2 * 64);
        w->dp2.alloc(P2 * 32);
        w->g_e1.alloc(P1 * 32);
        w->g_e1a.alloc(P1 * 32);
        w->dp1.alloc(P1 * 16);
        w->g_e0.alloc(P0 * 16);
        w->g_e0a.alloc(P0 * 16);
        w->din.alloc(P0 * 16);
    }
    LCK(cudaStreamSynchronize(st));
    return w;
}

// U-Net forward of ws->in ([B][H][W][16], channels 0..2 used) into ws->out.
void net_forward(pg_net* n, Workspace* w, cudaStream_t st, const int* skip, bool pdl = false) {
    const int B = w->B;
    const int H0 = n->H, W0 = n->W, H1 = H0 / 2, W1 = W0 / 2, H2 = H1 / 2, W2 = W1 / 2, H3 = H2 / 2, W3 = W2 / 2;
    const pgn::LayerTable& T = n->T;
    auto wf = [&](int k) { return n->wf.p + T.l[k].off_f; };
    using namespace pgn;
    conv(OUT_BF16_RELU, 16, 16, cargs(B, H0, W0, w->in.p, 16, wf(E0A), 16, w->e0a.p, 16, 0, 16, skip), st, pdl);
    conv(OUT_BF16_RELU, 16, 16, pooled(cargs(B, H0, W0, w->e0a.p, 16, wf(E0B), 16, w->cat0.p, 48, 0, 16, skip), w->p1.p, 16), st, pdl);
    conv(OUT_BF16_RELU, 16, 32, cargs(B, H1, W1, w->p1.p, 16, wf(E1A), 32, w->e1a.p, 32, 0, 32, skip), st, pdl);
    conv(OUT_BF16_RELU, 32, 32, pooled(cargs(B, H1, W1, w->e1a.p, 32, wf(E1B), 32, w->cat1.p, 96, 0, 32, skip), w->p2.p, 32), st, pdl);
    conv(OUT_BF16_RELU, 32, 64, cargs(B, H2, W2, w->p2.p, 32, wf(E2A), 64, w->e2a.p, 64, 0, 64, skip), st, pdl);
    conv(OUT_BF16_RELU, 64, 64, pooled(cargs(B, H2, W2, w->e2a.p, 64, wf(E2B), 64, w->cat2.p, 192, 0, 64, skip), w->p3.p, 64), st, pdl);
    conv(OUT_BF16_RELU, 64, 128, cargs(B, H3, W3, w->p3.p, 64, wf(E3A), 128, w->e3a.p, 128, 0, 128, skip), st, pdl);
    conv(OUT_BF16_RELU, 128, 128, cargs(B, H3, W3, w->e3a.p, 128, wf(E3B), 128, w->e3.p, 128, 0, 128, skip), st, pdl);
    launch(pdl, up2_kernel, dim3(ew_grid((long)B * H2 * W2 * 16)), dim3(256), 0, st, B, H2, W2, w->e3.p, 128, 128, w->cat2.p, 192, 64, skip);
    conv(OUT_BF16_RELU, 192, 64, cargs(B, H2, W2, w->cat2.p, 192, wf(D2A), 64, w->d2a.p, 64, 0, 64, skip), st, pdl);
    conv(OUT_BF16_RELU, 64, 64, cargs(B, H2, W2, w->d2a.p, 64, wf(D2B), 64, w->d2.p, 64, 0, 64, skip), st, pdl);
    launch(pdl, up2_kernel, dim3(ew_grid((long)B * H1 * W1 * 8)), dim3(256), 0, st, B, H1, W1, w->d2.p, 64, 64, w->cat1.p, 96, 32, skip);
    conv(OUT_BF16_RELU, 96, 32, cargs(B, H1, W1, w->cat1.p, 96, wf(D1A), 32, w->d1a.p, 32, 0, 32, skip), st, pdl);
    conv(OUT_BF16_RELU, 32, 32, cargs(B, H1, W1, w->d1a.p, 32, wf(D1B), 32, w->d1.p, 32, 0, 32, skip), st, pdl);
    launch(pdl, up2_kernel, dim3(ew_grid((long)B * H0 * W0 * 4)), dim3(256), 0, st, B, H0, W0, w->d1.p, 32, 32, w->cat0.p, 48, 16, skip);
    conv(OUT_BF16_RELU, 48, 16, cargs(B, H0, W0, w->cat0.p, 48, wf(D0A), 16, w->d0a.p, 16, 0, 16, skip), st, pdl);
    conv(OUT_BF16_RELU, 16, 16, cargs(B, H0, W0, w->d0a.p, 16, wf(D0B), 16, w->d0.p, 16, 0, 16, skip), st, pdl);
    conv(OUT_F32, 16, 16, cargs(B, H0, W0, w->d0.p, 16, wf(OUTL), 16, w->out.p, 4, 0, 3, skip), st, pdl);
    LCK(cudaGetLastError());
}

void wgrad(pg_net* n, int k, int B, int H, int W, const bf16* x, int x_cs, const bf16* g, int g_cs,
           cudaStream_t st) {
    const pgn::LayerDesc& L = n->T.l[k];
    pgn::WgradArgs a{};
    a.B = B;
    a.H = H;
    a.W = W;
    a.x = x;
    a.x_cs = x_cs;
    a.g = g;
    a.g_cs = g_cs;
    a.dw = n->g.p + L.off;
    a.cin = L.cin;
    a.cout = L.cout;
    a.tiles = B * ((H + 7) / 8) * ((W + 7) / 8);
    const int cot = L.cout % 32 == 0 ? 32 : 16, cit = L.cin % 32 == 0 ? 32 : 16;
    const int gy = L.cout / cot, gz = L.cin / cit;
    const int gx = std::max(1, std::min(a.tiles, 148 * 4 / (gy * gz)));
    dim3 grid(gx, gy, gz);
    if (cot == 32 && cit == 32)
        pgn::wgrad_kernel<32, 32><<<grid, 128, 0, st>>>(a);
    else if (cot == 32)
        pgn::wgrad_kernel<32, 16><<<grid, 64, 0, st>>>(a);
    else if (cit == 32)
        pgn::wgrad_kernel<16, 32><<<grid, 64, 0, st>>>(a);
    else
        pgn::wgrad_kernel<16, 16><<<grid, 32, 0, st>>>(a);
    LCK(cudaGetLastError());
}

// Input gradient of layer k: dX = conv(G, W flipped/transposed), masked by
// (X > 0) when X is a ReLU output.
void dgrad(pg_net* n, int k, int B, int H, int W, const bf16* g, bf16* out, int out_cs, const bf16* mask,
           int mask_cs, cudaStream_t st) {
    const pgn::LayerDesc& L = n->T.l[k];
    pgn::ConvArgs a = cargs(B, H, W, g, L.cout, n->wd.p + L.off_d, L.cin, out, out_cs, 0, L.cin, nullptr);
    a.mask = mask;
    a.mask_cs = mask_cs;
    conv(mask ? pgn::OUT_BF16_MASKED : pgn::OUT_BF16, L.cout, L.cin, a, st);
}

// Backward of the forward pass held in w, from w->gout (dL/d out, [B][H][W][16],
// channels 0..2): accumulates into n->g (zero it first).  With din, also
// the gradient of the network input (w->din).
void net_backward(pg_net* n, Workspace* w, cudaStream_t st, bool din) {
    const int B = w->B;
    const int H0 = n->H, W0 = n->W, H1 = H0 / 2, W1 = W0 / 2, H2 = H1 / 2, W2 = W1 / 2, H3 = H2 / 2, W3 = W2 / 2;
    using namespace pgn;
    // output layer and level-0 decoder
    wgrad(n, OUTL, B, H0, W0, w->d0.p, 16, w->gout.p, 16, st);
    dgrad(n, OUTL, B, H0, W0, w->gout.p, w->g_d0.p, 16, w->d0.p, 16, st);
    wgrad(n, D0B, B, H0, W0, w->d0a.p, 16, w->g_d0.p, 16, st);
    dgrad(n, D0B, B, H0, W0, w->g_d0.p, w->g_d0a.p, 16, w->d0a.p, 16, st);
    wgrad(n, D0A, B, H0, W0, w->cat0.p, 48, w->g_d0a.p, 16, st);
    dgrad(n, D0A, B, H0, W0, w->g_d0a.p, w->dcat0.p, 48, w->cat0.p, 48, st);
    up2_bwd_kernel<<<ew_grid((long)B * H1 * W1 * 4), 256, 0, st>>>(B, H1, W1, w->dcat0.p, 48, 16, 32, w->g_d1.p, 32);
    // level-1 decoder
    wgrad(n, D1B, B, H1, W1, w->d1a.p, 32, w->g_d1.p, 32, st);
    dgrad(n, D1B, B, H1, W1, w->g_d1.p, w->g_d1a.p, 32, w->d1a.p, 32, st);
    wgrad(n, D1A, B, H1, W1, w->cat1.p, 96, w->g_d1a.p, 32, st);
    dgrad(n, D1A, B, H1, W1, w->g_d1a.p, w->dcat1.p, 96, w->cat1.p, 96, st);
    up2_bwd_kernel<<<ew_grid((long)B * H2 * W2 * 8), 256, 0, st>>>(B, H2, W2, w->dcat1.p, 96, 32, 64, w->g_d2.p, 64);
    // level-2 decoder
    wgrad(n, D2B, B, H2, W2, w->d2a.p, 64, w->g_d2.p, 64, st);
    dgrad(n, D2B, B, H2, W2, w->g_d2.p, w->g_d2a.p, 64, w->d2a.p, 64, st);
    wgrad(n, D2A, B, H2, W2, w->cat2.p, 192, w->g_d2a.p, 64, st);
    dgrad(n, D2A, B, H2, W2, w->g_d2a.p, w->dcat2.p, 192, w->cat2.p, 192, st);
    up2_bwd_kernel<<<ew_grid((long)B * H3 * W3 * 16), 256, 0, st>>>(B, H3, W3, w->dcat2.p, 192, 64, 128, w->g_e3.p, 128);
    // bottleneck
    wgrad(n, E3B, B, H3, W3, w->e3a.p, 128, w->g_e3.p, 128, st);
    dgrad(n, E3B, B, H3, W3, w->g_e3.p, w->g_e3a.p, 128, w->e3a.p, 128, st);
    wgrad(n, E3A, B, H3, W3, w->p3.p, 64, w->g_e3a.p, 128, st);
    dgrad(n, E3A, B, H3, W3, w->g_e3a.p, w->dp3.p, 64, nullptr, 0, st);
    // level-2 encoder
    pool2_bwd_add_kernel<<<ew_grid((long)B * H2 * W2 * 8), 256, 0, st>>>(B, H2, W2, w->dcat2.p, w->cat2.p, 192,
                                                                         w->dp3.p, 64, w->g_e2.p);
    wgrad(n, E2B, B, H2, W2, w->e2a.p, 64, w->g_e2.p, 64, st);
    dgrad(n, E2B, B, H2, W2, w->g_e2.p, w->g_e2a.p, 64, w->e2a.p, 64, st);
    wgrad(n, E2A, B, H2, W2, w->p2.p, 32, w->g_e2a.p, 64, st);
    dgrad(n, E2A, B, H2, W2, w->g_e2a.p, w->dp2.p, 32, nullptr, 0, st);
    // level-1 encoder
    pool2_bwd_add_kernel<<<ew_grid((long)B * H1 * W1 * 4), 256, 0, st>>>(B, H1, W1, w->dcat1.p, w->cat1.p, 96,
                                                                         w->dp2.p, 32, w->g_e1.p);
    wgrad(n, E1B, B, H1, W1, w->e1a.p, 32, w->g_e1.p, 32, st);
    dgrad(n, E1B, B, H1, W1, w->g_e1.p, w->g_e1a.p, 32, w->e1a.p, 32, st);
    wgrad(n, E1A, B, H1, W1, w->p1.p, 16, w->g_e1a.p, 32, st);
    dgrad(n, E1A, B, H1, W1, w->g_e1a.p, w->dp1.p, 16, nullptr, 0, st);
    // level-0 encoder
    pool2_bwd_add_kernel<<<ew_grid((long)B * H0 * W0 * 2), 256, 0, st>>>(B, H0, W0, w->dcat0.p, w->cat0.p, 48,
                                                                         w->dp1.p, 16, w->g_e0.p);
    wgrad(n, E0B, B, H0, W0, w->e0a.p, 16, w->g_e0.p, 16, st);
    dgrad(n, E0B, B, H0, W0, w->g_e0.p, w->g_e0a.p, 16, w->e0a.p, 16, st);
    wgrad(n, E0A, B, H0, W0, w->in.p, 16, w->g_e0a.p, 16, st);
    if (din) dgrad(n, E0A, B, H0, W0, w->g_e0a.p, w->din.p, 16, nullptr, 0, st);
    LCK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// operator kernels (plate side)
// ---------------------------------------------------------------------------

struct Op {
    int Nn;
    const int* inc_ptr;
    const int* inc_idx;
    const uint32_t* el;
    const float* ke32;
    const double* ke64;
    const float* binv32;
    const uint8_t* cons;
    // floats between element matrices in the FP32 K products: (3 npe)^2, or 0
    // when every element matrix equals the first to FP32 precision (a
    // uniform structured mesh), so that one matrix serves all elements from
    // L1; the FP64 products (true residual, pairs) always use each element's
    int ke_stride;
    // optional node-block form of the FP32 operator (sliced ELL): nodes in
    // slices of 32, slice s owning slots [nm_off[s], nm_off[s + 1]); slot j
    // holds, for each lane (node 32 s + lane), a neighbour column
    // nm_col[32 j + lane] and the assembled 3x3 block K_(node, column) in
    // nm_val[(9 j + q) 32 + lane] (row-major q), summed over the shared
    // elements in FP64 and rounded once; padding slots have zero blocks.
    const int* nm_off = nullptr;
    const int* nm_col = nullptr;
    const float* nm_val = nullptr;
    // threads per node of the flexible-PCG kernels (1 or 2): a plate that
    // fills less than a wave of the device at one thread per node splits
    // each node's K product between two threads
    int tpn = 1;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sums of K values into parts[blockIdx.x * K + k] (blockDim.x <= 1024).
template <int K>
__device__ void block_partials(double (&v)[K], double* parts) {
    __shared__ double red[K][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double s = warp_sum(v[k]);
        if (lane == 0) red[k][warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double s = warp_sum(lane < nw ? red[k][lane] : 0.0);
            if (lane == 0) parts[blockIdx.x * K + k] = s;
        }
    }
}

// Sum of nb blocks' partials, the same fixed order in every block (thread
// t adds partials t, t + blockDim.x, ..., then a fixed tree over lanes and
// warps); every thread of the block receives the K sums.  All threads load
// at once, so a grid of hundreds of blocks costs about one L2 round trip.
template <int K>
__device__ void reduce_parts(const double* parts, int nb, double (&out)[K]) {
    __shared__ double red[K][32];
    __shared__ double res[K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    double v[K];
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; k++) v[k] += parts[i * K + k];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double t = warp_sum(v[k]);
        if (lane == 0) red[k][warp] = t;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const double t = warp_sum(lane < nw ? red[k][lane] : 0.0);
            if (lane == 0) res[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = res[k];
    __syncthreads();
}

// (K v)_n for node n with v read through getv(m, d) (FP32 element matrices),
// constrained rows replaced by the identity (y_c = v_c).
// Partial sums of (K v)_n over the node's incident elements h, h + step, ...
// (FP32 element matrices).
template <int NPE, typename GetV>
__device__ __forceinline__ void kv_elem_sum(const Op& op, int n, int h, int step, GetV getv, float& s0, float& s1,
                                            float& s2) {
    constexpr int ND = 3 * NPE;
    for (int q = op.inc_ptr[n] + h; q < op.inc_ptr[n + 1]; q += step) {
        const int e = op.inc_idx[q] >> 2, k = op.inc_idx[q] & 3;
        const float* Ke = op.ke32 + (size_t)e * op.ke_stride + 3 * k * ND;
#pragma unroll
        for (int b = 0; b < NPE; b++) {
            const int m = (int)op.el[(size_t)e * NPE + b];
            const float v0 = getv(m, 0), v1 = getv(m, 1), v2 = getv(m, 2);
            const float* c0 = Ke + 3 * b;
            s0 += c0[0] * v0 + c0[1] * v1 + c0[2] * v2;
            s1 += c0[ND] * v0 + c0[ND + 1] * v1 + c0[ND + 2] * v2;
            s2 += c0[2 * ND] * v0 + c0[2 * ND + 1] * v1 + c0[2 * ND + 2] * v2;
        }
    }
}

// Partial sums of (K v)_n over the node's node-block slots h, h + step,
// ... (op.nm_* set); the loads of a slot are coalesced across the nodes of
// a slice.
template <typename GetV>
__device__ __forceinline__ void kv_block_sum(const Op& op, int n, int h, int step, GetV getv, float& s0,
                                             float& s1, float& s2) {
    const int s = n >> 5, lane = n & 31;
    const int j1 = op.nm_off[s + 1];
#pragma unroll 3
    for (int j = op.nm_off[s] + h; j < j1; j += step) {
        const int m = op.nm_col[32 * j + lane];
        const float* B = op.nm_val + (size_t)288 * j + lane;
        const float v0 = getv(m, 0), v1 = getv(m, 1), v2 = getv(m, 2);
        s0 += B[0] * v0 + B[32] * v1 + B[64] * v2;
        s1 += B[96] * v0 + B[128] * v1 + B[160] * v2;
        s2 += B[192] * v0 + B[224] * v1 + B[256] * v2;
    }
}

// (K v)_n for node n with v read through getv(m, d) (FP32 element
// matrices), constrained rows replaced by the identity (y_c = v_c).
template <int NPE, typename GetV>
__device__ __forceinline__ void kv_node(const Op& op, int n, GetV getv, float (&out)[3]) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    kv_elem_sum<NPE>(op, n, 0, 1, getv, s0, s1, s2);
    out[0] = op.cons[3 * n] ? getv(n, 0) : s0;
    out[1] = op.cons[3 * n + 1] ? getv(n, 1) : s1;
    out[2] = op.cons[3 * n + 2] ? getv(n, 2) : s2;
}

// (K v)_n by op.tpn threads per node: with two, lanes 2i and 2i + 1 of a
// warp share node n (h = lane parity), each sums half its slots
// (node-block form) or half its elements, and they exchange their sums.
// Every lane of the warp must call it; lanes with n >= Nn take part with
// zero sums and get zeros.
template <int NPE, typename GetV>
__device__ __forceinline__ void kv2(const Op& op, int n, int h, GetV getv, float (&out)[3]) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    const bool live = n < op.Nn;
    if (live) {
        if (op.nm_off)
            kv_block_sum(op, n, h, op.tpn, getv, s0, s1, s2);
        else
            kv_elem_sum<NPE>(op, n, h, op.tpn, getv, s0, s1, s2);
    }
    if (op.tpn == 2) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
        s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
        s2 += __shfl_xor_sync(0xffffffffu, s2, 1);
    }
    out[0] = out[1] = out[2] = 0.f;
    if (live) {
        out[0] = op.cons[3 * n] ? getv(n, 0) : s0;
        out[1] = op.cons[3 * n + 1] ? getv(n, 1) : s1;
        out[2] = op.cons[3 * n + 2] ? getv(n, 2) : s2;
    }
}

constexpr int kMaxNbr = 32;  // node-block form: largest neighbour count

// The distinct nodes of the elements around node n (n included), in
// increasing order, into nb; their count, or -1 past kMaxNbr.
template <int NPE>
__device__ int node_nbrs(const Op& op, int n, int (&nb)[kMaxNbr]) {
    int c = 0;
    for (int q = op.inc_ptr[n]; q < op.inc_ptr[n + 1]; q++) {
        const int e = op.inc_idx[q] >> 2;
        for (int b = 0; b < NPE; b++) {
            const int m = (int)op.el[(size_t)e * NPE + b];
            int i = 0;
            while (i < c && nb[i] < m) i++;
            if (i < c && nb[i] == m) continue;
            if (c == kMaxNbr) return -1;
            for (int k = c; k > i; k--) nb[k] = nb[k - 1];
            nb[i] = m;
            c++;
        }
    }
    return c;
}

// Node-block form, pass 1: the widest neighbour count of each slice of 32
// nodes (the grid covers exactly Ns * 32 threads in blocks of whole warps);
// *bad = 1 when some node has more than kMaxNbr neighbours.
template <int NPE>
__global__ void nm_width_kernel(Op op, int Ns, int* __restrict__ width, int* __restrict__ bad) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    int c = 0;
    if (n < op.Nn) {
        int nb[kMaxNbr];
        c = node_nbrs<NPE>(op, n, nb);
        if (c < 0) {
            atomicOr(bad, 1);
            c = 0;
        }
    }
    c = __reduce_max_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && (n >> 5) < Ns) width[n >> 5] = c;
}

// Pass 2: columns and FP64-assembled blocks of every slot (padding slots:
// column n, or 0 past the last node, and a zero block).
template <int NPE>
__global__ void nm_fill_kernel(Op op, int Ns, const int* __restrict__ off, int* __restrict__ col,
                               float* __restrict__ val) {
    constexpr int ND = 3 * NPE;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = n >> 5, lane = n & 31;
    if (s >= Ns) return;
    const int j0 = off[s], w = off[s + 1] - j0;
    int nb[kMaxNbr];
    int c = n < op.Nn ? node_nbrs<NPE>(op, n, nb) : 0;
    if (c < 0) c = 0;
    for (int j = 0; j < w; j++) {
        double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        int m = n < op.Nn ? n : 0;
        if (j < c) {
            m = nb[j];
            for (int q = op.inc_ptr[n]; q < op.inc_ptr[n + 1]; q++) {
                const int e = op.inc_idx[q] >> 2, k = op.inc_idx[q] & 3;
                const double* Ke = op.ke64 + (size_t)e * ND * ND;
                for (int b = 0; b < NPE; b++) {
                    if ((int)op.el[(size_t)e * NPE + b] != m) continue;
                    for (int r = 0; r < 3; r++)
                        for (int cc = 0; cc < 3; cc++) blk[3 * r + cc] += Ke[(3 * k + r) * ND + 3 * b + cc];
                }
            }
        }
        const size_t slot = (size_t)(j0 + j);
        col[32 * slot + lane] = m;
        for (int q = 0; q < 9; q++) val[(9 * slot + q) * 32 + lane] = (float)blk[q];
    }
}

__device__ __forceinline__ float binv_row(const float* B9, int d, float a, float b, float c) {
    return B9[3 * d] * a + B9[3 * d + 1] * b + B9[3 * d + 2] * c;
}

// ----- training data --------------------------------------------------------

// Residual/error pairs from solver output: r = F - K x_k (FP64), e = x* - x_k.
template <int NPE>
__global__ void make_pairs_kernel(Op op, int count, const float* __restrict__ F, const double* __restrict__ xs,
                                  const double* __restrict__ xk, float* __restrict__ R, float* __restrict__ E) {
    constexpr int ND = 3 * NPE;
    const int n = blockIdx.x * blockDim.x + threadIdx.x, p = blockIdx.y;
    if (n >= op.Nn || p >= count) return;
    const size_t base = (size_t)p * 3 * op.Nn;
    double s[3] = {0, 0, 0};
    if (xk) {
        for (int q = op.inc_ptr[n]; q < op.inc_ptr[n + 1]; q++) {
            const int e = op.inc_idx[q] >> 2, k = op.inc_idx[q] & 3;
            const double* Ke = op.ke64 + (size_t)e * ND * ND + 3 * k * ND;
            for (int b = 0; b < NPE; b++) {
                const int m = (int)op.el[(size_t)e * NPE + b];
                for (int d = 0; d < 3; d++)
                    for (int c = 0; c < 3; c++) s[d] += Ke[d * ND + 3 * b + c] * xk[base + 3 * m + c];
            }
        }
    }
    for (int d = 0; d < 3; d++) {
        const size_t i = base + 3 * n + d;
        const double kx = xk ? (op.cons[3 * n + d] ? xk[i] : s[d]) : 0.0;
        R[i] = (float)((double)F[i] - kx);
        E[i] = (float)(xs[i] - (xk ? xk[i] : 0.0));
    }
}

// Pre-smoothed pairs: t = omega D^-1 r, r1 = r - K t, e1 = e - t.  mode 0 sums
// r1_c^2 and e1_c^2 (stats[6]); mode 1 writes the scaled r1 into the
// compact image set img[p][pixel][4] (BF16, channels 0..2), e1 into E1,
// e1^T K e1 into den[p] and sum_c (e1_c / s_out_c)^2 into den2[p].
template <int NPE>
__global__ void prep_pairs_kernel(Op op, int count, const float* __restrict__ R, const float* __restrict__ E,
                                  const int* __restrict__ node_pixel, int HW, int mode, float omega, float s0,
                                  float s1, float s2, float so0, float so1, float so2, double* __restrict__ stats,
                                  bf16* __restrict__ img, float* __restrict__ E1, double* __restrict__ den,
                                  double* __restrict__ den2) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, p = blockIdx.y;
    const bool live = n < op.Nn;
    const size_t base = (size_t)p * 3 * op.Nn;
    const float* r = R + base;
    const float* e = E + base;
    auto tv = [&](int m, int d) {
        const float* B9 = op.binv32 + 9 * m;
        return omega * binv_row(B9, d, r[3 * m], r[3 * m + 1], r[3 * m + 2]);
    };
    auto e1v = [&](int m, int d) { return e[3 * m + d] - tv(m, d); };
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (live) {
        float u[3];
        kv_node<NPE>(op, n, tv, u);
        float r1[3], e1[3];
        for (int d = 0; d < 3; d++) {
            r1[d] = r[3 * n + d] - u[d];
            e1[d] = e1v(n, d);
        }
        if (mode == 0) {
            for (int d = 0; d < 3; d++) {
                acc[d] = (double)r1[d] * r1[d];
                acc[3 + d] = (double)e1[d] * e1[d];
            }
        } else {
            const float sc[3] = {s0, s1, s2};
            bf16* px = img + ((size_t)p * HW + node_pixel[n]) * 4;
            for (int d = 0; d < 3; d++) px[d] = __float2bfloat16_rn(sc[d] * r1[d]);
            px[3] = __float2bfloat16_rn(0.f);
            for (int d = 0; d < 3; d++) E1[base + 3 * n + d] = e1[d];
            float ke1[3];
            kv_node<NPE>(op, n, e1v, ke1);
            acc[0] = (double)e1[0] * ke1[0] + (double)e1[1] * ke1[1] + (double)e1[2] * ke1[2];
            const float so[3] = {so0, so1, so2};
            for (int d = 0; d < 3; d++) acc[1] += (double)(e1[d] / so[d]) * (e1[d] / so[d]);
        }
    }
    __shared__ double red[6][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 6; k++) {
        const double s = warp_sum(acc[k]);
        if (lane == 0) red[k][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        if (mode == 0) {
            for (int k = 0; k < 6; k++) {
                double s = 0;
                for (int i = 0; i < nw; i++) s += red[k][i];
                atomicAdd(stats + k, s);
            }
        } else {
            double s = 0, s2 = 0;
            for (int i = 0; i < nw; i++) {
                s += red[0][i];
                s2 += red[1][i];
            }
            atomicAdd(den + p, s);
            atomicAdd(den2 + p, s2);
        }
    }
}

// Batch input: in[b][pixel][0..15] = img[idx_b][pixel][0..2] (other channels 0).
// idx_b = perm[(step - 1) * B + b] when step is given (training), else idx[b].
__global__ void gather_batch_kernel(int B, int HW, const bf16* __restrict__ img, const int* __restrict__ perm,
                                    const int* __restrict__ step, bf16* __restrict__ in) {
    const long total = (long)B * HW;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int b = (int)(q / HW), px = (int)(q - (long)b * HW);
        const int idx = step ? perm[(size_t)(*step - 1) * B + b] : perm[b];
        const uint2 v = *reinterpret_cast<const uint2*>(img + ((size_t)idx * HW + px) * 4);
        uint4 o0, o1;
        o0.x = v.x;
        o0.y = v.y & 0xFFFFu;  // channel 3 cleared
        o0.z = o0.w = 0;
        o1.x = o1.y = o1.z = o1.w = 0;
        uint4* dst = reinterpret_cast<uint4*>(in + ((size_t)b * HW + px) * 16);
        dst[0] = o0;
        dst[1] = o1;
    }
}

// Loss of a batch, d = e1 - y with y = s_out * N(r1) (0 on constrained
// DOFs).  kind PG_LOSS_ENERGY: the energy norm of the error after the
// correction, loss += (d^T K d) / (B e1^T K e1), dL/d(out) = -2 s_out (K d) /
// (B e1^T K e1); kind PG_LOSS_SCALED_L2: the error in the network's output
// units, loss += sum (d / s_out)^2 / (B sum (e1 / s_out)^2), dL/d(out) =
// -2 (d / s_out) / (B sum (e1 / s_out)^2).  The gradient goes to
// gout[b][pixel][0..2] when gout is given.
template <int NPE>
__global__ void loss_kernel(Op op, int B, int HW, const int* __restrict__ node_pixel, const float* __restrict__ out,
                            const float* __restrict__ E1, const double* __restrict__ den,
                            const double* __restrict__ den2, int kind, const int* __restrict__ perm,
                            const int* __restrict__ step, float so0, float so1, float so2,
                            double* __restrict__ loss_hist, bf16* __restrict__ gout) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    const int idx = step ? perm[(size_t)(*step - 1) * B + b] : perm[b];
    const float so[3] = {so0, so1, so2};
    const float* e1 = E1 + (size_t)idx * 3 * op.Nn;
    const float* ob = out + (size_t)b * HW * 4;
    auto dv = [&](int m, int d) {
        const float y = op.cons[3 * m + d] ? 0.f : so[d] * ob[(size_t)node_pixel[m] * 4 + d];
        return e1[3 * m + d] - y;
    };
    double acc[1] = {0.0};
    if (n < op.Nn && kind == PG_LOSS_SCALED_L2) {
        const double sc = 1.0 / ((double)B * den2[idx]);
        float q[3];
        for (int d = 0; d < 3; d++) q[d] = op.cons[3 * n + d] ? 0.f : dv(n, d) / so[d];
        acc[0] = ((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2]) * sc;
        if (gout) {
            bf16* g = gout + ((size_t)b * HW + node_pixel[n]) * 16;
            for (int d = 0; d < 3; d++) g[d] = __float2bfloat16_rn((float)(-2.0 * sc * q[d]));
        }
    } else if (n < op.Nn) {
        const double sc = 1.0 / ((double)B * den[idx]);
        float kd[3];
        kv_node<NPE>(op, n, dv, kd);
        acc[0] = ((double)dv(n, 0) * kd[0] + (double)dv(n, 1) * kd[1] + (double)dv(n, 2) * kd[2]) * sc;
        if (gout) {
            bf16* g = gout + ((size_t)b * HW + node_pixel[n]) * 16;
            for (int d = 0; d < 3; d++)
                g[d] = __float2bfloat16_rn(op.cons[3 * n + d] ? 0.f : (float)(-2.0 * sc * so[d] * kd[d]));
        }
    }
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double s = warp_sum(acc[0]);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < (int)((blockDim.x + 31) >> 5); i++) t += red[i];
        atomicAdd(loss_hist + (step ? *step - 1 : 0), t);
    }
}

// PG_LOSS_SMOOTHED_ENERGY: the energy norm of the error after the
// correction and the solve's smoothing sweeps, |M^nu (e1 - y)|_K^2 / |e1|_K^2
// with M = I - S K, S = omega D^-1, nu = kCorrectionSweeps; its gradient is
// dL/dy = -2 (M^T)^nu K M^nu (e1 - y) / |e1|_K^2, M^T = I - K S.  Batched over
// [B][3 Nn] vectors; pair b is perm[(step - 1) B + b] (training) or perm[b].
__device__ __forceinline__ int pair_of(const int* perm, const int* step, int B, int b) {
    return step ? perm[(size_t)(*step - 1) * B + b] : perm[b];
}

// g = e1 - y (0 on constrained DOFs)
__global__ void sl_diff_kernel(Op op, int B, int HW, const int* __restrict__ node_pixel,
                               const float* __restrict__ out, const float* __restrict__ E1,
                               const int* __restrict__ perm, const int* __restrict__ step, float so0, float so1,
                               float so2, float* __restrict__ g) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (n >= op.Nn) return;
    const int idx = pair_of(perm, step, B, b);
    const float so[3] = {so0, so1, so2};
    const float* e1 = E1 + (size_t)idx * 3 * op.Nn;
    const float* ob = out + (size_t)b * HW * 4 + (size_t)node_pixel[n] * 4;
    for (int d = 0; d < 3; d++) {
        const int i = 3 * n + d;
        g[(size_t)b * 3 * op.Nn + i] = op.cons[i] ? 0.f : e1[i] - so[d] * ob[d];
    }
}

// forward sweep: out = in - S K in
template <int NPE>
__global__ void sl_sweep_kernel(Op op, float omega, const float* __restrict__ in, float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (n >= op.Nn) return;
    const float* gi = in + (size_t)b * 3 * op.Nn;
    auto gv = [&](int m, int d) { return gi[3 * m + d]; };
    float k[3];
    kv_node<NPE>(op, n, gv, k);
    const float* B9 = op.binv32 + 9 * n;
    for (int d = 0; d < 3; d++)
        out[(size_t)b * 3 * op.Nn + 3 * n + d] = gi[3 * n + d] - omega * binv_row(B9, d, k[0], k[1], k[2]);
}

// h = K g and loss += g.h / (B e1^T K e1)
template <int NPE>
__global__ void sl_energy_kernel(Op op, int B, const float* __restrict__ g, float* __restrict__ h,
                                 const double* __restrict__ den, const int* __restrict__ perm,
                                 const int* __restrict__ step, double* __restrict__ loss_hist) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    const int idx = pair_of(perm, step, B, b);
    const float* gi = g + (size_t)b * 3 * op.Nn;
    auto gv = [&](int m, int d) { return gi[3 * m + d]; };
    double acc = 0.0;
    if (n < op.Nn) {
        float k[3];
        kv_node<NPE>(op, n, gv, k);
        for (int d = 0; d < 3; d++) {
            h[(size_t)b * 3 * op.Nn + 3 * n + d] = k[d];
            acc += (double)gi[3 * n + d] * k[d];
        }
        acc /= (double)B * den[idx];
    }
    __shared__ double red[32];
    const double s = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int i = 0; i < (int)((blockDim.x + 31) >> 5); i++) t += red[i];
        atomicAdd(loss_hist + (step ? *step - 1 : 0), t);
    }
}

// backward sweep: out = in - K S in
template <int NPE>
__global__ void sl_bsweep_kernel(Op op, float omega, const float* __restrict__ in, float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (n >= op.Nn) return;
    const float* hi = in + (size_t)b * 3 * op.Nn;
    auto sv = [&](int m, int d) {
        const float* B9 = op.binv32 + 9 * m;
        return omega * binv_row(B9, d, hi[3 * m], hi[3 * m + 1], hi[3 * m + 2]);
    };
    float k[3];
    kv_node<NPE>(op, n, sv, k);
    for (int d = 0; d < 3; d++) out[(size_t)b * 3 * op.Nn + 3 * n + d] = hi[3 * n + d] - k[d];
}

// dL/d(out) = -2 s_out h / (B e1^T K e1), 0 on constrained DOFs
__global__ void sl_grad_kernel(Op op, int B, int HW, const int* __restrict__ node_pixel, const float* __restrict__ h,
                               const double* __restrict__ den, const int* __restrict__ perm,
                               const int* __restrict__ step, float so0, float so1, float so2,
                               bf16* __restrict__ gout) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (n >= op.Nn) return;
    const int idx = pair_of(perm, step, B, b);
    const float so[3] = {so0, so1, so2};
    const double sc = 1.0 / ((double)B * den[idx]);
    bf16* g = gout + ((size_t)b * HW + node_pixel[n]) * 16;
    for (int d = 0; d < 3; d++) {
        const int i = 3 * n + d;
        g[d] = __float2bfloat16_rn(op.cons[i] ? 0.f : (float)(-2.0 * sc * so[d] * h[(size_t)b * 3 * op.Nn + i]));
    }
}

__global__ void step_begin_kernel(int* step) { *step += 1; }

__global__ void train_tick_kernel(cudaGraphConditionalHandle h, const int* step, const int* stop) {
    cudaGraphSetConditional(h, *step < *stop ? 1u : 0u);
}

// ----- flexible PCG ---------------------------------------------------------

struct FState {
    int it, done, converged, stop_reason, tr_ran, net_off, net_off_at, bad_count, use_net, skip_net;
    int iterations, net_iters, replacements, error;
    float net_step;  // the last iteration's step c along the network's correction
    int stall;       // set by the stall guard, folded into net_off by the tick
    double tr_prev;  // true residual^2 at the last periodic replacement
    double bnorm2, rr, true_rr, alpha, beta, gamma_prev, gamma_next;
};

// Damped block-Jacobi sweeps applied to the network's correction before
// it is used (w <- w + S (r1 - K w)): they remove the rough part of the
// correction -- BF16 rounding alone leaves white noise whose energy is
// comparable to the whole error's -- and the training loss
// PG_LOSS_SMOOTHED_ENERGY measures the error after the same sweeps.
constexpr int kCorrectionSweeps = 2;

struct FArgs {
    Op op;
    int HW;
    const int* node_pixel;
    bf16* img_in;        // [HW][16]
    const float* img_out;  // [HW][4]
    float si0, si1, si2, so0, so1, so2;
    float omega;  // damping of the block-Jacobi smoothing steps
    const float* F;
    double* x;
    float *r, *r_prev, *r1, *y, *r2, *z, *p0, *p1, *q;
    float *y2, *v2;  // the correction and its K product after odd sweeps (double buffer)
    float* t;        // omega D^-1 r (modes 1 and 2), written with r
    double *pU, *pTR, *pA, *pB, *pC, *pD, *pI;
    FState* st;
    int G;
    double tol2;
    int stop_rule, maxit, replace_every, mode, fallback_after;
};

__device__ __forceinline__ bool stop_test(const FArgs& a, double rr, double bn2) {
    return a.stop_rule == PG_STOP_RELATIVE ? rr < a.tol2 * bn2 : (rr < a.tol2 || rr < a.tol2 * bn2);
}

// t_n = omega D_n^-1 r_n, the first smoothing step, for the gathers of the
// smoothing input (modes 1 and 2)
__device__ __forceinline__ void write_t(const FArgs& a, int n, const float (&rv)[3]) {
    const float* B9 = a.op.binv32 + 9 * n;
    for (int d = 0; d < 3; d++) a.t[3 * n + d] = a.omega * binv_row(B9, d, rv[0], rv[1], rv[2]);
}

// op.tpn threads per node in the flexible-PCG kernels: thread t works on
// node t / tpn (h = t mod tpn); the K products split the node's sums
// between them (kv2), node-local work runs on the first thread only.
__device__ __forceinline__ int fp_node(const Op& op, int& h) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    h = op.tpn == 2 ? (t & 1) : 0;
    return op.tpn == 2 ? (t >> 1) : t;
}

__global__ void fp_init_kernel(FArgs a) {
    int h;
    const int n = fp_node(a.op, h);
    double acc[1] = {0.0};
    if (n < a.op.Nn && h == 0) {
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            const float f = a.F[i];
            a.x[i] = 0.0;
            a.r[i] = f;
            a.r_prev[i] = f;
            a.p0[i] = a.p1[i] = a.q[i] = 0.f;
            acc[0] += (double)f * f;
        }
    }
    block_partials<1>(acc, a.pI);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        FState s{};
        s.gamma_prev = 1.0;
        *a.st = s;
    }
}

// U: x += alpha p, r -= alpha q with alpha = p.r / p.Kp of the last
// direction (0 at the first iteration).
__global__ void fp_update_kernel(FArgs a) {
    pgn::pdl_wait();
    FState* st = a.st;
    const int it = st->it;
    double alpha = 0.0, bn2 = 0.0;
    int stop = 0;  // 1 zero rhs, 2 breakdown, 3 non-finite
    if (it == 0) {
        double s[1];
        reduce_parts<1>(a.pI, a.G, s);
        bn2 = s[0];
        if (!isfinite(bn2)) stop = 3;
        else if (bn2 < 1e-60) stop = 1;
    } else {
        double s[2];
        reduce_parts<2>(a.pD, a.G, s);
        if (!isfinite(s[0]) || !isfinite(s[1])) stop = 3;
        else if (fabs(s[0]) < 1e-30) stop = 2;
        else alpha = s[1] / s[0];
    }
    const float* p = (it & 1) ? a.p1 : a.p0;
    int h;
    const int n = fp_node(a.op, h);
    double acc[1] = {0.0};
    if (n < a.op.Nn && h == 0 && !stop) {
        float rv[3];
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            const float ri = a.r[i];
            a.x[i] += alpha * (double)p[i];
            a.r_prev[i] = ri;
            const float rn = (float)((double)ri - alpha * (double)a.q[i]);
            a.r[i] = rn;
            rv[d] = rn;
            acc[0] += (double)rn * rn;
        }
        if (a.mode != 0) write_t(a, n, rv);
    }
    block_partials<1>(acc, a.pU);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (it == 0) st->bnorm2 = bn2;
        st->alpha = alpha;
        if (stop) {
            st->done = 1;
            st->converged = stop == 1;
            st->stop_reason = stop == 1 ? PG_STOP_ZERO_RHS : PG_STOP_BREAKDOWN;
            st->error = stop == 3;
            st->iterations = it;
            st->skip_net = 1;
        }
    }
}

// TR: when the recursive residual meets the tolerance, every replace_every
// iterations and at the iteration limit: r = F - K x in FP64 (then rounded),
// and |F - K x|^2 for the stop test.
template <int NPE>
__global__ void fp_true_res_kernel(FArgs a) {
    pgn::pdl_wait();
    constexpr int ND = 3 * NPE;
    FState* st = a.st;
    if (st->done) return;
    const int it = st->it;
    double s[1];
    reduce_parts<1>(a.pU, a.G, s);
    const bool trig = stop_test(a, s[0], st->bnorm2) || (it > 0 && it % a.replace_every == 0) ||
                      it >= a.maxit || !isfinite(s[0]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->tr_ran = trig;
        st->rr = s[0];
        if (trig) st->replacements++;
    }
    if (!trig) return;
    int h;
    const int n = fp_node(a.op, h);
    double acc[1] = {0.0};
    // the node's FP64 product split between the two threads (every other
    // incident element), then exchanged
    double kx[3] = {0, 0, 0};
    if (n < a.op.Nn)
        for (int q = a.op.inc_ptr[n] + h; q < a.op.inc_ptr[n + 1]; q += a.op.tpn) {
            const int e = a.op.inc_idx[q] >> 2, k = a.op.inc_idx[q] & 3;
            const double* Ke = a.op.ke64 + (size_t)e * ND * ND + 3 * k * ND;
            for (int b = 0; b < NPE; b++) {
                const int m = (int)a.op.el[(size_t)e * NPE + b];
                const double x0 = a.x[3 * m], x1 = a.x[3 * m + 1], x2 = a.x[3 * m + 2];
                for (int d = 0; d < 3; d++) kx[d] += Ke[d * ND + 3 * b] * x0 + Ke[d * ND + 3 * b + 1] * x1 +
                                                     Ke[d * ND + 3 * b + 2] * x2;
            }
        }
    if (a.op.tpn == 2)
        for (int d = 0; d < 3; d++) kx[d] += __shfl_xor_sync(0xffffffffu, kx[d], 1);
    if (n < a.op.Nn && h == 0) {
        float rv[3];
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            const double rt = (double)a.F[i] - (a.op.cons[i] ? a.x[i] : kx[d]);
            rv[d] = (float)rt;
            a.r[i] = rv[d];
            acc[0] += rt * rt;
        }
        if (a.mode != 0) write_t(a, n, rv);
    }
    block_partials<1>(acc, a.pTR);
}

// A: stop decision on the true residual; then r1 = r - K t, t = omega D^-1 r,
// and the network input image (s_in r1).
template <int NPE>
__global__ void fp_prep_kernel(FArgs a) {
    pgn::pdl_wait();
    FState* st = a.st;
    if (st->done) return;
    const int it = st->it;
    if (st->tr_ran) {
        double s[1];
        reduce_parts<1>(a.pTR, a.G, s);
        const bool fin = isfinite(s[0]);
        const bool conv = fin && stop_test(a, s[0], st->bnorm2);
        if (conv || it >= a.maxit || !fin) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->done = 1;
                st->converged = conv;
                st->stop_reason = conv ? PG_STOP_CONVERGED : PG_STOP_MAX_ITER;
                st->error = !fin;
                st->true_rr = s[0];
                st->iterations = it;
                st->skip_net = 1;
            }
            return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            // stall guard: with the network on, a replacement interval that did
            // not cut the true residual norm by 20% switches it off (a weak
            // network can keep y.r1 > 0 while flexible PCG stagnates); the
            // first interval compares with |F|
            const double prev = st->tr_prev > 0 ? st->tr_prev : st->bnorm2;
            if (a.mode == 1 && !st->net_off && it % a.replace_every == 0 && s[0] > 0.64 * prev) st->stall = 1;
            if (it % a.replace_every == 0) st->tr_prev = s[0];
            st->true_rr = s[0];
        }
    }
    const bool skip = a.mode != 1 || st->net_off;
    if (blockIdx.x == 0 && threadIdx.x == 0) st->skip_net = skip;
    if (a.mode == 0 || (a.mode == 1 && st->net_off)) return;
    int h;
    const int n = fp_node(a.op, h);
    double acc[1] = {0.0};
    const float* r = a.r;
    const float* t = a.t;
    auto tv = [&](int m, int d) { return t[3 * m + d]; };
    float u[3];
    kv2<NPE>(a.op, n, h, tv, u);
    if (n < a.op.Nn && h == 0) {
        const float sc[3] = {a.si0, a.si1, a.si2};
        // only mode 1 has a network (and its input image and pixel map)
        bf16* px = a.mode == 1 ? a.img_in + (size_t)a.node_pixel[n] * 16 : nullptr;
        for (int d = 0; d < 3; d++) {
            const float r1 = r[3 * n + d] - u[d];
            a.r1[3 * n + d] = r1;
            if (px) px[d] = __float2bfloat16_rn(sc[d] * r1);
            acc[0] += (double)r1 * r1;
        }
    }
    block_partials<1>(acc, a.pA);
}

// The next smoothing sweep's correction at node n: w' = w + omega D^-1
// (r1 - v), v = K w (0 on constrained DOFs).
__device__ __forceinline__ void write_sweep(const FArgs& a, int n, const float (&w)[3], const float (&v)[3],
                                            float* __restrict__ w_next) {
    const int i = 3 * n;
    const float* B9 = a.op.binv32 + 9 * n;
    const float d0 = a.r1[i] - v[0], d1 = a.r1[i + 1] - v[1], d2 = a.r1[i + 2] - v[2];
    for (int d = 0; d < 3; d++)
        w_next[i + d] = a.op.cons[i + d] ? 0.f : w[d] + a.omega * binv_row(B9, d, d0, d1, d2);
}

// B: y = s_out N(r1) (0 on constrained DOFs) into a.y and v = K y into
// a.r2; partial sums of y.r1 and y.v for the correction's step; w_next
// (when the correction gets smoothing sweeps): the first sweep's w.
template <int NPE>
__global__ void fp_net_kernel(FArgs a, float* __restrict__ w_next) {
    pgn::pdl_wait();
    FState* st = a.st;
    if (st->done || st->skip_net) return;
    int h;
    const int n = fp_node(a.op, h);
    const float so[3] = {a.so0, a.so1, a.so2};
    auto yv = [&](int m, int d) {
        return a.op.cons[3 * m + d] ? 0.f : so[d] * a.img_out[(size_t)a.node_pixel[m] * 4 + d];
    };
    double acc[2] = {0.0, 0.0};
    float v[3], y[3];
    kv2<NPE>(a.op, n, h, yv, v);
    if (n < a.op.Nn && h == 0) {
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            y[d] = yv(n, d);
            a.y[i] = y[d];
            a.r2[i] = v[d];
            acc[0] += (double)y[d] * a.r1[i];
            acc[1] += (double)y[d] * v[d];
        }
        if (w_next) write_sweep(a, n, y, v, w_next);
    }
    block_partials<2>(acc, a.pB);
}

// One smoothing sweep on the network's correction: v = K w for the w the
// previous kernel formed (w = w_prev + omega D^-1 (r1 - K w_prev)), partial
// sums of w.r1 and w.v for the step, and (w_next) the next sweep's w.
template <int NPE>
__global__ void fp_sweep_kernel(FArgs a, const float* __restrict__ w_in, float* __restrict__ v_out,
                                float* __restrict__ w_next) {
    pgn::pdl_wait();
    FState* st = a.st;
    if (st->done || st->skip_net) return;
    auto wv = [&](int m, int d) { return w_in[3 * m + d]; };
    int h;
    const int n = fp_node(a.op, h);
    double acc[2] = {0.0, 0.0};
    float v[3], w[3];
    kv2<NPE>(a.op, n, h, wv, v);
    if (n < a.op.Nn && h == 0) {
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            w[d] = w_in[i];
            v_out[i] = v[d];
            acc[0] += (double)w[d] * a.r1[i];
            acc[1] += (double)w[d] * v[d];
        }
        if (w_next) write_sweep(a, n, w, v, w_next);
    }
    block_partials<2>(acc, a.pB);
}

// C: with the network's correction y (mode 1), its energy-optimal step
// c = y.r1 / y.K y (the multiple of y that most reduces the energy norm of
// the error e1 = K^-1 r1: by (y.r1)^2 / y.K y) and
// z = t + c y + omega D^-1 (r1 - c K y), t = omega D^-1 r; the correction is
// used only when y.r1 > 0 and y.K y > 0 (otherwise it cannot reduce the
// error) and the iteration falls back to plain block Jacobi z = D^-1 r.
// Mode 2 (the smoothing steps without the network): z = t + omega D^-1 r1.
// Mode 0: z = D^-1 r.
__global__ void fp_prec_kernel(FArgs a) {
    pgn::pdl_wait();
    FState* st = a.st;
    if (st->done) return;
    bool use = false;
    float c = 0.f;
    if (a.mode == 1 && !st->skip_net) {
        double s[2];
        reduce_parts<2>(a.pB, a.G, s);
        const double cd = s[0] / s[1];
        use = s[0] > 0.0 && s[1] > 0.0 && isfinite(cd);
        c = use ? (float)cd : 0.f;
    }
    const bool smooth2 = a.mode == 2;
    int h;
    const int n = fp_node(a.op, h);
    double acc[2] = {0.0, 0.0};
    if (n < a.op.Nn && h == 0) {
        const float* B9 = a.op.binv32 + 9 * n;
        const int i = 3 * n;
        const float r0 = a.r[i], r1_ = a.r[i + 1], r2_ = a.r[i + 2];
        const float om = a.omega;
        float z[3];
        for (int d = 0; d < 3; d++) z[d] = binv_row(B9, d, r0, r1_, r2_);
        if (use) {
            const float q0 = a.r1[i] - c * a.r2[i], q1 = a.r1[i + 1] - c * a.r2[i + 1],
                        q2 = a.r1[i + 2] - c * a.r2[i + 2];
            for (int d = 0; d < 3; d++) z[d] = om * z[d] + c * a.y[i + d] + om * binv_row(B9, d, q0, q1, q2);
        } else if (smooth2) {
            const float q0 = a.r1[i], q1 = a.r1[i + 1], q2 = a.r1[i + 2];
            for (int d = 0; d < 3; d++) z[d] = om * z[d] + om * binv_row(B9, d, q0, q1, q2);
        }
        for (int d = 0; d < 3; d++) {
            a.z[i + d] = z[d];
            acc[0] += (double)z[d] * a.r[i + d];
            acc[1] += (double)z[d] * a.r_prev[i + d];
        }
    }
    block_partials<2>(acc, a.pC);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->use_net = use;
        if (a.mode == 1 && !st->skip_net) {
            st->bad_count = use ? 0 : st->bad_count + 1;
            st->net_iters += use;
            st->net_step = c;
        }
    }
}

// D: beta (Polak-Ribiere), p = z + beta p_old, q = K p.
template <int NPE>
__global__ void fp_dir_kernel(FArgs a) {
    pgn::pdl_wait();
    FState* st = a.st;
    if (st->done) return;
    const int it = st->it;
    double s[2];
    reduce_parts<2>(a.pC, a.G, s);
    double beta = it == 0 ? 0.0 : (s[0] - s[1]) / st->gamma_prev;
    if (!isfinite(beta)) beta = 0.0;
    const float* po = (it & 1) ? a.p1 : a.p0;
    float* pn = (it & 1) ? a.p0 : a.p1;
    const float bf = (float)beta;
    auto pv = [&](int m, int d) { return a.z[3 * m + d] + bf * po[3 * m + d]; };
    int h;
    const int n = fp_node(a.op, h);
    double acc[2] = {0.0, 0.0};
    float qv[3];
    kv2<NPE>(a.op, n, h, pv, qv);
    if (n < a.op.Nn && h == 0) {
        for (int d = 0; d < 3; d++) {
            const int i = 3 * n + d;
            const float pi = pv(n, d);
            pn[i] = pi;
            a.q[i] = qv[d];
            acc[0] += (double)pi * qv[d];
            acc[1] += (double)pi * a.r[i];
        }
    }
    block_partials<2>(acc, a.pD);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->gamma_next = s[0];
        st->beta = beta;
    }
}

// y = K x by the flexible PCG's operator (pg_learned_apply_k)
template <int NPE>
__global__ void apply_op_kernel(Op op, const float* __restrict__ x, float* __restrict__ y) {
    int h;
    const int n = fp_node(op, h);
    auto xv = [&](int m, int d) { return x[3 * m + d]; };
    float v[3];
    kv2<NPE>(op, n, h, xv, v);
    if (n < op.Nn && h == 0)
        for (int d = 0; d < 3; d++) y[3 * n + d] = v[d];
}

__global__ void fp_tick_kernel(FArgs a, cudaGraphConditionalHandle h, int in_graph) {
    pgn::pdl_wait();
    FState* st = a.st;
    st->gamma_prev = st->gamma_next;
    if (a.mode == 1 && !st->net_off && (st->bad_count >= a.fallback_after || st->stall)) {
        st->net_off = 1;
        st->net_off_at = st->it;
    }
    st->it += 1;
    if (in_graph) cudaGraphSetConditional(h, (!st->done && st->it <= a.maxit + 1) ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

template <typename F>
int lguarded(pg_ctx* c, F&& body) {
    if (!c) return PG_EINVAL;
    std::lock_guard<std::mutex> lk(pgi::ctx_mutex(c));
    try {
        LCK(cudaSetDevice(pgi::ctx_device(c)));
        body();
    } catch (const LFail& f) {
        pgi::ctx_set_error(c, f.msg);
        return f.status;
    } catch (const std::bad_alloc&) {
        pgi::ctx_set_error(c, "host allocation failed");
        return PG_ENOMEM;
    }
    return PG_OK;
}

}  // namespace

// Flexible-PCG solver state on one operator: its vectors, reduction
// partials, device state record and the solve graph (the learned solver's,
// and the global-memory path's for plates past shared-memory capacity).
struct FpcgSolver {
    pg_ctx* ctx = nullptr;
    Op op{};
    int npe = 4;
    float omega = 1.f;
    Buf<float> F, r, r_prev, r1, y, r2, z, p0, p1, q, y2, v2, t;
    Buf<double> x, parts;
    Buf<int> nm_off, nm_col;  // node-block form of the operator (op.nm_*)
    Buf<float> nm_val;
    Buf<FState> st;
    cudaStream_t cap = nullptr;  // capture stream
    cudaGraphExec_t exec = nullptr;
    bool pdl = false, pdl_refused = false;  // graph built with programmatic dependent launch
    int mode = -1, maxit = -1, rule = -1, version = -1;
    double tol = -1;
    ~FpcgSolver() {
        if (exec) cudaGraphExecDestroy(exec);
        if (cap) cudaStreamDestroy(cap);
    }
};

// The learned solver of one plan: the node -> pixel map, the training set
// and the flexible-PCG solver.
struct pg_learned {
    pg_plan* plan = nullptr;
    pg_net* net = nullptr;
    pg_ctx* ctx = nullptr;
    pgi::OperatorView ov{};
    Op op{};
    int HW = 0;
    float omega = 1.f;  // damping of the smoothing steps (training and solve)
    Buf<int> node_pixel;
    // training set
    int P = 0;
    Buf<bf16> img;
    Buf<float> E1;
    Buf<double> den, den2, stats, loss_hist;
    Buf<float> sg, sh;  // [batch][3 Nn] vectors of the smoothed energy loss
    int sl_batch = 0;
    Buf<int> perm, stop_step;
    FpcgSolver S;
    cudaGraphExec_t train_exec = nullptr;
    int train_B = 0;
    ~pg_learned() {
        if (train_exec) cudaGraphExecDestroy(train_exec);
    }
};

namespace {

// Largest |Ke_e - Ke_0| and |Ke_0| entries (FP32 element matrices) as
// float bit patterns (non-negative floats order like their bits).
__global__ void ke_spread_kernel(long total, int kk, const float* __restrict__ ke, unsigned* out) {
    unsigned md = 0, m0 = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const float a = ke[i], b = ke[i % kk];
        md = max(md, __float_as_uint(fabsf(a - b)));
        if (i < kk) m0 = max(m0, __float_as_uint(fabsf(a)));
    }
    atomicMax(out, md);
    atomicMax(out + 1, m0);
}

// The operator of a plan for the flexible-PCG kernels: one shared FP32
// element matrix when all agree with the first within 1e-6 of its largest
// entry (FP32's own rounding is 6e-8), else each element's own.
Op make_op(const pgi::OperatorView& v, cudaStream_t st) {
    Op op{v.Nn, v.inc_ptr, v.inc_idx, v.elements, v.ke32, v.ke64, v.binv32, v.cons, 9 * v.npe * v.npe};
    if (v.Ne <= 1) return op;
    Buf<unsigned> mx;
    mx.alloc(2);
    mx.zero(st);
    const int kk = 9 * v.npe * v.npe;
    const long total = (long)v.Ne * kk;
    ke_spread_kernel<<<(int)std::min<long>((total + 255) / 256, 2048), 256, 0, st>>>(total, kk, v.ke32, mx.p);
    LCK(cudaGetLastError());
    unsigned h[2];
    LCK(cudaMemcpyAsync(h, mx.p, sizeof h, cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    float d, m;
    std::memcpy(&d, &h[0], 4);
    std::memcpy(&m, &h[1], 4);
    if (m > 0 && d <= 1e-6f * m) op.ke_stride = 0;
    return op;
}

// Real (unpadded, oracle-order) parameters <-> padded master layout.
void real_to_padded(const pg_net* n, const float* real, std::vector<float>& pad) {
    pad.assign(n->T.total, 0.f);
    long k = 0;
    for (int l = 0; l < pgn::kLayers; l++) {
        const pgn::LayerDesc& L = n->T.l[l];
        for (int co = 0; co < kSpec[l].cout; co++)
            for (int tap = 0; tap < 9; tap++)
                for (int ci = 0; ci < kSpec[l].cin; ci++) pad[L.off + ((long)co * 9 + tap) * L.cin + ci] = real[k++];
    }
}

void padded_to_real(const pg_net* n, const std::vector<float>& pad, float* real) {
    long k = 0;
    for (int l = 0; l < pgn::kLayers; l++) {
        const pgn::LayerDesc& L = n->T.l[l];
        for (int co = 0; co < kSpec[l].cout; co++)
            for (int tap = 0; tap < 9; tap++)
                for (int ci = 0; ci < kSpec[l].cin; ci++) real[k++] = pad[L.off + ((long)co * 9 + tap) * L.cin + ci];
    }
}

void refresh_bf16(pg_net* n, cudaStream_t st) {
    pgn::weights_to_bf16_kernel<<<ew_grid(n->T.total), 256, 0, st>>>(n->T, n->w.p, n->wf.p, n->wd.p);
    LCK(cudaGetLastError());
}

// FP32 [B][H][W][3] <-> the workspace's BF16 [B][H][W][16] / FP32 [B][H][W][4]
__global__ void pack_in_kernel(long P, const float* __restrict__ src, bf16* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < 16; c++) dst[i * 16 + c] = __float2bfloat16_rn(c < 3 ? src[i * 3 + c] : 0.f);
}
__global__ void unpack_out_kernel(long P, const float* __restrict__ src, float* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) dst[i * 3 + c] = src[i * 4 + c];
}
__global__ void pack_gout_kernel(long P, const float* __restrict__ src, bf16* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < 16; c++) dst[i * 16 + c] = __float2bfloat16_rn(c < 3 ? src[i * 3 + c] : 0.f);
}
__global__ void unpack_din_kernel(long P, const bf16* __restrict__ src, float* __restrict__ dst) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) dst[i * 3 + c] = __bfloat162float(src[i * 16 + c]);
}

// blocks of 256 threads: for the flexible-PCG kernels (tpn threads per
// node), and for the training kernels (one thread per node)
int grid_nodes(int Nn, int tpn) { return (int)(((long)tpn * Nn + 255) / 256); }
int grid_nodes1(int Nn) { return (Nn + 255) / 256; }

// Nodes below which the flexible-PCG kernels run two threads per node
// (measured: plate_q4_141, 20,164 nodes, K products 10-20% faster with two;
// plate_q4_400, 160,801 nodes, 15% slower)
constexpr int kTwoThreadNodes = 75000;

// Buffers of a flexible-PCG solver for an operator with Nn nodes.
// The node-block form of S's operator (Op::nm_*): slice widths on the
// device, their offsets on the host, then the columns and blocks.  A mesh
// with a node of more than kMaxNbr neighbours keeps the element gather.
void build_node_blocks(FpcgSolver* S, cudaStream_t st) {
    const int Nn = S->op.Nn;
    if (Nn < 1 || !S->op.ke64) return;
    const int Ns = (Nn + 31) / 32;
    const int grid = (int)(((long)Ns * 32 + 255) / 256);
    Buf<int> width, bad;
    width.alloc(Ns);
    bad.alloc(1);
    bad.zero(st);
    (S->npe == 4 ? nm_width_kernel<4> : nm_width_kernel<3>)<<<grid, 256, 0, st>>>(S->op, Ns, width.p, bad.p);
    LCK(cudaGetLastError());
    std::vector<int> w(Ns);
    int hb = 0;
    LCK(cudaMemcpyAsync(w.data(), width.p, Ns * sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    if (hb) return;
    std::vector<int> off(Ns + 1, 0);
    for (int k = 0; k < Ns; k++) off[k + 1] = off[k] + w[k];
    S->nm_off.alloc(Ns + 1);
    S->nm_col.alloc(32 * (size_t)std::max(1, off[Ns]));
    S->nm_val.alloc(288 * (size_t)std::max(1, off[Ns]));
    LCK(cudaMemcpyAsync(S->nm_off.p, off.data(), (Ns + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
    (S->npe == 4 ? nm_fill_kernel<4> : nm_fill_kernel<3>)<<<grid, 256, 0, st>>>(S->op, Ns, S->nm_off.p,
                                                                              S->nm_col.p, S->nm_val.p);
    LCK(cudaGetLastError());
    LCK(cudaStreamSynchronize(st));  // off leaves scope
    S->op.nm_off = S->nm_off.p;
    S->op.nm_col = S->nm_col.p;
    S->op.nm_val = S->nm_val.p;
}

void fpcg_init(FpcgSolver* S, pg_ctx* c, const Op& op, int npe, float omega) {
    S->ctx = c;
    S->op = op;
    S->npe = npe;
    S->omega = omega;
    cudaStream_t st = pgi::ctx_stream(c);
    const size_t n3 = 3 * (size_t)op.Nn;
    for (Buf<float>* b : {&S->F, &S->r, &S->r_prev, &S->r1, &S->y, &S->r2, &S->z, &S->p0, &S->p1, &S->q, &S->y2,
                          &S->v2, &S->t}) {
        b->alloc(n3);
        b->zero(st);
    }
    S->x.alloc(n3);
    S->op.tpn = op.Nn < kTwoThreadNodes ? 2 : 1;
    S->parts.alloc(14 * (size_t)grid_nodes(op.Nn, S->op.tpn));
    S->st.alloc(1);
    LCK(cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking));
    build_node_blocks(S, st);
    LCK(cudaStreamSynchronize(st));
}

// The kernels of one flexible-PCG iteration, on cs.  in_graph: the tick
// sets the WHILE node's condition.  ev (9 events, optional) brackets the
// groups update, true residual, smoothing + network input, network, K y +
// sweeps, preconditioner, direction + K p, tick for timing.
void queue_body(FpcgSolver* S, const FArgs& a, int mode, pg_net* n, Workspace* w, cudaStream_t cs, bool pdl,
                cudaGraphConditionalHandle h, bool in_graph, cudaEvent_t* ev) {
    const int G = a.G;
    const bool q4 = S->npe == 4;
    auto mark = [&](int k) {
        if (ev) LCK(cudaEventRecord(ev[k], cs));
    };
    mark(0);
    fp_update_kernel<<<G, 256, 0, cs>>>(a);
    LCK(cudaGetLastError());
    mark(1);
    launch(pdl, q4 ? fp_true_res_kernel<4> : fp_true_res_kernel<3>, dim3(G), dim3(256), 0, cs, a);
    mark(2);
    launch(pdl, q4 ? fp_prep_kernel<4> : fp_prep_kernel<3>, dim3(G), dim3(256), 0, cs, a);
    mark(3);
    FArgs ac = a;  // the preconditioner reads the correction after the sweeps
    if (mode == 1) {
        net_forward(n, w, cs, &S->st.p->skip_net, pdl);
        mark(4);
        // w_0 = y in a.y with v_0 in a.r2; sweep k's w_k alternates between
        // a.y2 (odd k) and a.y, its v_k between a.v2 and a.r2
        float* w_cur = a.y;
        float* v_cur = a.r2;
        float* w_nxt = kCorrectionSweeps > 0 ? a.y2 : nullptr;
        launch(pdl, q4 ? fp_net_kernel<4> : fp_net_kernel<3>, dim3(G), dim3(256), 0, cs, a, w_nxt);
        for (int k = 1; k <= kCorrectionSweeps; k++) {
            w_cur = w_nxt;
            v_cur = (k & 1) ? a.v2 : a.r2;
            w_nxt = k < kCorrectionSweeps ? (w_cur == a.y2 ? a.y : a.y2) : nullptr;
            launch(pdl, q4 ? fp_sweep_kernel<4> : fp_sweep_kernel<3>, dim3(G), dim3(256), 0, cs, a,
                   (const float*)w_cur, v_cur, w_nxt);
        }
        ac.y = w_cur;
        ac.r2 = v_cur;
    } else {
        mark(4);
    }
    mark(5);
    launch(pdl, fp_prec_kernel, dim3(G), dim3(256), 0, cs, ac);
    mark(6);
    launch(pdl, q4 ? fp_dir_kernel<4> : fp_dir_kernel<3>, dim3(G), dim3(256), 0, cs, a);
    mark(7);
    launch(pdl, fp_tick_kernel, dim3(1), dim3(1), 0, cs, a, h, in_graph ? 1 : 0);
    mark(8);
}

// Builds the solve graph of S: an init node, then a conditional WHILE node
// whose body is one flexible-PCG iteration (mode 1 includes the network
// forward pass on net's batch-1 workspace).
// The kernel arguments of S's iteration for these options and mode (w: the
// network's batch-1 workspace in mode 1).
FArgs make_fargs(FpcgSolver* S, const pg_options& o, int mode, pg_net* n, Workspace* w, const int* node_pixel,
                 int HW, int fallback_after, int replace_every) {
    const int G = grid_nodes(S->op.Nn, S->op.tpn);
    FArgs a{};
    a.op = S->op;
    a.HW = HW;
    a.node_pixel = node_pixel;
    a.img_in = w ? w->in.p : nullptr;
    a.img_out = w ? w->out.p : nullptr;
    const float one[6] = {1, 1, 1, 1, 1, 1};
    const float* sc = n ? n->scale : one;
    a.si0 = sc[0];
    a.si1 = sc[1];
    a.si2 = sc[2];
    a.so0 = sc[3];
    a.so1 = sc[4];
    a.so2 = sc[5];
    a.omega = S->omega;
    a.F = S->F.p;
    a.x = S->x.p;
    a.r = S->r.p;
    a.r_prev = S->r_prev.p;
    a.r1 = S->r1.p;
    a.y = S->y.p;
    a.r2 = S->r2.p;
    a.y2 = S->y2.p;
    a.v2 = S->v2.p;
    a.t = S->t.p;
    a.z = S->z.p;
    a.p0 = S->p0.p;
    a.p1 = S->p1.p;
    a.q = S->q.p;
    double* P = S->parts.p;
    a.pU = P;
    a.pTR = P + 2 * G;
    a.pA = P + 4 * G;
    a.pB = P + 6 * G;
    a.pC = P + 8 * G;
    a.pD = P + 10 * G;
    a.pI = P + 12 * G;
    a.st = S->st.p;
    a.G = G;
    a.tol2 = o.tolerance * o.tolerance;
    a.stop_rule = o.stop_rule;
    a.maxit = o.max_iterations;
    a.replace_every = replace_every;
    a.mode = mode;
    a.fallback_after = fallback_after;
    return a;
}

void fpcg_build(FpcgSolver* S, const pg_options& o, int mode, pg_net* n, const int* node_pixel, int HW,
                int fallback_after, int replace_every, bool pdl) {
    cudaStream_t cs = S->cap;
    Workspace* w = mode == 1 ? workspace(n, 1, false) : nullptr;
    const int G = grid_nodes(S->op.Nn, S->op.tpn);
    FArgs a = make_fargs(S, o, mode, n, w, node_pixel, HW, fallback_after, replace_every);

    if (S->exec) {
        cudaGraphExecDestroy(S->exec);
        S->exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    LCK(cudaGraphCreate(&g, 0));
    try {
        cudaGraphConditionalHandle h;
        LCK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        // the state and vectors are reset by the first node, before the loop
        cudaGraphNode_t init_node, loop;
        cudaKernelNodeParams kp{};
        void* init_args[] = {&a};
        kp.func = (void*)fp_init_kernel;
        kp.gridDim = dim3(G);
        kp.blockDim = dim3(256);
        kp.kernelParams = init_args;
        LCK(cudaGraphAddKernelNode(&init_node, g, nullptr, 0, &kp));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        LCK(cudaGraphAddNode(&loop, g, &init_node, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        LCK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        // every kernel after the body's first may start while its predecessor
        // finishes (pdl); each waits in pdl_wait before reading
        cudaError_t ce = cudaSuccess;
        try {
            queue_body(S, a, mode, n, w, cs, pdl, h, true, nullptr);
            ce = cudaGetLastError();
        } catch (const LFail&) {
            cudaGraph_t got = nullptr;
            cudaStreamEndCapture(cs, &got);
            cudaGetLastError();
            throw;
        }
        cudaGraph_t got = nullptr;
        cudaError_t ee = cudaStreamEndCapture(cs, &got);
        LCK(ce);
        LCK(ee);
        LCK(cudaGraphInstantiate(&S->exec, g, 0));
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    S->pdl = pdl;
    cudaGraphDestroy(g);
    S->mode = mode;
    S->version = n ? n->version : 0;
    S->maxit = o.max_iterations;
    S->rule = o.stop_rule;
    S->tol = o.tolerance;
}

// One solve with S (graph rebuilt when the options, the mode or the
// network's scales changed).  F and x on the host or the device.
void fpcg_run(FpcgSolver* S, const pg_options& o, int mode, pg_net* n, const int* node_pixel, int HW,
              const float* F, bool host_F, double* x_out, bool host_x, pg_info* info, pg_learned_stats* ls) {
    if (!(o.tolerance >= 0) || o.max_iterations < 0) throw LFail{PG_EINVAL, "bad tolerance / max_iterations"};
    if (!F || !x_out) throw LFail{PG_EINVAL, "F / x is NULL"};
    cudaStream_t st = pgi::ctx_stream(S->ctx);
    const size_t n3 = 3 * (size_t)S->op.Nn;
    auto t0 = std::chrono::steady_clock::now();
    if (!S->exec || S->mode != mode || S->maxit != o.max_iterations || S->rule != o.stop_rule ||
        S->tol != o.tolerance || S->version != (n ? n->version : 0)) {
        // with programmatic dependent launch where the driver takes it in a
        // captured conditional body, else without
        try {
            fpcg_build(S, o, mode, n, node_pixel, HW, 3, 50, !S->pdl_refused);
        } catch (const LFail&) {
            if (S->pdl_refused) throw;
            S->pdl_refused = true;
            fpcg_build(S, o, mode, n, node_pixel, HW, 3, 50, false);
        }
    }
    if (host_F) {
        for (size_t i = 0; i < n3; i++)
            if (!std::isfinite(F[i])) throw LFail{PG_ENONFINITE, "F contains NaN or Inf"};
    }
    LCK(cudaMemcpyAsync(S->F.p, F, n3 * sizeof(float), host_F ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                        st));
    cudaEvent_t e0, e1;
    LCK(cudaEventCreate(&e0));
    LCK(cudaEventCreate(&e1));
    double phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int timed_its = 0;
    LCK(cudaEventRecord(e0, st));
    if (!o.phase_timing) {
        LCK(cudaGraphLaunch(S->exec, st));
    } else {
        // the same kernels without the graph (profilers cannot look inside a
        // graph with conditional nodes): each iteration's kernel groups timed
        // with events, and the host reading the stop flag after every
        // iteration (so solve_ms includes those waits)
        Workspace* w = mode == 1 ? workspace(n, 1, false) : nullptr;
        const FArgs a = make_fargs(S, o, mode, n, w, node_pixel, HW, 3, 50);
        fp_init_kernel<<<a.G, 256, 0, st>>>(a);
        LCK(cudaGetLastError());
        cudaEvent_t ev[9];
        for (auto& e : ev) LCK(cudaEventCreate(&e));
        for (int it = 0; it <= o.max_iterations + 1; it++) {
            queue_body(S, a, mode, n, w, st, false, 0, false, ev);
            int done = 0;
            LCK(cudaMemcpyAsync(&done, &S->st.p->done, sizeof(int), cudaMemcpyDeviceToHost, st));
            LCK(cudaStreamSynchronize(st));
            for (int k = 0; k < 8; k++) {
                float ms = 0;
                LCK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
                phase[k] += ms;
            }
            timed_its++;
            if (done) break;
        }
        for (auto& e : ev) cudaEventDestroy(e);
    }
    LCK(cudaEventRecord(e1, st));
    LCK(cudaMemcpyAsync(x_out, S->x.p, n3 * sizeof(double),
                        host_x ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
    FState s{};
    LCK(cudaMemcpyAsync(&s, S->st.p, sizeof s, cudaMemcpyDeviceToHost, st));
    LCK(cudaStreamSynchronize(st));
    float ms = 0;
    LCK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s.error) throw LFail{PG_ENONFINITE, "non-finite value in the flexible PCG iteration"};
    if (info) {
        info->iterations = s.iterations;
        info->converged = s.converged;
        info->stop_reason = s.stop_reason;
        info->b_norm = std::sqrt(s.bnorm2);
        info->final_residual = std::sqrt(s.true_rr);
        info->true_rel_residual = s.bnorm2 > 0 ? std::sqrt(s.true_rr / s.bnorm2) : 0.0;
        info->solve_ms = ms;
        info->reliable_updates = s.replacements;
        info->reductions = s.iterations;
        info->plan_cached = 1;
        info->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        for (int k = 0; k < 8; k++) info->phase_us[k] = timed_its ? 1e3 * phase[k] / timed_its : 0.0;
    }
    if (ls) {
        ls->network_iterations = s.net_iters;
        ls->network_off_at = s.net_off ? s.net_off_at : -1;
        ls->replacements = s.replacements;
        ls->mode = mode;
        ls->pdl = S->pdl;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

int pg_net_create(pg_ctx* ctx, int height, int width, uint64_t seed, pg_net** out) {
    if (out) *out = nullptr;
    return lguarded(ctx, [&] {
        if (!out) throw LFail{PG_EINVAL, "out is NULL"};
        if (height < 8 || width < 8 || height % 8 || width % 8 || (long)height * width > (1L << 22))
            throw LFail{PG_EINVAL, "network grid must be at least 8 x 8, multiples of 8, at most 4M pixels"};
        auto n = std::make_unique<pg_net>();
        n->ctx = ctx;
        n->H = height;
        n->W = width;
        n->T = make_table();
        const size_t tot = (size_t)n->T.total;
        n->w.alloc(tot);
        n->m.alloc(tot);
        n->v.alloc(tot);
        n->g.alloc(tot);
        n->wf.alloc(tot);
        n->wd.alloc(tot);
        n->step.alloc(1);
        cudaStream_t st = pgi::ctx_stream(ctx);
        // He-normal initialisation (std sqrt(2 / (9 cin)), sqrt(1 / (9 cin)) for
        // the linear output layer), padded weights 0
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd(0.0, 1.0);
        std::vector<float> real((size_t)real_param_count()), pad;
        long k = 0;
        for (int l = 0; l < pgn::kLayers; l++) {
            const double sd = std::sqrt((l == OUTL ? 1.0 : 2.0) / (9.0 * kSpec[l].cin));
            for (long i = 0; i < 9L * kSpec[l].cin * kSpec[l].cout; i++) real[k++] = (float)(sd * nd(rng));
        }
        real_to_padded(n.get(), real.data(), pad);
        LCK(cudaMemcpyAsync(n->w.p, pad.data(), tot * sizeof(float), cudaMemcpyHostToDevice, st));
        n->m.zero(st);
        n->v.zero(st);
        n->g.zero(st);
        n->step.zero(st);
        refresh_bf16(n.get(), st);
        LCK(cudaStreamSynchronize(st));
        *out = n.release();
    });
}

void pg_net_destroy(pg_net* n) {
    if (!n) return;
    {
        std::lock_guard<std::mutex> lk(pgi::ctx_mutex(n->ctx));
        cudaSetDevice(pgi::ctx_device(n->ctx));
        cudaStreamSynchronize(pgi::ctx_stream(n->ctx));
        n->ws.clear();
    }
    delete n;
}

int64_t pg_net_param_count(const pg_net* n) { return n ? real_param_count() : 0; }

int pg_net_set_params(pg_net* n, const float* params, const float* scales) {
    if (!n) return PG_EINVAL;
    return lguarded(n->ctx, [&] {
        cudaStream_t st = pgi::ctx_stream(n->ctx);
        if (params) {
            std::vector<float> pad;
            real_to_padded(n, params, pad);
            LCK(cudaMemcpyAsync(n->w.p, pad.data(), pad.size() * sizeof(float), cudaMemcpyHostToDevice, st));
            refresh_bf16(n, st);
            n->m.zero(st);
            n->v.zero(st);
            n->step.zero(st);
        }
        if (scales) {
            for (int i = 0; i < 6; i++)
                if (!(scales[i] > 0) || !std::isfinite(scales[i])) throw LFail{PG_EINVAL, "scales must be > 0"};
            std::memcpy(n->scale, scales, sizeof n->scale);
            n->version++;
        }
        LCK(cudaStreamSynchronize(st));
    });
}

int pg_net_get_params(pg_net* n, float* params, float* scales) {
    if (!n) return PG_EINVAL;
    return lguarded(n->ctx, [&] {
        cudaStream_t st = pgi::ctx_stream(n->ctx);
        if (params) {
            std::vector<float> pad(n->T.total);
            LCK(cudaMemcpyAsync(pad.data(), n->w.p, pad.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
            LCK(cudaStreamSynchronize(st));
            padded_to_real(n, pad, params);
        }
        if (scales) std::memcpy(scales, n->scale, sizeof n->scale);
    });
}

int pg_net_forward(pg_net* n, int batch, const float* in_dev, float* out_dev) {
    if (!n) return PG_EINVAL;
    return lguarded(n->ctx, [&] {
        if (batch < 1 || !in_dev || !out_dev) throw LFail{PG_EINVAL, "batch < 1 or NULL buffer"};
        cudaStream_t st = pgi::ctx_stream(n->ctx);
        Workspace* w = workspace(n, batch, true);
        const long P = (long)batch * n->H * n->W;
        pack_in_kernel<<<ew_grid(P), 256, 0, st>>>(P, in_dev, w->in.p);
        net_forward(n, w, st, nullptr);
        unpack_out_kernel<<<ew_grid(P), 256, 0, st>>>(P, w->out.p, out_dev);
        LCK(cudaGetLastError());
        LCK(cudaStreamSynchronize(st));
    });
}

int pg_net_backward(pg_net* n, int batch, const float* gout_dev, float* gin_dev, float* gparams) {
    if (!n) return PG_EINVAL;
    return lguarded(n->ctx, [&] {
        if (batch < 1 || !gout_dev) throw LFail{PG_EINVAL, "batch < 1 or NULL buffer"};
        auto it = n->ws.find(batch);
        if (it == n->ws.end() || !it->second->grads) throw LFail{PG_EINVAL, "call pg_net_forward first"};
        Workspace* w = it->second.get();
        cudaStream_t st = pgi::ctx_stream(n->ctx);
        const long P = (long)batch * n->H * n->W;
        pack_gout_kernel<<<ew_grid(P), 256, 0, st>>>(P, gout_dev, w->gout.p);
        n->g.zero(st);
        net_backward(n, w, st, gin_dev != nullptr);
        if (gin_dev) unpack_din_kernel<<<ew_grid(P), 256, 0, st>>>(P, w->din.p, gin_dev);
        LCK(cudaGetLastError());
        if (gparams) {
            std::vector<float> pad(n->T.total);
            LCK(cudaMemcpyAsync(pad.data(), n->g.p, pad.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
            LCK(cudaStreamSynchronize(st));
            padded_to_real(n, pad, gparams);
        }
        LCK(cudaStreamSynchronize(st));
    });
}

int pg_net_adam_step(pg_net* n, const float* grads, float lr) {
    if (!n) return PG_EINVAL;
    return lguarded(n->ctx, [&] {
        if (!grads) throw LFail{PG_EINVAL, "grads is NULL"};
        cudaStream_t st = pgi::ctx_stream(n->ctx);
        std::vector<float> pad;
        real_to_padded(n, grads, pad);
        LCK(cudaMemcpyAsync(n->g.p, pad.data(), pad.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        step_begin_kernel<<<1, 1, 0, st>>>(n->step.p);
        pgn::adam_kernel<<<ew_grid(n->T.total), 256, 0, st>>>(n->T, n->w.p, n->m.p, n->v.p, n->g.p, n->step.p, lr,
                                                              0.9f, 0.999f, 1e-8f, 0, n->wf.p, n->wd.p);
        LCK(cudaGetLastError());
        LCK(cudaStreamSynchronize(st));
    });
}

int pg_learned_create(pg_plan* plan, pg_net* net, const int32_t* node_pixel, pg_learned** out) {
    if (out) *out = nullptr;
    if (!plan || !net) return PG_EINVAL;
    pg_ctx* c = pgi::plan_ctx(plan);
    if (c != net->ctx) return PG_EINVAL;
    return lguarded(c, [&] {
        if (!out || !node_pixel) throw LFail{PG_EINVAL, "out / node_pixel is NULL"};
        auto L = std::make_unique<pg_learned>();
        L->plan = plan;
        L->net = net;
        L->ctx = c;
        std::string e = pgi::plan_operator(plan, &L->ov);
        if (!e.empty()) throw LFail{PG_ECUDA, e};
        if (L->ov.npe != 4 && L->ov.npe != 3) throw LFail{PG_EINVAL, "unsupported element type"};
        L->op = make_op(L->ov, pgi::ctx_stream(c));
        L->HW = net->H * net->W;
        const int Nn = L->ov.Nn;
        std::vector<char> seen(L->HW, 0);
        for (int i = 0; i < Nn; i++) {
            const int px = node_pixel[i];
            if (px < 0 || px >= L->HW || seen[px])
                throw LFail{PG_EINVAL, "node_pixel must map every node to a distinct pixel of the grid"};
            seen[px] = 1;
        }
        cudaStream_t st = pgi::ctx_stream(c);
        L->node_pixel.alloc(Nn);
        LCK(cudaMemcpyAsync(L->node_pixel.p, node_pixel, Nn * sizeof(int), cudaMemcpyHostToDevice, st));
        L->stats.alloc(6);
        // damped smoothing steps: omega lambda_max(D^-1 K) <= 1.5 keeps the
        // pre-/post-smoothing pair positive definite (plates have lambda_max
        // just above 2)
        const double lam = pgi::plan_lambda_max(plan);
        L->omega = (float)std::min(1.0, 1.5 / std::max(lam, 1e-30));
        fpcg_init(&L->S, c, L->op, L->ov.npe, L->omega);
        *out = L.release();
    });
}

void pg_learned_destroy(pg_learned* L) {
    if (!L) return;
    {
        std::lock_guard<std::mutex> lk(pgi::ctx_mutex(L->ctx));
        cudaSetDevice(pgi::ctx_device(L->ctx));
        cudaStreamSynchronize(pgi::ctx_stream(L->ctx));
    }
    delete L;
}

int pg_learned_make_pairs(pg_learned* L, int count, const float* F_dev, const double* xstar_dev,
                          const double* xk_dev, float* R_out, float* E_out) {
    if (!L) return PG_EINVAL;
    return lguarded(L->ctx, [&] {
        if (count < 0 || (count > 0 && (!F_dev || !xstar_dev || !R_out || !E_out)))
            throw LFail{PG_EINVAL, "NULL buffer"};
        if (count == 0) return;
        cudaStream_t st = pgi::ctx_stream(L->ctx);
        dim3 grid(grid_nodes1(L->op.Nn), count);
        if (L->ov.npe == 4)
            make_pairs_kernel<4><<<grid, 256, 0, st>>>(L->op, count, F_dev, xstar_dev, xk_dev, R_out, E_out);
        else
            make_pairs_kernel<3><<<grid, 256, 0, st>>>(L->op, count, F_dev, xstar_dev, xk_dev, R_out, E_out);
        LCK(cudaGetLastError());
        LCK(cudaStreamSynchronize(st));
    });
}

namespace {

// Pre-smooths `count` pairs into the training set (replacing it).  With
// set_scales, the network's input / output scales become 1 / rms(r1_c)
// and rms(e1_c) over the pairs.
void load_pairs(pg_learned* L, int count, const float* R, const float* E, bool set_scales) {
    pg_net* n = L->net;
    cudaStream_t st = pgi::ctx_stream(L->ctx);
    dim3 grid(grid_nodes1(L->op.Nn), count);
    if (set_scales) {
        L->stats.zero(st);
        if (L->ov.npe == 4)
            prep_pairs_kernel<4><<<grid, 256, 0, st>>>(L->op, count, R, E, L->node_pixel.p, L->HW, 0, L->omega, 1, 1, 1,
                                                        1, 1, 1, L->stats.p, nullptr, nullptr, nullptr, nullptr);
        else
            prep_pairs_kernel<3><<<grid, 256, 0, st>>>(L->op, count, R, E, L->node_pixel.p, L->HW, 0, L->omega, 1, 1, 1,
                                                        1, 1, 1, L->stats.p, nullptr, nullptr, nullptr, nullptr);
        LCK(cudaGetLastError());
        double s[6];
        LCK(cudaMemcpyAsync(s, L->stats.p, sizeof s, cudaMemcpyDeviceToHost, st));
        LCK(cudaStreamSynchronize(st));
        const double cnt = (double)count * L->op.Nn;
        for (int d = 0; d < 3; d++) {
            const double ri = std::sqrt(s[d] / cnt), eo = std::sqrt(s[3 + d] / cnt);
            n->scale[d] = ri > 0 && std::isfinite(ri) ? (float)(1.0 / ri) : 1.f;
            n->scale[3 + d] = eo > 0 && std::isfinite(eo) ? (float)eo : 1.f;
        }
        n->version++;
    }
    L->P = count;
    L->img.alloc((size_t)count * L->HW * 4);
    L->img.zero(st);
    L->E1.alloc((size_t)count * 3 * L->op.Nn);
    L->den.alloc(count);
    L->den.zero(st);
    L->den2.alloc(count);
    L->den2.zero(st);
    if (L->ov.npe == 4)
        prep_pairs_kernel<4><<<grid, 256, 0, st>>>(L->op, count, R, E, L->node_pixel.p, L->HW, 1, L->omega, n->scale[0],
                                                    n->scale[1], n->scale[2], n->scale[3], n->scale[4], n->scale[5],
                                                    nullptr, L->img.p, L->E1.p, L->den.p, L->den2.p);
    else
        prep_pairs_kernel<3><<<grid, 256, 0, st>>>(L->op, count, R, E, L->node_pixel.p, L->HW, 1, L->omega, n->scale[0],
                                                    n->scale[1], n->scale[2], n->scale[3], n->scale[4], n->scale[5],
                                                    nullptr, L->img.p, L->E1.p, L->den.p, L->den2.p);
    LCK(cudaGetLastError());
    LCK(cudaStreamSynchronize(st));
}

// Queues the loss of a batch (outputs `out`, pair ids via perm/step) into
// loss_hist, and with gout its gradient with respect to the network output.
void queue_loss(pg_learned* L, int B, const float* out, const int* perm, const int* step, int kind,
                double* loss_hist, bf16* gout, cudaStream_t st) {
    pg_net* n = L->net;
    const Op& op = L->op;
    dim3 grid(grid_nodes1(op.Nn), B);
    const bool q4 = L->ov.npe == 4;
    if (kind != PG_LOSS_SMOOTHED_ENERGY) {
        auto k = q4 ? loss_kernel<4> : loss_kernel<3>;
        k<<<grid, 256, 0, st>>>(op, B, L->HW, L->node_pixel.p, out, L->E1.p, L->den.p, L->den2.p, kind, perm, step,
                                n->scale[3], n->scale[4], n->scale[5], loss_hist, gout);
        LCK(cudaGetLastError());
        return;
    }
    if (L->sl_batch < B) {
        L->sg.alloc((size_t)B * 3 * op.Nn);
        L->sh.alloc((size_t)B * 3 * op.Nn);
        L->sl_batch = B;
    }
    float *g = L->sg.p, *h = L->sh.p;
    sl_diff_kernel<<<grid, 256, 0, st>>>(op, B, L->HW, L->node_pixel.p, out, L->E1.p, perm, step, n->scale[3],
                                         n->scale[4], n->scale[5], g);
    for (int k = 0; k < kCorrectionSweeps; k++) {
        (q4 ? sl_sweep_kernel<4> : sl_sweep_kernel<3>)<<<grid, 256, 0, st>>>(op, L->omega, g, h);
        std::swap(g, h);
    }
    (q4 ? sl_energy_kernel<4> : sl_energy_kernel<3>)<<<grid, 256, 0, st>>>(op, B, g, h, L->den.p, perm, step,
                                                                          loss_hist);
    std::swap(g, h);  // g = K M^nu d
    if (gout) {
        for (int k = 0; k < kCorrectionSweeps; k++) {
            (q4 ? sl_bsweep_kernel<4> : sl_bsweep_kernel<3>)<<<grid, 256, 0, st>>>(op, L->omega, g, h);
            std::swap(g, h);
        }
        sl_grad_kernel<<<grid, 256, 0, st>>>(op, B, L->HW, L->node_pixel.p, g, L->den.p, perm, step, n->scale[3],
                                             n->scale[4], n->scale[5], gout);
    }
    LCK(cudaGetLastError());
}

// Mean loss of pairs [first, first + count) of the training set (forward
// passes of up to `batch` pairs, no gradient); per-pair losses into per
// (host, optional).
double eval_loss(pg_learned* L, int first, int count, int batch, double* per) {
    pg_net* n = L->net;
    cudaStream_t st = pgi::ctx_stream(L->ctx);
    Workspace* w = workspace(n, batch, false);
    Buf<int> idx;
    idx.alloc(batch);
    Buf<double> acc;
    acc.alloc(1);
    double total = 0.0;
    std::vector<int> ids(batch);
    for (int s = 0; s < count; s += batch) {
        const int b = std::min(batch, count - s);
        for (int i = 0; i < batch; i++) ids[i] = first + s + std::min(i, b - 1);
        LCK(cudaMemcpyAsync(idx.p, ids.data(), batch * sizeof(int), cudaMemcpyHostToDevice, st));
        gather_batch_kernel<<<ew_grid((long)batch * L->HW), 256, 0, st>>>(batch, L->HW, L->img.p, idx.p, nullptr,
                                                                        w->in.p);
        net_forward(n, w, st, nullptr);
        for (int i = 0; i < b; i++) {
            // one pair at a time so each pair's loss is separate (B = 1 scaling)
            acc.zero(st);
            const float* outb = w->out.p + (size_t)i * L->HW * 4;
            queue_loss(L, 1, outb, idx.p + i, nullptr, PG_LOSS_SMOOTHED_ENERGY, acc.p, nullptr, st);
            double v = 0;
            LCK(cudaMemcpyAsync(&v, acc.p, sizeof v, cudaMemcpyDeviceToHost, st));
            LCK(cudaStreamSynchronize(st));
            if (per) per[s + i] = v;
            total += v;
        }
    }
    return count > 0 ? total / count : 0.0;
}

void build_train_graph(pg_learned* L, int B, int total_steps, float lr, bool cosine, int loss_kind) {
    pg_net* n = L->net;
    Workspace* w = workspace(n, B, true);
    if (L->sl_batch < B) {  // before the capture: no allocation inside it
        L->sg.alloc((size_t)B * 3 * L->op.Nn);
        L->sh.alloc((size_t)B * 3 * L->op.Nn);
        L->sl_batch = B;
    }
    cudaStream_t cs = L->S.cap;
    if (L->train_exec) {
        cudaGraphExecDestroy(L->train_exec);
        L->train_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    LCK(cudaGraphCreate(&g, 0));
    try {
        cudaGraphConditionalHandle h;
        LCK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        LCK(cudaGraphAddNode(&loop, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        LCK(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        step_begin_kernel<<<1, 1, 0, cs>>>(n->step.p);
        cudaMemsetAsync(n->g.p, 0, n->g.n * sizeof(float), cs);
        gather_batch_kernel<<<ew_grid((long)B * L->HW), 256, 0, cs>>>(B, L->HW, L->img.p, L->perm.p, n->step.p,
                                                                    w->in.p);
        net_forward(n, w, cs, nullptr);
        queue_loss(L, B, w->out.p, L->perm.p, n->step.p, loss_kind, L->loss_hist.p, w->gout.p, cs);
        net_backward(n, w, cs, false);
        pgn::adam_kernel<<<ew_grid(n->T.total), 256, 0, cs>>>(n->T, n->w.p, n->m.p, n->v.p, n->g.p, n->step.p, lr,
                                                              0.9f, 0.999f, 1e-8f, cosine ? total_steps : 0,
                                                              n->wf.p, n->wd.p);
        train_tick_kernel<<<1, 1, 0, cs>>>(h, n->step.p, L->stop_step.p);
        cudaError_t ce = cudaGetLastError();
        cudaGraph_t got = nullptr;
        cudaError_t ee = cudaStreamEndCapture(cs, &got);
        LCK(ce);
        LCK(ee);
        LCK(cudaGraphInstantiate(&L->train_exec, g, 0));
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraphDestroy(g);
    L->train_B = B;
}

}  // namespace

void pg_train_options_default(pg_train_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->struct_size = sizeof *o;
    o->epochs = 20;
    o->batch = 32;
    o->lr = 1e-3f;
    o->cosine = 1;
    o->seed = 1;
    o->val_count = 0;
    o->set_scales = 1;
    o->loss = PG_LOSS_ENERGY;
}

int pg_learned_train(pg_learned* L, int count, const float* R_dev, const float* E_dev,
                     const pg_train_options* opt, pg_train_info* info) {
    if (!L) return PG_EINVAL;
    if (info) std::memset(info, 0, sizeof *info);
    return lguarded(L->ctx, [&] {
        pg_train_options o;
        pg_train_options_default(&o);
        if (opt) {
            if (opt->struct_size != sizeof(pg_train_options)) throw LFail{PG_EINVAL, "pg_train_options size mismatch"};
            o = *opt;
        }
        if (count < 2 || !R_dev || !E_dev) throw LFail{PG_EINVAL, "need at least 2 pairs"};
        if (o.batch < 1 || o.epochs < 0 || !(o.lr > 0) || o.val_count < 0 || o.val_count >= count)
            throw LFail{PG_EINVAL, "bad training options"};
        if (o.epochs > PG_TRAIN_MAX_EPOCHS) throw LFail{PG_EINVAL, "too many epochs"};
        if (o.loss != PG_LOSS_ENERGY && o.loss != PG_LOSS_SCALED_L2 && o.loss != PG_LOSS_SMOOTHED_ENERGY)
            throw LFail{PG_EINVAL, "unknown loss"};
        pg_net* n = L->net;
        cudaStream_t st = pgi::ctx_stream(L->ctx);
        auto t0 = std::chrono::steady_clock::now();
        load_pairs(L, count, R_dev, E_dev, o.set_scales != 0);
        const int ntrain = count - o.val_count;
        const int B = std::min(o.batch, ntrain);
        const int spe = ntrain / B;  // steps per epoch (the remainder of a shuffle is left out)
        const int total = spe * o.epochs;
        // one shuffle of the training pairs per epoch, all uploaded at once
        std::mt19937_64 rng(o.seed);
        std::vector<int> perm((size_t)std::max(1, total) * B), ids(ntrain);
        for (int e = 0; e < o.epochs; e++) {
            for (int i = 0; i < ntrain; i++) ids[i] = i;
            std::shuffle(ids.begin(), ids.end(), rng);
            std::copy(ids.begin(), ids.begin() + (size_t)spe * B, perm.begin() + (size_t)e * spe * B);
        }
        L->perm.alloc(perm.size());
        LCK(cudaMemcpyAsync(L->perm.p, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        L->loss_hist.alloc(std::max(1, total));
        L->loss_hist.zero(st);
        L->stop_step.alloc(1);
        n->step.zero(st);
        n->m.zero(st);
        n->v.zero(st);
        const int vb = std::min(64, std::max(1, o.val_count));
        if (info) {
            info->val_loss_before = o.val_count ? eval_loss(L, ntrain, o.val_count, vb, nullptr) : 0.0;
            info->steps = total;
            info->batch = B;
        }
        if (total > 0) {
            build_train_graph(L, B, total, o.lr, o.cosine != 0, o.loss);
            double tms = 0.0;
            cudaEvent_t e0, e1;
            LCK(cudaEventCreate(&e0));
            LCK(cudaEventCreate(&e1));
            for (int e = 0; e < o.epochs; e++) {
                const int stop = (e + 1) * spe;
                LCK(cudaMemcpyAsync(L->stop_step.p, &stop, sizeof stop, cudaMemcpyHostToDevice, st));
                LCK(cudaEventRecord(e0, st));
                LCK(cudaGraphLaunch(L->train_exec, st));
                LCK(cudaEventRecord(e1, st));
                LCK(cudaStreamSynchronize(st));
                float ms = 0;
                LCK(cudaEventElapsedTime(&ms, e0, e1));
                tms += ms;
                if (info) {
                    std::vector<double> h(spe);
                    LCK(cudaMemcpy(h.data(), L->loss_hist.p + (size_t)e * spe, spe * sizeof(double),
                                   cudaMemcpyDeviceToHost));
                    double s = 0;
                    for (double v : h) s += v;
                    info->epoch_loss[e] = s / spe;
                    info->epoch_val_loss[e] = o.val_count ? eval_loss(L, ntrain, o.val_count, vb, nullptr) : 0.0;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            int steps_done = 0;
            LCK(cudaMemcpy(&steps_done, n->step.p, sizeof(int), cudaMemcpyDeviceToHost));
            if (steps_done != total) throw LFail{PG_ECUDA, "training graph ran an unexpected number of steps"};
            if (info) {
                info->train_ms = tms;
                double first = 0, last = 0;
                LCK(cudaMemcpy(&first, L->loss_hist.p, sizeof(double), cudaMemcpyDeviceToHost));
                LCK(cudaMemcpy(&last, L->loss_hist.p + total - 1, sizeof(double), cudaMemcpyDeviceToHost));
                info->loss_first_step = first;
                info->loss_last_step = last;
            }
        }
        if (info) {
            info->val_loss = o.val_count ? eval_loss(L, ntrain, o.val_count, vb, nullptr) : 0.0;
            info->total_ms =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

int pg_learned_loss(pg_learned* L, int count, const float* R_dev, const float* E_dev, double* loss_out) {
    if (!L) return PG_EINVAL;
    return lguarded(L->ctx, [&] {
        if (count < 1 || !R_dev || !E_dev || !loss_out) throw LFail{PG_EINVAL, "NULL buffer or count < 1"};
        load_pairs(L, count, R_dev, E_dev, false);
        eval_loss(L, 0, count, std::min(count, 16), loss_out);
    });
}

namespace {

void learned_solve(pg_learned* L, const pg_options* opt, int mode, const float* F, bool host, double* x_out,
                   pg_info* info, pg_learned_stats* ls) {
    pg_options o;
    pg_options_default(&o);
    if (opt) {
        if (opt->struct_size != sizeof(pg_options)) throw LFail{PG_EINVAL, "pg_options size mismatch"};
        o = *opt;
    }
    if (mode < 0 || mode > 2) throw LFail{PG_EINVAL, "mode must be 0, 1 or 2"};
    fpcg_run(&L->S, o, mode, L->net, L->node_pixel.p, L->HW, F, host, x_out, host, info, ls);
}

}  // namespace

int pg_learned_solve_device(pg_learned* L, const pg_options* opt, int mode, const float* F_dev, double* x_dev,
                            pg_info* info, pg_learned_stats* stats) {
    if (info) std::memset(info, 0, sizeof *info);
    if (!L) return PG_EINVAL;
    const int st = lguarded(L->ctx, [&] { learned_solve(L, opt, mode, F_dev, false, x_dev, info, stats); });
    if (info) info->status = st;
    return st;
}

int pg_learned_solve(pg_learned* L, const pg_options* opt, int mode, const float* F, double* x_out,
                     pg_info* info, pg_learned_stats* stats) {
    if (info) std::memset(info, 0, sizeof *info);
    if (!L) return PG_EINVAL;
    const int st = lguarded(L->ctx, [&] { learned_solve(L, opt, mode, F, true, x_out, info, stats); });
    if (info) info->status = st;
    return st;
}

int pg_learned_apply_k(pg_learned* L, const float* x, float* y) {
    if (!L) return PG_EINVAL;
    return lguarded(L->ctx, [&] {
        if (!x || !y) throw LFail{PG_EINVAL, "x / y is NULL"};
        const size_t n3 = 3 * (size_t)L->S.op.Nn;
        if (n3 == 0) return;
        cudaStream_t st = pgi::ctx_stream(L->ctx);
        Buf<float> dx, dy;
        dx.alloc(n3);
        dy.alloc(n3);
        LCK(cudaMemcpyAsync(dx.p, x, n3 * sizeof(float), cudaMemcpyHostToDevice, st));
        const int grid = grid_nodes(L->S.op.Nn, L->S.op.tpn);
        (L->S.npe == 4 ? apply_op_kernel<4> : apply_op_kernel<3>)<<<grid, 256, 0, st>>>(L->S.op, dx.p, dy.p);
        LCK(cudaGetLastError());
        LCK(cudaMemcpyAsync(y, dy.p, n3 * sizeof(float), cudaMemcpyDeviceToHost, st));
        LCK(cudaStreamSynchronize(st));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// global-memory path of plategpu.cu (plates past shared-memory capacity)
// ---------------------------------------------------------------------------

struct pgi::GlobalPcg {
    FpcgSolver S;
};

namespace pgi {

GlobalPcg* global_pcg_create(pg_ctx* c, const OperatorView& ov, double lambda_max, std::string* err) {
    try {
        auto g = std::make_unique<GlobalPcg>();
        const float omega = (float)std::min(1.0, 1.5 / std::max(lambda_max, 1e-30));
        fpcg_init(&g->S, c, make_op(ov, pgi::ctx_stream(c)), ov.npe, omega);
        return g.release();
    } catch (const LFail& f) {
        *err = f.msg;
        return nullptr;
    }
}

void global_pcg_destroy(GlobalPcg* g) { delete g; }

int global_pcg_solve(GlobalPcg* g, const pg_options& o, int mode, const float* F_dev, void* x_dst, bool x_host,
                     pg_info* info, std::string* err) {
    try {
        fpcg_run(&g->S, o, mode, nullptr, nullptr, 0, F_dev, false, static_cast<double*>(x_dst), x_host, info,
                 nullptr);
        return PG_OK;
    } catch (const LFail& f) {
        *err = f.msg;
        return f.status;
    }
}

}  // namespace pgi
