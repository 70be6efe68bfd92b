// Kernels of the learned preconditioner's network: a 4-level U-Net over the
// structured nodal grid (channels 16/32/64/128, 3 x 3 convolutions without
// bias, ReLU, 2 x 2 average pooling, nearest 2x upsampling, skip connections
// by channel concatenation), trained and applied on the GPU.
//
// Tensor-core path: every convolution -- forward, input gradient and
// weight gradient -- is an implicit GEMM on mma.sync.m16n8k16 with BF16
// operands and FP32 accumulation (the legacy tensor path; the layers are
// 16-192 channels wide on grids of 18^2-144^2 pixels, far below the tile
// sizes where tcgen05/TMEM pays off).  Operands are staged in shared memory
// with cp.async and read with ldmatrix (.trans where the GEMM needs the
// transposed tile); rows are padded to an odd multiple of 16 bytes so the
// eight rows of every ldmatrix land in distinct banks.
//
// Layouts: activations [B][H][W][cs] BF16, channels last (cs, the channel
// stride, a multiple of 16 so that every 8-channel chunk is a 16-byte
// access); forward weights [9][cout][cin] BF16 (tap-major, so one tap's
// cout x cin block is contiguous); input-gradient weights [9][cin][cout]
// with the taps flipped; FP32 master weights, Adam moments and weight
// gradients [cout][9][cin].
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace pgn {

using bf16 = __nv_bfloat16;
using bf162 = __nv_bfloat162;

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start before its predecessor in the stream has
// finished; it waits here, before reading anything the predecessor wrote
// (a no-op for an ordinary launch).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t* r, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}

// d += a (16 x 16, row) * b (16 x 8, col); BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 16-byte global -> shared copy; zero-fill when !valid (the source is then
// not read, src must still be a valid address)
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

enum ConvOut {
    OUT_BF16 = 0,        // y = z
    OUT_BF16_RELU = 1,   // y = max(z, 0)
    OUT_F32 = 2,         // y = z, FP32 (the network's output layer)
    OUT_BF16_MASKED = 3  // y = z where mask > 0, else 0 (input gradient through a ReLU)
};

struct ConvArgs {
    int B, H, W;
    const bf16* in;  // [B][H][W][in_cs], channels [0, CIN)
    int in_cs;
    const bf16* w;   // [9][w_rows][CIN]; this block uses rows co0 .. co0+COT-1
    int w_rows;
    void* out;       // channel co stored at [..][out_coff + co] when co < cout_real
    int out_cs, out_coff, cout_real;
    const bf16* mask;  // OUT_BF16_MASKED: [B][H][W][mask_cs], channel co
    int mask_cs;
    const int* skip;   // non-NULL and *skip != 0: the launch does nothing
    bf16* pool_out;    // OUT_BF16_RELU, non-NULL: also the 2 x 2 average of the outputs,
    int pool_cs;       //   [B][H/2][W/2][pool_cs], channel co (H and W even)
};

constexpr int kConvThreads = 128;

__host__ __device__ constexpr int conv_smem_bytes(int cin, int cot) {
    return (100 + 9 * cot) * (cin + 8) * 2;
}

// 3 x 3 convolution, zero padding, no bias.  A block computes an 8 x 8
// pixel tile (four warps, each a 2-row x 8-column m16 tile) for COT output
// channels.  The 10 x 10 input halo (CIN channels) and all nine taps'
// COT x CIN weights are staged in shared memory by one cp.async group, so
// the block pays one L2 round trip before its MMAs (streaming the taps one
// by one left each small layer waiting nine times); COT is chosen so the
// weights fit (conv_smem_bytes).
// Grid: (ceil(W/8), ceil(H/8) * B, w_rows / COT).
template <int CIN, int COT, int MODE>
__global__ void __launch_bounds__(kConvThreads) conv3x3_kernel(ConvArgs a) {
    static_assert(CIN % 16 == 0 && COT % 16 == 0, "channels in multiples of 16");
    pdl_wait();
    if (a.skip && *a.skip) return;
    constexpr int SP = CIN + 8;  // padded pixel / weight-row stride in shared memory
    constexpr int C8 = CIN / 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* sIn = reinterpret_cast<bf16*>(smem_raw);
    bf16* sW = sIn + 100 * SP;  // [9][COT][SP]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_y = (a.H + 7) >> 3;
    const int b = blockIdx.y / tiles_y;
    const int ty0 = (blockIdx.y - b * tiles_y) * 8, tx0 = blockIdx.x * 8;
    const int co0 = blockIdx.z * COT;
    for (int q = tid; q < 100 * C8; q += kConvThreads) {
        const int pix = q / C8, c8 = q - pix * C8;
        const int gy = ty0 - 1 + pix / 10, gx = tx0 - 1 + pix % 10;
        const bool ok = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W;
        const bf16* src = ok ? a.in + (((size_t)b * a.H + gy) * a.W + gx) * a.in_cs + c8 * 8 : a.in;
        cp_async16(sIn + pix * SP + c8 * 8, src, ok);
    }
    for (int q = tid; q < 9 * COT * C8; q += kConvThreads) {
        const int row = q / C8, c8 = q - row * C8;  // row = tap * COT + co
        const int tap = row / COT, co = row - tap * COT;
        cp_async16(sW + row * SP + c8 * 8, a.w + ((size_t)tap * a.w_rows + co0 + co) * CIN + c8 * 8, true);
    }
    cp_async_commit();
    float acc[COT / 8][4];
#pragma unroll
    for (int i = 0; i < COT / 8; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    const int j = lane >> 3, i8 = lane & 7;
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll 1
    for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
        const bf16* sWt = sW + tap * COT * SP;
        // A rows: matrix j covers m rows (j & 1) * 8 .. +7 (tile row 2*warp + (j & 1),
        // columns 0..7) and k half j >> 1
        const bf16* aRow = sIn + ((2 * warp + (j & 1) + dy) * 10 + i8 + dx) * SP + (j >> 1) * 8;
#pragma unroll
        for (int ks = 0; ks < CIN / 16; ks++) {
            uint32_t af[4];
            ldsm_x4(af, aRow + ks * 16);
#pragma unroll
            for (int np = 0; np < COT / 16; np++) {
                uint32_t bw[4];
                // matrix j: n tile 2*np + (j >> 1), k half j & 1
                ldsm_x4(bw, sWt + ((2 * np + (j >> 1)) * 8 + i8) * SP + ks * 16 + (j & 1) * 8);
                mma_bf16(acc[2 * np], af, bw[0], bw[1]);
                mma_bf16(acc[2 * np + 1], af, bw[2], bw[3]);
            }
        }
    }
    const int g = lane >> 2, q4 = lane & 3;
#pragma unroll
    for (int nt = 0; nt < COT / 8; nt++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int m = g + 8 * h;
            const int gy = ty0 + 2 * warp + (m >> 3), gx = tx0 + (m & 7);
            if (gy >= a.H || gx >= a.W) continue;
            const int co = co0 + nt * 8 + 2 * q4;
            if (co >= a.cout_real) continue;
            float v0 = acc[nt][2 * h], v1 = acc[nt][2 * h + 1];
            const size_t pix = ((size_t)b * a.H + gy) * a.W + gx;
            if constexpr (MODE == OUT_F32) {
                float* o = static_cast<float*>(a.out) + pix * a.out_cs + a.out_coff + co;
                o[0] = v0;
                if (co + 1 < a.cout_real) o[1] = v1;
            } else {
                if constexpr (MODE == OUT_BF16_RELU) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                if constexpr (MODE == OUT_BF16_MASKED) {
                    const bf162 mk = *reinterpret_cast<const bf162*>(a.mask + pix * a.mask_cs + co);
                    if (!(__bfloat162float(mk.x) > 0.f)) v0 = 0.f;
                    if (!(__bfloat162float(mk.y) > 0.f)) v1 = 0.f;
                }
                *reinterpret_cast<bf162*>(static_cast<bf16*>(a.out) + pix * a.out_cs + a.out_coff + co) =
                    __floats2bfloat162_rn(v0, v1);
            }
        }
    }
    if constexpr (MODE == OUT_BF16_RELU) {
        if (a.pool_out) {
            // 2 x 2 average pooling of the tile's stored (BF16) outputs: a thread
            // holds rows 2w and 2w+1 of column g, and lane ^ 4 holds column g ^ 1
            // (the tile is 8-aligned and H, W are even, so a window never
            // straddles the image edge)
            const int Hp = a.H >> 1, Wp = a.W >> 1;
            const int py = (ty0 >> 1) + warp, px = (tx0 >> 1) + (g >> 1);
            auto bfr = [](float v) { return __bfloat162float(__float2bfloat16_rn(fmaxf(v, 0.f))); };
#pragma unroll
            for (int nt = 0; nt < COT / 8; nt++) {
                float s0 = bfr(acc[nt][0]) + bfr(acc[nt][2]);
                float s1 = bfr(acc[nt][1]) + bfr(acc[nt][3]);
                s0 += __shfl_xor_sync(0xffffffffu, s0, 4);
                s1 += __shfl_xor_sync(0xffffffffu, s1, 4);
                const int co = co0 + nt * 8 + 2 * q4;
                if ((g & 1) == 0 && py < Hp && px < Wp && co < a.cout_real)
                    *reinterpret_cast<bf162*>(a.pool_out + (((size_t)b * Hp + py) * Wp + px) * a.pool_cs + co) =
                        __floats2bfloat162_rn(0.25f * s0, 0.25f * s1);
            }
        }
    }
}

struct WgradArgs {
    int B, H, W;
    const bf16* x;  // layer input [B][H][W][x_cs], channels [0, cin)
    int x_cs;
    const bf16* g;  // gradient of the layer's pre-activation [B][H][W][g_cs], channels [0, cout)
    int g_cs;
    float* dw;      // [cout][9][cin], accumulated into (atomics)
    int cin, cout;
    int tiles;      // B * ceil(H/8) * ceil(W/8)
};

// dw[co][tap][ci] += sum over pixels of g[p][co] * x[p + tap][ci].  A block
// owns a COT x CIT output tile for all nine taps (accumulators in
// registers) and walks over 8 x 8 pixel tiles (the GEMM's K): the gradient
// tile and the input halo are staged in shared memory and both operands
// read with ldmatrix.trans (pixels are the rows of both tiles).  One
// atomicAdd per accumulator at the end.
// Grid: (pixel-tile splits, cout / COT, cin / CIT); block (COT/16)*(CIT/16) warps.
template <int COT, int CIT>
__global__ void __launch_bounds__((COT / 16) * (CIT / 16) * 32) wgrad_kernel(WgradArgs a) {
    constexpr int NWN = CIT / 16;
    constexpr int NT = (COT / 16) * NWN * 32;
    constexpr int SX = CIT + 8, SG = COT + 8;
    __shared__ __align__(16) bf16 sX[100 * SX];
    __shared__ __align__(16) bf16 sG[64 * SG];
    const int co0 = blockIdx.y * COT, ci0 = blockIdx.z * CIT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp / NWN, wn = warp - wm * NWN;
    const int tiles_x = (a.W + 7) >> 3, tiles_y = (a.H + 7) >> 3;
    float acc[9][2][4];
#pragma unroll
    for (int t = 0; t < 9; t++)
#pragma unroll
        for (int n = 0; n < 2; n++) acc[t][n][0] = acc[t][n][1] = acc[t][n][2] = acc[t][n][3] = 0.f;
    const int j = lane >> 3, i8 = lane & 7;
    for (int t = blockIdx.x; t < a.tiles; t += gridDim.x) {
        const int tx = t % tiles_x, rest = t / tiles_x;
        const int ty = rest % tiles_y, b = rest / tiles_y;
        const int ty0 = ty * 8, tx0 = tx * 8;
        for (int q = tid; q < 100 * (CIT / 8); q += NT) {
            const int pix = q / (CIT / 8), c8 = q - pix * (CIT / 8);
            const int gy = ty0 - 1 + pix / 10, gx = tx0 - 1 + pix % 10;
            const bool ok = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W;
            const bf16* src =
                ok ? a.x + (((size_t)b * a.H + gy) * a.W + gx) * a.x_cs + ci0 + c8 * 8 : a.x;
            cp_async16(sX + pix * SX + c8 * 8, src, ok);
        }
        for (int q = tid; q < 64 * (COT / 8); q += NT) {
            const int pix = q / (COT / 8), c8 = q - pix * (COT / 8);
            const int gy = ty0 + pix / 8, gx = tx0 + pix % 8;
            const bool ok = gy < a.H && gx < a.W;
            const bf16* src =
                ok ? a.g + (((size_t)b * a.H + gy) * a.W + gx) * a.g_cs + co0 + c8 * 8 : a.g;
            cp_async16(sG + pix * SG + c8 * 8, src, ok);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 4; s++) {  // K step: 16 pixels, tile rows 2s and 2s+1
            uint32_t af[4];
            // A = g^T: matrix j has pixels of tile row 2s + (j >> 1), output channels
            // wm*16 + (j & 1)*8 .. +7
            ldsm_x4_t(af, sG + ((2 * s + (j >> 1)) * 8 + i8) * SG + wm * 16 + (j & 1) * 8);
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                uint32_t bx[4];
                // B = shifted x: matrix j has pixels of tile row 2s + (j & 1), input
                // channels wn*16 + (j >> 1)*8 .. +7
                ldsm_x4_t(bx, sX + ((2 * s + (j & 1) + dy) * 10 + i8 + dx) * SX + wn * 16 + (j >> 1) * 8);
                mma_bf16(acc[tap][0], af, bx[0], bx[1]);
                mma_bf16(acc[tap][1], af, bx[2], bx[3]);
            }
        }
        __syncthreads();
    }
    const int g = lane >> 2, q4 = lane & 3;
#pragma unroll
    for (int tap = 0; tap < 9; tap++)
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int co = co0 + wm * 16 + g + 8 * h;
                const int ci = ci0 + wn * 16 + n * 8 + 2 * q4;
                float* d = a.dw + ((size_t)co * 9 + tap) * a.cin + ci;
                atomicAdd(d, acc[tap][n][2 * h]);
                atomicAdd(d + 1, acc[tap][n][2 * h + 1]);
            }
}

// Nearest 2x upsampling into a concatenation buffer:
// out[b][y][x][coff + c] = in[b][y/2][x/2][c], c < C.
__global__ void up2_kernel(int B, int H, int W, const bf16* __restrict__ in, int in_cs, int C,
                           bf16* __restrict__ out, int out_cs, int coff, const int* skip) {
    pdl_wait();
    if (skip && *skip) return;
    const int C8 = C / 8;
    const long total = (long)B * H * W * C8;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int c8 = (int)(q % C8);
        const long p = q / C8;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long)W * H));
        const uint4 v = *reinterpret_cast<const uint4*>(
            in + (((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * in_cs + c8 * 8);
        *reinterpret_cast<uint4*>(out + (((size_t)b * H + y) * W + x) * out_cs + coff + c8 * 8) = v;
    }
}

// Gradient of up2 (sum over each 2 x 2 block):
// out[b][y][x][c] = sum_{i,j} in[b][2y+i][2x+j][coff + c], c < C.
__global__ void up2_bwd_kernel(int B, int Ho, int Wo, const bf16* __restrict__ in, int in_cs, int coff,
                               int C, bf16* __restrict__ out, int out_cs) {
    const int C8 = C / 8;
    const long total = (long)B * Ho * Wo * C8;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int c8 = (int)(q % C8);
        const long p = q / C8;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), b = (int)(p / ((long)Wo * Ho));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 2; i++)
            for (int k = 0; k < 2; k++) {
                const uint4 v = *reinterpret_cast<const uint4*>(
                    in + (((size_t)b * 2 * Ho + 2 * y + i) * 2 * Wo + 2 * x + k) * in_cs + coff + c8 * 8);
                const bf162* h = reinterpret_cast<const bf162*>(&v);
                for (int e = 0; e < 4; e++) {
                    const float2 f = __bfloat1622float2(h[e]);
                    s[2 * e] += f.x;
                    s[2 * e + 1] += f.y;
                }
            }
        uint4 o;
        bf162* ho = reinterpret_cast<bf162*>(&o);
        for (int e = 0; e < 4; e++) ho[e] = __floats2bfloat162_rn(s[2 * e], s[2 * e + 1]);
        *reinterpret_cast<uint4*>(out + (((size_t)b * Ho + y) * Wo + x) * out_cs + c8 * 8) = o;
    }
}

// Gradient reaching an encoder output e (a ReLU output that feeds both the
// decoder's concatenation and the pooling to the next level):
// out[b][y][x][c] = dcat[b][y][x][c] + (e[b][y][x][c] > 0 ? dp[b][y/2][x/2][c] / 4 : 0)
// where dcat (already masked) and e live in the concatenation buffers
// (stride cat_cs, channels [0, C)) and dp is the gradient of the pooled
// tensor [B][H/2][W/2][C].
__global__ void pool2_bwd_add_kernel(int B, int H, int W, const bf16* __restrict__ dcat,
                                     const bf16* __restrict__ e, int cat_cs, const bf16* __restrict__ dp,
                                     int C, bf16* __restrict__ out) {
    const int C8 = C / 8;
    const long total = (long)B * H * W * C8;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int c8 = (int)(q % C8);
        const long p = q / C8;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long)W * H));
        const size_t ci = (((size_t)b * H + y) * W + x) * cat_cs + c8 * 8;
        const uint4 vd = *reinterpret_cast<const uint4*>(dcat + ci);
        const uint4 ve = *reinterpret_cast<const uint4*>(e + ci);
        const uint4 vp = *reinterpret_cast<const uint4*>(
            dp + (((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c8 * 8);
        const bf162* hd = reinterpret_cast<const bf162*>(&vd);
        const bf162* he = reinterpret_cast<const bf162*>(&ve);
        const bf162* hp = reinterpret_cast<const bf162*>(&vp);
        uint4 o;
        bf162* ho = reinterpret_cast<bf162*>(&o);
        for (int k = 0; k < 4; k++) {
            const float2 d = __bfloat1622float2(hd[k]), ee = __bfloat1622float2(he[k]),
                         pp = __bfloat1622float2(hp[k]);
            ho[k] = __floats2bfloat162_rn(d.x + (ee.x > 0.f ? 0.25f * pp.x : 0.f),
                                          d.y + (ee.y > 0.f ? 0.25f * pp.y : 0.f));
        }
        *reinterpret_cast<uint4*>(out + (((size_t)b * H + y) * W + x) * C + c8 * 8) = o;
    }
}

// One layer's place in the parameter arrays.
struct LayerDesc {
    int cin, cout;      // stored (padded to multiples of 16)
    long off;           // [cout][9][cin] block in the master / moment / gradient arrays
    long off_f, off_d;  // [9][cout][cin] forward and [9][cin][cout] input-gradient BF16 copies
};
constexpr int kLayers = 15;
struct LayerTable {
    LayerDesc l[kLayers];
    long total;
};

// BF16 copies of the FP32 master weights: forward layout and the flipped,
// transposed layout of the input-gradient convolution (tap' = 8 - tap).
__device__ __forceinline__ void write_bf16_copies(const LayerTable& T, long i, float w, bf16* wf, bf16* wd) {
    int k = 0;
    while (k + 1 < kLayers && i >= T.l[k + 1].off) k++;
    const LayerDesc& L = T.l[k];
    const long r = i - L.off;
    const int ci = (int)(r % L.cin), tap = (int)((r / L.cin) % 9), co = (int)(r / ((long)L.cin * 9));
    const bf16 h = __float2bfloat16_rn(w);
    wf[L.off_f + ((long)tap * L.cout + co) * L.cin + ci] = h;
    wd[L.off_d + ((long)(8 - tap) * L.cin + ci) * L.cout + co] = h;
}

__global__ void weights_to_bf16_kernel(LayerTable T, const float* __restrict__ w, bf16* wf, bf16* wd) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < T.total; i += (long)gridDim.x * blockDim.x)
        write_bf16_copies(T, i, w[i], wf, wd);
}

// Adam (Kingma & Ba): m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
// w -= lr_t * m_hat / (sqrt(v_hat) + eps) with bias-corrected moments, at
// step *step (counted from 1); lr_t = lr, or with total_steps > 0 the
// cosine decay lr (1 + cos(pi min(step, total) / total)) / 2.  Writes the
// BF16 copies of the updated weights.
__global__ void adam_kernel(LayerTable T, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, const int* __restrict__ step, float lr, float b1,
                            float b2, float eps, int total_steps, bf16* wf, bf16* wd) {
    const int t = *step;
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    float lr_t = lr;
    if (total_steps > 0) {
        const float f = fminf((float)t, (float)total_steps) / (float)total_steps;
        lr_t = 0.5f * lr * (1.f + cospif(f));
    }
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < T.total; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr_t * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        write_bf16_copies(T, i, wi, wf, wd);
    }
}

}  // namespace pgn
