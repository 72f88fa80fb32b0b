// unet.cu — the learned warm start: a 4-level convolutional U-Net trained on
// snapshots that the plain solver generates, predicting the first potential
// correction of a time step (and the microwave field) as an initial guess for
// the multigrid, which then converges to the unchanged tolerance.  The network
// has no counterpart in the reference.
//
// Tensors are NHWC bfloat16 (channels innermost, a channel stride per tensor so
// that the skip connections live inside the concatenation buffers), weights
// [Cout][3][3][Cin] bfloat16 with FP32 master copies, FP32 accumulation.
// Convolutions are implicit GEMMs on the tensor cores (mma.sync m16n8k16 bf16):
//   forward       D[pixel][co] = sum_{tap,ci} X[pixel+tap][ci] W[co][tap][ci]
//   input grad    the forward kernel with W'[ci][tap][co] = W[co][8-tap][ci]
//   weight grad   dW[co][tap][ci] = sum_pixel dY[pixel][co] X[pixel+tap][ci]
// The ReLU derivative is applied by every kernel that writes a gradient into a
// ReLU output (gate = that output > 0), so no pre-activations are stored.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "fluid.cuh"

typedef __nv_bfloat16 bf16;

namespace cth {
namespace unet {

constexpr int TH = 8, TW = 16;           // output tile of a conv CTA (pixels)
constexpr int HP = TH + 2, WP = TW + 2;  // with the 3x3 halo
constexpr int SR16 = 24;                 // smem row stride (bf16) of 16-channel rows: 48 B
constexpr int SR32 = 40;                 // smem row stride (bf16) of 32-channel rows: 80 B

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void mma16816(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// a channel slice of an NHWC tensor
struct TensorRef {
    bf16* p;
    int cs;    // channel stride (pixel pitch)
    int coff;  // first channel
};

struct ConvArgs {
    const bf16* in;
    int in_cs, in_coff, Cin;
    const bf16* w;       // [Cout][9][Cin]
    const bf16* wtc;     // the same weights [Cin/8][9][Cout][8] (tcgen05 path)
    const float* bias;   // null: none
    bf16* out;
    int out_cs, out_coff, Cout;
    int H, W;
    int relu;
    const bf16* gate;    // null: none; else out *= (gate > 0)
    int gate_cs, gate_coff;
    int accumulate;      // add to the existing output
    int wait_polls;      // tcgen05 path: polls of each mbarrier wait before it gives up
    int stall;           // tcgen05 path, test of the bounded waits: no loads are issued
};

// 3x3 convolution, SAME zero padding.  CTA: 8 x 16 output pixels x 32 output
// channels, 4 warps (two image rows each); Cin in chunks of 16 staged in
// shared memory with the halo.
__global__ void __launch_bounds__(128) k_conv3_fwd(ConvArgs a) {
    __shared__ alignas(16) bf16 s_in[HP * WP * SR16];
    __shared__ alignas(16) bf16 s_w[32 * 9 * SR16];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH, co0 = blockIdx.z * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;
    for (int c0 = 0; c0 < a.Cin; c0 += 16) {
        for (int idx = tid; idx < HP * WP * 2; idx += 128) {
            const int pix = idx >> 1, half = idx & 1;
            const int gy = y0 + pix / WP - 1, gx = x0 + pix % WP - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < a.H && gx >= 0 && gx < a.W)
                v = *reinterpret_cast<const uint4*>(a.in + ((size_t)gy * a.W + gx) * a.in_cs + a.in_coff + c0 +
                                                    half * 8);
            *reinterpret_cast<uint4*>(s_in + pix * SR16 + half * 8) = v;
        }
        for (int idx = tid; idx < 32 * 9 * 2; idx += 128) {
            const int row = idx >> 1, half = idx & 1;
            const int co = co0 + row / 9, tap = row % 9;
            const uint4 v = *reinterpret_cast<const uint4*>(a.w + ((size_t)co * 9 + tap) * a.Cin + c0 + half * 8);
            *reinterpret_cast<uint4*>(s_w + row * SR16 + half * 8) = v;
        }
        __syncthreads();
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            const int dy = tap / 3, dx = tap % 3;
            uint32_t b[4][2];
#pragma unroll
            for (int nb = 0; nb < 2; nb++) {
                const int m = lane >> 3, r = lane & 7;
                const int col = nb * 16 + (m >> 1) * 8 + r;
                const int koff = (m & 1) * 8;
                ldsm_x4(smem_u32(s_w + (col * 9 + tap) * SR16 + koff), b[2 * nb][0], b[2 * nb][1],
                        b[2 * nb + 1][0], b[2 * nb + 1][1]);
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int ry = warp * 2 + mt;
                const int m = lane >> 3, r = lane & 7;
                const int px = (m & 1) * 8 + r, koff = (m >> 1) * 8;
                uint32_t a0, a1, a2, a3;
                ldsm_x4(smem_u32(s_in + ((ry + dy) * WP + px + dx) * SR16 + koff), a0, a1, a2, a3);
#pragma unroll
                for (int nt = 0; nt < 4; nt++) mma16816(acc[mt][nt], a0, a1, a2, a3, b[nt][0], b[nt][1]);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        const int gy = y0 + warp * 2 + mt;
        if (gy >= a.H) continue;
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            const int gx = x0 + (lane >> 2) + hf * 8;
            if (gx >= a.W) continue;
            const size_t pix = (size_t)gy * a.W + gx;
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                const int co = co0 + nt * 8 + 2 * (lane & 3);
                float v0 = acc[mt][nt][2 * hf], v1 = acc[mt][nt][2 * hf + 1];
                if (a.bias) { v0 += a.bias[co]; v1 += a.bias[co + 1]; }
                if (a.relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                if (a.gate) {
                    const __nv_bfloat162 g =
                        *reinterpret_cast<const __nv_bfloat162*>(a.gate + pix * a.gate_cs + a.gate_coff + co);
                    if (!(__bfloat162float(g.x) > 0.f)) v0 = 0.f;
                    if (!(__bfloat162float(g.y) > 0.f)) v1 = 0.f;
                }
                __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(a.out + pix * a.out_cs + a.out_coff + co);
                if (a.accumulate) {
                    const __nv_bfloat162 q = *o;
                    v0 += __bfloat162float(q.x);
                    v1 += __bfloat162float(q.y);
                }
                *o = __floats2bfloat162_rn(v0, v1);
            }
        }
    }
}

struct WgradArgs {
    const bf16* dy;
    int dy_cs, dy_coff, Cout;
    const bf16* in;
    int in_cs, in_coff, Cin;
    int H, W;
    float* dw;   // [Cout][9][Cin], accumulated
    int patches_per_cta;
};

// weight gradient: CTA = 32 output channels x 32 input channels x 9 taps (one
// warp per tap) over a run of 8 x 16 pixel patches; partial sums are added to
// dw with FP32 atomics.
__global__ void __launch_bounds__(288) k_conv3_wgrad(WgradArgs a) {
    __shared__ alignas(16) bf16 s_dy[TH * TW * SR32];
    __shared__ alignas(16) bf16 s_in[HP * WP * SR32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int co0 = blockIdx.y * 32, ci0 = blockIdx.z * 32;
    const int npx = (a.W + TW - 1) / TW, npy = (a.H + TH - 1) / TH, npatch = npx * npy;
    const int tap = warp, dy_ = tap / 3, dx_ = tap % 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;
    const int p_begin = blockIdx.x * a.patches_per_cta;
    const int p_end = min(npatch, p_begin + a.patches_per_cta);
    for (int pt = p_begin; pt < p_end; pt++) {
        const int y0 = (pt / npx) * TH, x0 = (pt % npx) * TW;
        for (int idx = tid; idx < TH * TW * 4; idx += 288) {
            const int pix = idx >> 2, q = idx & 3;
            const int gy = y0 + pix / TW, gx = x0 + pix % TW;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy < a.H && gx < a.W)
                v = *reinterpret_cast<const uint4*>(a.dy + ((size_t)gy * a.W + gx) * a.dy_cs + a.dy_coff + co0 + q * 8);
            *reinterpret_cast<uint4*>(s_dy + pix * SR32 + q * 8) = v;
        }
        for (int idx = tid; idx < HP * WP * 4; idx += 288) {
            const int pix = idx >> 2, q = idx & 3;
            const int gy = y0 + pix / WP - 1, gx = x0 + pix % WP - 1;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < a.H && gx >= 0 && gx < a.W)
                v = *reinterpret_cast<const uint4*>(a.in + ((size_t)gy * a.W + gx) * a.in_cs + a.in_coff + ci0 + q * 8);
            *reinterpret_cast<uint4*>(s_in + pix * SR32 + q * 8) = v;
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < TH; r++) {
            const int m = lane >> 3, rr = lane & 7;
            uint32_t af[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int px = (m >> 1) * 8 + rr, coff = mt * 16 + (m & 1) * 8;
                ldsm_x4_t(smem_u32(s_dy + (r * TW + px) * SR32 + coff), af[mt][0], af[mt][1], af[mt][2],
                          af[mt][3]);
            }
            uint32_t bfr[4][2];
#pragma unroll
            for (int nb = 0; nb < 2; nb++) {
                const int px = (m & 1) * 8 + rr, cioff = nb * 16 + (m >> 1) * 8;
                ldsm_x4_t(smem_u32(s_in + ((r + dy_) * WP + px + dx_) * SR32 + cioff), bfr[2 * nb][0],
                          bfr[2 * nb][1], bfr[2 * nb + 1][0], bfr[2 * nb + 1][1]);
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    mma16816(acc[mt][nt], af[mt][0], af[mt][1], af[mt][2], af[mt][3], bfr[nt][0], bfr[nt][1]);
        }
        __syncthreads();
    }
    if (p_begin >= p_end) return;
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int hf = 0; hf < 2; hf++) {
                const int co = co0 + mt * 16 + (lane >> 2) + hf * 8;
                const int ci = ci0 + nt * 8 + 2 * (lane & 3);
                float* d = a.dw + ((size_t)co * 9 + tap) * a.Cin + ci;
                atomicAdd(d, acc[mt][nt][2 * hf]);
                atomicAdd(d + 1, acc[mt][nt][2 * hf + 1]);
            }
}

// 8 bf16 <-> 8 floats (16-byte vectors; channel slices start on multiples of 8)
__device__ __forceinline__ void unpack8(const uint4& v, float f[8]) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        f[2 * j] = __bfloat162float(h[j].x);
        f[2 * j + 1] = __bfloat162float(h[j].y);
    }
}
__device__ __forceinline__ uint4 pack8(const float f[8]) {
    uint4 v;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
    for (int j = 0; j < 4; j++) h[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
    return v;
}
__device__ __forceinline__ uint4 ld8(const bf16* p) { return *reinterpret_cast<const uint4*>(p); }
__device__ __forceinline__ void st8(bf16* p, const uint4& v) { *reinterpret_cast<uint4*>(p) = v; }

// bias gradient db[c] += sum over pixels of dy[.][c].  256 threads: thread t
// sums channels 8g..8g+7 (g = t % G, G = C/8) of every (256/G)-th pixel of the
// block's share; the lanes are then reduced in shared memory and each channel
// gets one atomic per block.  C a multiple of 8, at most 256.
__global__ void __launch_bounds__(256) k_bias_grad(const bf16* __restrict__ dy, int cs, int coff, int C, int npix,
                                                   float* __restrict__ db) {
    __shared__ float red[256 * 8];
    const int G = C >> 3, L = 256 / G, tid = threadIdx.x;
    const int g = tid % G, lane = tid / G;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (lane < L)
        for (int p = blockIdx.x * L + lane; p < npix; p += gridDim.x * L) {
            float f[8];
            unpack8(ld8(dy + (size_t)p * cs + coff + 8 * g), f);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] += f[j];
        }
#pragma unroll
    for (int j = 0; j < 8; j++) red[tid * 8 + j] = acc[j];
    __syncthreads();
    if (tid < C) {
        const int gg = tid >> 3, j = tid & 7;
        float sum = 0.f;
        for (int l = 0; l < L; l++) sum += red[(l * G + gg) * 8 + j];
        atomicAdd(db + tid, sum);
    }
}

// bf16 copies of one convolution's FP32 weights W[co][tap][ci]: W itself, the
// flipped transpose W'[ci][tap][co] = W[co][8-tap][ci] (input gradients), and
// both again in the tcgen05 layout [Cin/32][9][Cout][32] (wbt of W, wtt of W';
// Cin and Cout multiples of 32)
__global__ void k_weights(const float* __restrict__ w, int Cout, int Cin, bf16* __restrict__ wb,
                          bf16* __restrict__ wt, bf16* __restrict__ wbt, bf16* __restrict__ wtt) {
    const size_t n = (size_t)Cout * 9 * Cin;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int ci = (int)(e % Cin);
        const int tap = (int)((e / Cin) % 9);
        const int co = (int)(e / ((size_t)Cin * 9));
        const bf16 v = __float2bfloat16_rn(w[e]);
        wb[e] = v;
        wt[((size_t)ci * 9 + (8 - tap)) * Cout + co] = v;
        wbt[(((size_t)(ci >> 5) * 9 + tap) * Cout + co) * 32 + (ci & 31)] = v;
        // W' has Cout' = Cin and Cin' = Cout: element (co' = ci, tap' = 8 - tap, ci' = co)
        wtt[(((size_t)(co >> 5) * 9 + (8 - tap)) * Cin + ci) * 32 + (co & 31)] = v;
    }
}

// 2x2 average pooling: out[y][x][c] = mean of in[2y..2y+1][2x..2x+1][c]; one
// thread per output pixel and 8 channels
__global__ void k_pool2(const bf16* __restrict__ in, int in_cs, int in_coff, int C, int Ho, int Wo,
                        bf16* __restrict__ out, int out_cs) {
    const int G = C >> 3, Wi = 2 * Wo;
    const size_t n = (size_t)Ho * Wo * G;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const size_t pix = e / G;
        const int y = (int)(pix / Wo), x = (int)(pix % Wo);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float f[8];
            unpack8(ld8(in + ((size_t)(2 * y + (k >> 1)) * Wi + 2 * x + (k & 1)) * in_cs + in_coff + 8 * g), f);
#pragma unroll
            for (int j = 0; j < 8; j++) s[j] += f[j];
        }
#pragma unroll
        for (int j = 0; j < 8; j++) s[j] *= 0.25f;
        st8(out + pix * out_cs + 8 * g, pack8(s));
    }
}

// gradient of k_pool2 added into the ReLU output it pooled:
// din[2y+a][2x+b][c] += dout[y][x][c] / 4 where x_in > 0; one thread per input
// pixel and 8 channels
__global__ void k_pool2_bwd(const bf16* __restrict__ dout, int dout_cs, int C, int Ho, int Wo,
                            bf16* __restrict__ din, int din_cs, int din_coff, const bf16* __restrict__ gate,
                            int gate_cs, int gate_coff) {
    const int G = C >> 3, Wi = 2 * Wo;
    const size_t n = (size_t)4 * Ho * Wo * G;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const size_t pi = e / G;
        const int yi = (int)(pi / Wi), xi = (int)(pi % Wi);
        float gd[8], on[8], d[8];
        unpack8(ld8(dout + ((size_t)(yi >> 1) * Wo + (xi >> 1)) * dout_cs + 8 * g), gd);
        unpack8(ld8(gate + pi * gate_cs + gate_coff + 8 * g), on);
        bf16* dp = din + pi * din_cs + din_coff + 8 * g;
        unpack8(ld8(dp), d);
#pragma unroll
        for (int j = 0; j < 8; j++) d[j] = d[j] + (on[j] > 0.f ? 0.25f * gd[j] : 0.f);
        st8(dp, pack8(d));
    }
}

// nearest 2x upsampling into a channel slice: out[y][x][c] = in[y/2][x/2][c];
// one thread per input pixel and 8 channels, writing the 4 children
__global__ void k_up2(const bf16* __restrict__ in, int in_cs, int C, int Hi, int Wi, bf16* __restrict__ out,
                      int out_cs, int out_coff) {
    const int G = C >> 3, Wo = 2 * Wi;
    const size_t n = (size_t)Hi * Wi * G;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const size_t pi = e / G;
        const int y = (int)(pi / Wi), x = (int)(pi % Wi);
        const uint4 v = ld8(in + pi * in_cs + 8 * g);
#pragma unroll
        for (int k = 0; k < 4; k++)
            st8(out + ((size_t)(2 * y + (k >> 1)) * Wo + 2 * x + (k & 1)) * out_cs + out_coff + 8 * g, v);
    }
}

// gradient of k_up2: din[y][x][c] = sum of the 4 children's gradients; one
// thread per input pixel and 8 channels
__global__ void k_up2_bwd(const bf16* __restrict__ dout, int dout_cs, int dout_coff, int C, int Hi, int Wi,
                          bf16* __restrict__ din, int din_cs) {
    const int G = C >> 3, Wo = 2 * Wi;
    const size_t n = (size_t)Hi * Wi * G;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const size_t pi = e / G;
        const int y = (int)(pi / Wi), x = (int)(pi % Wi);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float f[8];
            unpack8(ld8(dout + ((size_t)(2 * y + (k >> 1)) * Wo + 2 * x + (k & 1)) * dout_cs + dout_coff + 8 * g), f);
#pragma unroll
            for (int j = 0; j < 8; j++) s[j] += f[j];
        }
        st8(din + pi * din_cs + 8 * g, pack8(s));
    }
}

// FP32 NHWC input (cin channels) -> bf16 with cpad channels (zeros beyond cin);
// one thread per pixel
__global__ void k_pack(const float* __restrict__ in, int cin, int npix, int cpad, bf16* __restrict__ out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        for (int c0 = 0; c0 < cpad; c0 += 8) {
            float f[8];
#pragma unroll
            for (int j = 0; j < 8; j++) f[j] = (c0 + j < cin) ? in[(size_t)p * cin + c0 + j] : 0.f;
            st8(out + (size_t)p * cpad + c0, pack8(f));
        }
    }
}

// 1x1 output layer (linear): out[p][c] = sum_k wh[c][k] y[p][k] + bh[c], FP32;
// one thread per pixel, the layer's weights in shared memory; C, cout <= 32
__global__ void k_head_fwd(const bf16* __restrict__ y, int C, int npix, const float* __restrict__ wh,
                           const float* __restrict__ bh, int cout, float* __restrict__ out) {
    __shared__ float s_w[32 * 32], s_b[32];
    for (int e = threadIdx.x; e < cout * C; e += blockDim.x) s_w[e] = wh[e];
    for (int e = threadIdx.x; e < cout; e += blockDim.x) s_b[e] = bh[e];
    __syncthreads();
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float yv[32];
#pragma unroll
        for (int k0 = 0; k0 < 32; k0 += 8)
            if (k0 < C) unpack8(ld8(y + (size_t)p * C + k0), yv + k0);
        for (int c = 0; c < cout; c++) {
            float s = s_b[c];
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k < C) s += s_w[c * C + k] * yv[k];
            out[(size_t)p * cout + c] = s;
        }
    }
}

// backward of the output layer: dy = wh^T dout where y > 0 (bf16), and the
// layer's gradients dwh[c][k] = sum_p dout[p][c] y[p][k], dbh[c] = sum_p
// dout[p][c].  128 threads per block over tiles of 128 pixels: each thread
// writes its pixel's dy and parks y and dout in shared memory, then thread e
// accumulates entry e of [dwh | dbh] over the tile; one atomic per entry and
// block at the end.  C, cout <= 32.
__global__ void __launch_bounds__(128) k_head_bwd(const bf16* __restrict__ y, int C, int npix,
                                                  const float* __restrict__ wh, int cout,
                                                  const float* __restrict__ dout, bf16* __restrict__ dy,
                                                  float* __restrict__ dwh, float* __restrict__ dbh) {
    constexpr int kT = 128, kE = 9;  // tile, entries per thread (32 x 33 <= 128 x 9)
    __shared__ float s_y[kT * 33], s_d[kT * 33], s_w[32 * 32];
    const int tid = threadIdx.x, ne = cout * (C + 1);
    for (int e = tid; e < cout * C; e += kT) s_w[e] = wh[e];
    float acc[kE];
#pragma unroll
    for (int j = 0; j < kE; j++) acc[j] = 0.f;
    __syncthreads();
    for (int p0 = blockIdx.x * kT; p0 < npix; p0 += gridDim.x * kT) {
        const int p = p0 + tid;
        if (p < npix) {
            float yv[32], g[32];
#pragma unroll
            for (int k0 = 0; k0 < 32; k0 += 8)
                if (k0 < C) unpack8(ld8(y + (size_t)p * C + k0), yv + k0);
#pragma unroll
            for (int k = 0; k < 32; k++) g[k] = 0.f;
            for (int c = 0; c < cout; c++) {
                const float dc = dout[(size_t)p * cout + c];
                s_d[tid * 33 + c] = dc;
#pragma unroll
                for (int k = 0; k < 32; k++)
                    if (k < C) g[k] += s_w[c * C + k] * dc;
            }
#pragma unroll
            for (int k0 = 0; k0 < 32; k0 += 8)
                if (k0 < C) {
                    float gk[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) gk[j] = yv[k0 + j] > 0.f ? g[k0 + j] : 0.f;
                    st8(dy + (size_t)p * C + k0, pack8(gk));
                }
#pragma unroll
            for (int k = 0; k < 32; k++)
                if (k < C) s_y[tid * 33 + k] = yv[k];
            s_y[tid * 33 + C] = 1.f;
        } else {
            for (int k = 0; k <= C; k++) s_y[tid * 33 + k] = 0.f;
            for (int c = 0; c < cout; c++) s_d[tid * 33 + c] = 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kE; j++) {
            const int e = tid + j * kT;
            if (e < ne) {
                const int c = e / (C + 1), k = e % (C + 1);
                float s = 0.f;
                for (int q = 0; q < kT; q++) s += s_d[q * 33 + c] * s_y[q * 33 + k];
                acc[j] += s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < kE; j++) {
        const int e = tid + j * kT;
        if (e < ne) {
            const int c = e / (C + 1), k = e % (C + 1);
            if (k < C) atomicAdd(dwh + c * C + k, acc[j]);
            else atomicAdd(dbh + c, acc[j]);
        }
    }
}

// weighted masked MSE: loss = sum_p m_p sum_c w_c (o - t)^2 / sum_p m_p,
// dout = dloss/do; msum = sum_p m_p (host value)
__global__ void k_mse(const float* __restrict__ o, const float* __restrict__ t, const float* __restrict__ m, int npix,
                      int cout, const float* __restrict__ cw, double inv_msum, float* __restrict__ dout,
                      double* __restrict__ loss) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        const float mp = m[p];
        for (int c = 0; c < cout; c++) {
            const float diff = o[(size_t)p * cout + c] - t[(size_t)p * cout + c];
            acc += (double)mp * cw[c] * diff * diff;
            dout[(size_t)p * cout + c] = (float)(2.0 * mp * cw[c] * diff * inv_msum);
        }
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        atomicAdd(loss, s * inv_msum);
    }
}

// Adam on the FP32 master parameters; bf16 copies of the conv weights follow
__global__ void k_adam(float* __restrict__ prm, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[e];
        const float mi = b1 * m[e] + (1.f - b1) * gi;
        const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        prm[e] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// normalisation of the network's input and output channels (up to 32 each)
struct Stats {
    float in_mean[32], in_std[32], out_mean[32], out_std[32];
};

// input channels of the warm-start network from the field planes (library
// layout, grid cell (i, j) -> pixel (j-1, i-1)): log10 n_e, log10 nu_m, |B|,
// the microwave field (zero here), the first potential corrections of the
// steps before the previous one and of the previous one; normalised, zero
// outside the grid.  With the two previous corrections the network can follow
// the plasma oscillation of the correction (period a few steps at 1e17 m^-3).
__global__ void k_features(const double* __restrict__ rhoe, const double* __restrict__ nu_m,
                           const double* __restrict__ Bx, const double* __restrict__ Br,
                           const double* __restrict__ dphi_prev2, const double* __restrict__ dphi_prev, int ni,
                           int nj, int ld, int H, int W, Stats st, float* __restrict__ out) {
    const int npix = H * W;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += gridDim.x * blockDim.x) {
        const int y = q / W, x = q % W;
        float f[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (y < nj && x < ni) {
            const size_t p = (size_t)(y + 1) * ld + (x + 1);
            f[0] = (float)log10(fmax(rhoe[p], 1.0));
            f[1] = (float)log10(fmax(nu_m[p], 1.0));
            f[2] = (float)sqrt(Bx[p] * Bx[p] + Br[p] * Br[p]);
            f[4] = (float)dphi_prev2[p];
            f[5] = (float)dphi_prev[p];
#pragma unroll
            for (int c = 0; c < 6; c++) f[c] = (f[c] - st.in_mean[c]) / st.in_std[c];
        }
#pragma unroll
        for (int c = 0; c < 6; c++) out[(size_t)q * 6 + c] = f[c];
    }
}

// input channels of the microwave warm-start network: log10 n_e, log10 nu_m1, |B|
// and the real and imaginary parts of the previous microwave fields Ex, Er, Ephi
// per unit excitation current (interleaved complex planes times escale, plane
// stride pl), grid cell (i, j) -> pixel (j-1, i-1); normalised, zero outside
__global__ void k_mw_features(const double* __restrict__ rhoe, const double* __restrict__ nu_m1,
                              const double* __restrict__ Bx, const double* __restrict__ Br,
                              const double* __restrict__ E3, double escale, size_t pl, int ni, int nj, int ld,
                              int H, int W, Stats st, float* __restrict__ out) {
    const int npix = H * W;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npix; q += gridDim.x * blockDim.x) {
        const int y = q / W, x = q % W;
        float f[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (y < nj && x < ni) {
            const size_t p = (size_t)(y + 1) * ld + (x + 1);
            f[0] = (float)log10(fmax(rhoe[p], 1.0));
            f[1] = (float)log10(fmax(nu_m1[p], 1.0));
            f[2] = (float)sqrt(Bx[p] * Bx[p] + Br[p] * Br[p]);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                f[3 + 2 * c] = (float)(E3[2 * (c * pl + p)] * escale);
                f[4 + 2 * c] = (float)(E3[2 * (c * pl + p) + 1] * escale);
            }
#pragma unroll
            for (int c = 0; c < 9; c++) f[c] = (f[c] - st.in_mean[c]) / st.in_std[c];
        }
#pragma unroll
        for (int c = 0; c < 9; c++) out[(size_t)q * 9 + c] = f[c];
    }
}

// the microwave guess: E_guess = ratio E_prev + jnow x the network's predicted
// change of the field per unit excitation (channels 2c, 2c+1 = real, imaginary
// part of field c, de-normalised) on the grid cells i = 1..ni, j = 1..nj;
// ratio E_prev elsewhere.  ratio = jnow / jprev: the system is linear in the
// excitation, so the previous fields scaled to the new excitation are the guess
// of an unchanged plasma
__global__ void k_mw_unpack(const float* __restrict__ o, int W, Stats st, const double* __restrict__ Eprev,
                            double ratio, double jnow, double* __restrict__ Eguess, size_t pl, int ni, int nj,
                            int ld) {
    const size_t n = 3 * pl;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(k / pl);
        const size_t p = k % pl;
        const int j = (int)(p / ld), i = (int)(p % ld);
        double re = ratio * Eprev[2 * k], im = ratio * Eprev[2 * k + 1];
        if (i >= 1 && i <= ni && j >= 1 && j <= nj) {
            const size_t q = ((size_t)(j - 1) * W + (i - 1)) * 6;
            re += jnow * (double)(o[q + 2 * c] * st.out_std[2 * c] + st.out_mean[2 * c]);
            im += jnow * (double)(o[q + 2 * c + 1] * st.out_std[2 * c + 1] + st.out_mean[2 * c + 1]);
        }
        Eguess[2 * k] = re;
        Eguess[2 * k + 1] = im;
    }
}

// one pass of a 5-point smoother on channel c of the network output over the
// first ny x nx pixels (the grid cells): v <- (4 v + vN + vS + vE + vW) / 8, a
// neighbour outside the cells replaced by v itself (no flux through the edges)
__global__ void k_smooth5(const float* __restrict__ src, float* __restrict__ dst, int cout, int c, int ny, int nx,
                          int W) {
    const int n = ny * nx;
    const size_t row = (size_t)W * cout;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int y = q / nx, x = q % nx;
        const size_t p = ((size_t)y * W + x) * cout + c;
        const float v = src[p];
        const float vn = y + 1 < ny ? src[p + row] : v;
        const float vs = y > 0 ? src[p - row] : v;
        const float ve = x + 1 < nx ? src[p + cout] : v;
        const float vw = x > 0 ? src[p - cout] : v;
        dst[p] = (4.f * v + vn + vs + ve + vw) * 0.125f;
    }
}

// guess = base + channel c of the network output (de-normalised) in the grid
// cells: the network predicts the change from the previous step's correction
__global__ void k_unpack(const float* __restrict__ o, int cout, int c, int ni, int nj, int ld, int W, float om,
                         float os, const double* __restrict__ base, double* __restrict__ dst) {
    const int n = ni * nj;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int y = q / ni, x = q % ni;
        const size_t p = (size_t)(y + 1) * ld + (x + 1);
        dst[p] = base[p] + (double)(o[((size_t)y * W + x) * cout + c] * os + om);
    }
}

// ---------------------------------------------------------------------------
// 3x3 convolution on the 5th-generation tensor cores (tcgen05, accumulator in
// tensor memory) with operands brought in by the tensor memory accelerator.
// A tile = R image rows x 128 consecutive pixels (the MMA's M: one TMEM lane
// per pixel) x N output channels.  Input channels go in chunks of 16 through a
// ring of S shared-memory stages in the canonical K-major layout without
// swizzle (8-row core matrices of 16 bytes; the two 8-channel halves of a chunk
// are one TMA box each, LBO apart):
//   A: R+2 halo rows x 130 pixels      (pixel p of halo row h at (h*130+p)*16)
//   B: 9 tap slabs of N x 16 weights   (channel co of tap t at (t*N+co)*16)
// so the A operand of output row r and tap (dy, dx) is the same tile started
// ((r+dy)*130+dx)*16 bytes further: one descriptor offset per (row, tap), and
// the R output rows share their halo rows.  The weights have a layout of their
// own, [Cin/8][9][Cout][8], so that the B half of a chunk is one box.
//
// Persistent and warp-specialised: one CTA per SM walks the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...; warp 0 issues the loads (the
// stage's full barrier counts the transaction bytes), warp 1 the MMAs (M=128,
// N, K=16; tcgen05.commit to the stage's empty barrier releases it), and warps
// 2-5 drain the accumulator with tcgen05.ld (warp w reads TMEM lanes
// 32(w%4)..+31).  Two accumulator buffers in TMEM let the epilogue of one tile
// run under the loads and MMAs of the next.  Every wait is bounded: one that
// gives up sets the error flag (the call's output is then not valid), and the
// CTA waits, again bounded, for its copies and MMAs in flight before it frees
// its tensor memory.
// ---------------------------------------------------------------------------
constexpr int TC_M = 128;        // pixels per row tile
constexpr int TC_HW = TC_M + 2;  // halo row width
constexpr int TC_THREADS = 192;  // producer warp, MMA warp, 4 epilogue warps

template <int N, int R>
struct TcShape {
    // one stage = 32 input channels: the A box (R+2 halo rows x 130 pixels x 64 B)
    // and the B box (9 taps x N output channels x 64 B), each 1024-byte aligned
    static constexpr int kA = ((R + 2) * TC_HW * 64 + 1023) / 1024 * 1024;
    static constexpr int kB = (9 * N * 64 + 1023) / 1024 * 1024;
    static constexpr int kStage = kA + kB;
    static constexpr int kFit = (210 * 1024) / kStage;
    static constexpr int kStages = kFit < 2 ? 2 : (kFit > 8 ? 8 : kFit);
    // barriers after the stages: full[S], empty[S], tfull[2], tempty[2], fin; then the TMEM address
    static constexpr int kBar = kStages * kStage;
    static constexpr int kNBar = 2 * kStages + 5;
    static constexpr int kUsed = kBar + kNBar * 8 + 8 + 1024;  // + alignment slack of the dynamic base
    static constexpr int kSmem = kUsed < 120 * 1024 ? 120 * 1024 : kUsed;  // one CTA per SM
    static constexpr uint32_t kTx = (uint32_t)((R + 2) * TC_HW * 64 + 9 * N * 64);
    static constexpr uint32_t kCols = 2 * R * N <= 64 ? 64 : (2 * R * N <= 128 ? 128 : (2 * R * N <= 256 ? 256 : 512));
    static_assert(2 * R * N <= 512, "two accumulator buffers in the 512 TMEM columns");
    static_assert(kUsed <= 227 * 1024, "shared memory per CTA");
};

// the (N, R) tiles instantiated
#define CTH_TC_TILES(X) \
    X(128, 2) X(128, 1) X(96, 2) X(96, 1) X(64, 4) X(64, 2) X(64, 1) X(32, 4) X(32, 2) X(32, 1)

// shared-memory matrix descriptor, K-major with the 64-byte swizzle (rows of 64
// bytes = 32 bf16 along K, 8-row groups 512 bytes apart, layout type 4 in
// [61,64)).  TMA and the MMA both apply the swizzle to the absolute
// shared-memory address of a 1024-byte aligned tile, so a start on any 64-byte
// row reads the rows TMA wrote there; the base offset (bits [49,52)) stays 0.
__device__ __forceinline__ uint64_t tc_desc_sw64(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;              // leading byte offset 16 (unused within the 64-byte row)
    d |= (uint64_t)(512 >> 4) << 32;     // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;              // version
    d |= (uint64_t)4 << 61;              // SWIZZLE_64B
    return d;
}

// instruction descriptor of kind::f16: D F32, A and B BF16, both K-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, int polls) {
    for (int it = 0; it < polls; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 3-D tiled TMA load into this CTA's shared memory, completion on bar
__device__ __forceinline__ void tc_load3(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

template <int N, int R>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_conv3_tc(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tw, ConvArgs a,
               int* __restrict__ err) {
    using T = TcShape<N, R>;
    constexpr int S = T::kStages;
    extern __shared__ __align__(1024) unsigned char tsm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tx = (a.W + TC_M - 1) / TC_M, ty = (a.H + R - 1) / R;
    const int ntiles = tx * ty * (a.Cout / N), nk = a.Cin / 32;
    // the swizzled boxes want 1024-byte aligned stages
    const uint32_t base = (smem_u32(tsm) + 1023u) & ~1023u;
    unsigned char* tbase = tsm + (base - smem_u32(tsm));
    const uint32_t bars = base + (uint32_t)T::kBar;
    const uint32_t full0 = bars, empty0 = bars + 8u * S, tfull0 = bars + 16u * S, tempty0 = tfull0 + 16u,
                   fin = tempty0 + 16u;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(tbase + T::kBar + T::kNBar * 8);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(T::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 32) {
        for (int b = 0; b < 2 * S; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bars + 8u * b));
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tfull0 + 8u * b));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(tempty0 + 8u * b));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fin));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    int fail = 0, issued = 0;
    if (tid == 0 && !a.stall) {
        // producer: chunk after chunk of every tile through the ring
        int it = 0;
        for (int t = blockIdx.x; t < ntiles && !fail; t += gridDim.x) {
            const int x0 = (t % tx) * TC_M, y0 = ((t / tx) % ty) * R, co0 = (t / (tx * ty)) * N;
            for (int k = 0; k < nk; k++, it++) {
                const int s = it % S;
                if (it >= S && !tc_wait(empty0 + 8u * s, (uint32_t)((it / S - 1) & 1), a.wait_polls)) {
                    fail = 1;
                    break;
                }
                const uint32_t st = base + (uint32_t)(s * T::kStage), fb = full0 + 8u * s;
                tc_expect(fb, T::kTx);
                tc_load3(st, &tin, fb, 32 * k, x0 - 1, y0 - 1);
                tc_load3(st + T::kA, &tw, fb, 0, co0, 9 * k);
                issued = it + 1;
            }
        }
    } else if (tid == 32) {
        // MMA issuer: R x 9 MMAs per chunk into accumulator buffer (local tile & 1)
        constexpr uint32_t idesc = tc_idesc(N);
        int it = 0, lt = 0;
        for (int t = blockIdx.x; t < ntiles && !fail; t += gridDim.x, lt++) {
            const int b = lt & 1;
            if (lt >= 2 && !tc_wait(tempty0 + 8u * b, (uint32_t)((lt / 2 - 1) & 1), a.wait_polls)) {
                fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + (uint32_t)(b * R * N);
            for (int k = 0; k < nk; k++, it++) {
                const int s = it % S;
                if (!tc_wait(full0 + 8u * s, (uint32_t)((it / S) & 1), a.wait_polls)) {
                    fail = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t st = base + (uint32_t)(s * T::kStage);
#pragma unroll
                for (int r = 0; r < R; r++) {
#pragma unroll
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) {
                            const uint64_t da =
                                tc_desc_sw64(st + (uint32_t)(((r + dy) * TC_HW + dx) * 64 + kk * 32));
                            const uint64_t db = tc_desc_sw64(st + (uint32_t)(T::kA + tap * N * 64 + kk * 32));
                            tc_mma(acc + (uint32_t)(r * N), da, db, idesc, (k > 0 || tap > 0 || kk > 0) ? 1u : 0u);
                        }
                    }
                }
                tc_commit(empty0 + 8u * s);
            }
            if (!fail) tc_commit(tfull0 + 8u * b);
        }
        tc_commit(fin);
    } else if (warp >= 2) {
        // epilogue: pixel 32 (warp % 4) + lane of the tile, all R rows and N channels
        const int q = warp & 3;
        const float* __restrict__ bias = a.bias;
        const bf16* __restrict__ gate = a.gate;
        bf16* __restrict__ out = a.out;
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, lt++) {
            const int b = lt & 1;
            if (!tc_wait(tfull0 + 8u * b, (uint32_t)((lt / 2) & 1), a.wait_polls)) {
                fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int x0 = (t % tx) * TC_M, y0 = ((t / tx) % ty) * R, co0 = (t / (tx * ty)) * N;
            const int gx = x0 + 32 * q + lane;
#pragma unroll 1
            for (int r = 0; r < R; r++) {
                const int gy = y0 + r;
                const bool live = gx < a.W && gy < a.H;
                const size_t pix = (size_t)gy * a.W + gx;
#pragma unroll 1
                for (int cb = 0; cb < N / 32; cb++) {
                    uint32_t v[32];
                    tc_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * R * N + r * N + cb * 32), v);
                    if (!live) continue;
                    const int c0 = co0 + cb * 32;
                    uint4 gv[4], ov[4];
                    if (gate)
#pragma unroll
                        for (int g = 0; g < 4; g++) gv[g] = ld8(gate + pix * a.gate_cs + a.gate_coff + c0 + 8 * g);
                    if (a.accumulate)
#pragma unroll
                        for (int g = 0; g < 4; g++) ov[g] = ld8(out + pix * a.out_cs + a.out_coff + c0 + 8 * g);
#pragma unroll
                    for (int g = 0; g < 4; g++) {
                        float f[8];
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            f[j] = __uint_as_float(v[8 * g + j]);
                            if (bias) f[j] += __ldg(bias + c0 + 8 * g + j);
                            if (a.relu) f[j] = fmaxf(f[j], 0.f);
                        }
                        if (gate) {
                            float gf[8];
                            unpack8(gv[g], gf);
#pragma unroll
                            for (int j = 0; j < 8; j++)
                                if (!(gf[j] > 0.f)) f[j] = 0.f;
                        }
                        if (a.accumulate) {
                            float of[8];
                            unpack8(ov[g], of);
#pragma unroll
                            for (int j = 0; j < 8; j++) f[j] += of[j];
                        }
                        st8(out + pix * a.out_cs + a.out_coff + c0 + 8 * g, pack8(f));
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc_arrive(tempty0 + 8u * b);
        }
    }
    __syncwarp();
    // CTA-uniform outcome, so every thread takes the same path at the barriers
    const bool ok = __syncthreads_and(fail == 0 ? 1 : 0) != 0;
    if (!ok) {
        if (tid == 0) {
            atomicExch(err, 1);
            for (int k = issued > S ? issued - S : 0; k < issued; k++)
                tc_wait(full0 + 8u * (k % S), (uint32_t)((k / S) & 1), a.wait_polls);
        }
    }
    tc_wait(fin, 0u, a.wait_polls);  // the MMAs are complete before the tensor memory is freed
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::kCols));
}

inline dim3 grid1(size_t n, int bs = 256) {
    size_t b = (n + bs - 1) / bs;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return dim3((unsigned)b);
}

}  // namespace unet
}  // namespace cth

using namespace cth;
using namespace cth::unet;

// ---------------------------------------------------------------------------
// the network object
// ---------------------------------------------------------------------------
namespace {

struct Conv {
    int cin, cout, H, W;
    size_t w_off, b_off;  // into the FP32 parameter vector (weights [cout][9][cin], bias [cout])
    size_t wb_off;        // into the bf16 weight vector
    TensorRef in, out;    // forward operands
    TensorRef din, dout;  // gradients (din.p null: not needed)
    const bf16* out_gate_for_din;  // ReLU output that din belongs to (null: din is not gated)
    int din_accumulate;
};

}  // namespace

struct cth_unet {
    int device = 0;
    int sms = 148;  // multiprocessors of the device (persistent grids)
    int max_ctas = 0;  // cap of the persistent convolution grid (0: one CTA per SM)
    int H = 0, W = 0, cin = 0, cout = 0, base = 0;
    int cpad = 32;
    std::vector<Conv> convs;
    size_t nparam = 0, nw_bf16 = 0;
    size_t head_w = 0, head_b = 0;
    float* prm = nullptr;  // FP32 master parameters
    float* grad = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    bf16* wb = nullptr;    // bf16 conv weights
    bf16* wt = nullptr;    // transposed / flipped conv weights (input gradients)
    bf16* wbt = nullptr;   // wb and wt in the tcgen05 layout [Cin/8][9][Cout][8]
    bf16* wtt = nullptr;
    std::vector<void*> bufs;
    bf16* x_in = nullptr;  // packed input
    bf16* y_last = nullptr;  // last decoder activation (input of the head)
    bf16* dy_last = nullptr;
    float* out = nullptr;    // last forward output (FP32 NHWC)
    float* dout = nullptr;
    double* loss = nullptr;
    float* cw = nullptr;     // per-output-channel loss weights
    Stats stats{};
    float* feat = nullptr;   // input features of the warm-start prediction
    float* feat_mw = nullptr; // input features of the microwave prediction
    float* smooth = nullptr; // ping-pong buffer of the prediction smoother
    int smooth_passes = 0;   // 5-point smoothing passes on the predicted change
    long long launches = 0;  // kernels launched by the forward passes and predictions
    bool use_tc = true;      // convolutions on tcgen05 (false: warp-level mma.sync kernel)
    int wait_polls = 1 << 20;  // polls of each mbarrier wait of the tcgen05 kernel
    int stall = 0;             // test of the bounded waits: the tcgen05 kernel issues no loads
    int* err = nullptr;      // device flag: a bounded wait of a tcgen05 convolution gave up
    struct Pool { TensorRef src; bf16* dst; int C, Ho, Wo; bf16* ddst; };
    struct Up { bf16* src; int C, Hi, Wi; TensorRef dst; bf16* dsrc; TensorRef ddst; };
    std::vector<Pool> pools;
    std::vector<Up> ups;
};

namespace {

bf16* alloc_bf16(cth_unet* n, size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, count * sizeof(bf16)) != cudaSuccess) return nullptr;
    cth::zero_fill(p, count * sizeof(bf16));
    n->bufs.push_back(p);
    return (bf16*)p;
}

// forward order of the layers (indices into convs):
//   0 e0a 1 e0b | 2 e1a 3 e1b | 4 e2a 5 e2b | 6 ba 7 bb | 8 d2a 9 d2b | 10 d1a 11 d1b | 12 d0a 13 d0b
int build(cth_unet* n) {
    const int H0 = n->H, W0 = n->W, B = n->base;
    const int Hs[4] = {H0, H0 / 2, H0 / 4, H0 / 8}, Ws[4] = {W0, W0 / 2, W0 / 4, W0 / 8};
    const int C[4] = {B, 2 * B, 4 * B, 8 * B};
    auto px = [&](int l) { return (size_t)Hs[l] * Ws[l]; };
    n->x_in = alloc_bf16(n, px(0) * n->cpad);
    // activations and their gradients
    bf16 *e_a[3], *cat[3], *pool[3], *d_a[3], *d_b[3];
    bf16 *ge_a[3], *gcat[3], *gpool[3], *gd_a[3], *gd_b[3];
    for (int l = 0; l < 3; l++) {
        e_a[l] = alloc_bf16(n, px(l) * C[l]);
        cat[l] = alloc_bf16(n, px(l) * 3 * C[l]);
        pool[l] = alloc_bf16(n, px(l + 1) * C[l]);
        d_a[l] = alloc_bf16(n, px(l) * C[l]);
        d_b[l] = alloc_bf16(n, px(l) * C[l]);
        ge_a[l] = alloc_bf16(n, px(l) * C[l]);
        gcat[l] = alloc_bf16(n, px(l) * 3 * C[l]);
        gpool[l] = alloc_bf16(n, px(l + 1) * C[l]);
        gd_a[l] = alloc_bf16(n, px(l) * C[l]);
        gd_b[l] = alloc_bf16(n, px(l) * C[l]);
    }
    bf16* ba = alloc_bf16(n, px(3) * C[3]);
    bf16* bb = alloc_bf16(n, px(3) * C[3]);
    bf16* gba = alloc_bf16(n, px(3) * C[3]);
    bf16* gbb = alloc_bf16(n, px(3) * C[3]);
    for (void* p : n->bufs)
        if (!p) return CTH_ERR_ALLOC;
    size_t off = 0, woff = 0;
    auto add = [&](int cin, int cout, int l, TensorRef in, TensorRef out, TensorRef din, TensorRef dout,
                   const bf16* gate, int acc) {
        Conv c;
        c.cin = cin; c.cout = cout; c.H = Hs[l]; c.W = Ws[l];
        c.w_off = off; off += (size_t)cout * 9 * cin;
        c.b_off = off; off += cout;
        c.wb_off = woff; woff += (size_t)cout * 9 * cin;
        c.in = in; c.out = out; c.din = din; c.dout = dout;
        c.out_gate_for_din = gate;
        c.din_accumulate = acc;
        n->convs.push_back(c);
    };
    const TensorRef none{nullptr, 0, 0};
    // encoder
    TensorRef xin{n->x_in, n->cpad, 0};
    TensorRef src = xin;
    TensorRef dsrc = none;
    const bf16* gsrc = nullptr;
    for (int l = 0; l < 3; l++) {
        const int cin = (l == 0) ? n->cpad : C[l - 1];
        add(cin, C[l], l, src, TensorRef{e_a[l], C[l], 0}, dsrc, TensorRef{ge_a[l], C[l], 0}, gsrc, 0);
        add(C[l], C[l], l, TensorRef{e_a[l], C[l], 0}, TensorRef{cat[l], 3 * C[l], 0}, TensorRef{ge_a[l], C[l], 0},
            TensorRef{gcat[l], 3 * C[l], 0}, e_a[l], 0);
        n->pools.push_back({TensorRef{cat[l], 3 * C[l], 0}, pool[l], C[l], Hs[l + 1], Ws[l + 1], gpool[l]});
        src = TensorRef{pool[l], C[l], 0};
        dsrc = TensorRef{gpool[l], C[l], 0};
        gsrc = nullptr;  // pooled tensors are linear in the ReLU outputs
    }
    // bottom
    add(C[2], C[3], 3, src, TensorRef{ba, C[3], 0}, dsrc, TensorRef{gba, C[3], 0}, nullptr, 0);
    add(C[3], C[3], 3, TensorRef{ba, C[3], 0}, TensorRef{bb, C[3], 0}, TensorRef{gba, C[3], 0},
        TensorRef{gbb, C[3], 0}, ba, 0);
    // decoder
    bf16* below = bb;
    bf16* gbelow = gbb;
    int cbelow = C[3];
    for (int l = 2; l >= 0; l--) {
        n->ups.push_back({below, cbelow, Hs[l + 1], Ws[l + 1], TensorRef{cat[l], 3 * C[l], C[l]}, gbelow,
                          TensorRef{gcat[l], 3 * C[l], C[l]}});
        add(3 * C[l], C[l], l, TensorRef{cat[l], 3 * C[l], 0}, TensorRef{d_a[l], C[l], 0},
            TensorRef{gcat[l], 3 * C[l], 0}, TensorRef{gd_a[l], C[l], 0}, cat[l], 0);
        add(C[l], C[l], l, TensorRef{d_a[l], C[l], 0}, TensorRef{d_b[l], C[l], 0}, TensorRef{gd_a[l], C[l], 0},
            TensorRef{gd_b[l], C[l], 0}, d_a[l], 0);
        below = d_b[l];
        gbelow = gd_b[l];
        cbelow = C[l];
    }
    n->y_last = d_b[0];
    n->dy_last = gd_b[0];
    n->head_w = off; off += (size_t)n->cout * B;
    n->head_b = off; off += n->cout;
    n->nparam = off;
    n->nw_bf16 = woff;
    const size_t npx0 = px(0);
    CTH_CUDA(cudaMalloc(&n->prm, off * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->grad, off * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->adam_m, off * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->adam_v, off * sizeof(float)));
    CTH_CUDA(cth::zero_fill(n->prm, off * sizeof(float)));
    CTH_CUDA(cth::zero_fill(n->grad, off * sizeof(float)));
    CTH_CUDA(cth::zero_fill(n->adam_m, off * sizeof(float)));
    CTH_CUDA(cth::zero_fill(n->adam_v, off * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->wb, woff * sizeof(bf16)));
    CTH_CUDA(cudaMalloc(&n->wt, woff * sizeof(bf16)));
    CTH_CUDA(cudaMalloc(&n->wbt, woff * sizeof(bf16)));
    CTH_CUDA(cudaMalloc(&n->wtt, woff * sizeof(bf16)));
    CTH_CUDA(cudaMalloc(&n->out, npx0 * n->cout * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->dout, npx0 * n->cout * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->loss, sizeof(double)));
    CTH_CUDA(cudaMalloc(&n->cw, n->cout * sizeof(float)));
    CTH_CUDA(cudaMalloc(&n->err, sizeof(int)));
    CTH_CUDA(cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, n->device));
    CTH_CUDA(cth::zero_fill(n->err, sizeof(int)));
#define CTH_TC_ATTR(NN, RR)                                                                   \
    CTH_CUDA(cudaFuncSetAttribute(k_conv3_tc<NN, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  TcShape<NN, RR>::kSmem));
    CTH_TC_TILES(CTH_TC_ATTR)
#undef CTH_TC_ATTR
    std::vector<float> ones(n->cout, 1.f);
    CTH_CUDA(cudaMemcpy(n->cw, ones.data(), n->cout * sizeof(float), cudaMemcpyHostToDevice));
    return CTH_OK;
}

// bf16 weights (and their transposes) from the FP32 parameters
int sync_weights(cth_unet* n, cudaStream_t s) {
    for (const Conv& c : n->convs) {
        const size_t nw = (size_t)c.cout * 9 * c.cin;
        k_weights<<<grid1(nw), 256, 0, s>>>(n->prm + c.w_off, c.cout, c.cin, n->wb + c.wb_off, n->wt + c.wb_off,
                                            n->wbt + c.wb_off, n->wtt + c.wb_off);
    }
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

// cuTensorMapEncodeTiled from the driver (no link against it)
typedef CUresult (*TmapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

TmapEncodeFn tmap_encode() {
    static const TmapEncodeFn fn = []() -> TmapEncodeFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<TmapEncodeFn>(p);
    }();
    return fn;
}

// 3-D bf16 tensor map: extents d0 (contiguous), d1, d2; byte strides s1, s2 of
// dimensions 1 and 2; box b0 x b1 x b2; zero fill outside the extents; swizzle swz
bool tmap3(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1, uint64_t s2,
           uint32_t b0, uint32_t b1, uint32_t b2, CUtensorMapSwizzle swz) {
    const TmapEncodeFn fn = tmap_encode();
    if (!fn) return false;
    cuuint64_t dims[3] = {d0, d1, d2}, strides[2] = {s1, s2};
    cuuint32_t box[3] = {b0, b1, b2}, es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// tcgen05 tile of a convolution: the widest N (output channels) dividing Cout,
// then the most rows R that still give every SM two tiles; without such
// a tiling the widest N with one row
struct TcTile {
    int n, r;
};
TcTile tc_tile(int cout, int H, int W, int sms) {
    const int cols = (W + TC_M - 1) / TC_M;
    for (int N : {128, 96, 64, 32}) {
        if (cout % N) continue;
        for (int R : {4, 2, 1}) {
            if (R * N > 256) continue;
            if ((long)cols * ((H + R - 1) / R) * (cout / N) >= 2L * sms) return {N, R};
        }
    }
    for (int N : {128, 96, 64, 32})
        if (cout % N == 0) return {N, 1};
    return {0, 0};
}

int launch_conv(cth_unet* n, const ConvArgs& a, cudaStream_t s) {
    const TcTile t = n->use_tc ? tc_tile(a.Cout, a.H, a.W, n->sms) : TcTile{0, 0};
    if (t.n && a.Cin % 32 == 0 && a.Cout % 32 == 0 && a.in_cs % 8 == 0 && a.in_coff % 8 == 0) {
        // A: 32 channels x 130 pixels x R+2 rows per box; B: the [Cin/32][9][Cout][32]
        // weights, 32 channels x N x 9 taps per box; both in 64-byte swizzled rows
        CUtensorMap ti, tw;
        if (!tmap3(&ti, a.in + a.in_coff, (uint64_t)a.Cin, (uint64_t)a.W, (uint64_t)a.H, (uint64_t)a.in_cs * 2,
                   (uint64_t)a.W * a.in_cs * 2, 32, TC_HW, (uint32_t)(t.r + 2), CU_TENSOR_MAP_SWIZZLE_64B) ||
            !tmap3(&tw, a.wtc, 32, (uint64_t)a.Cout, (uint64_t)9 * a.Cin / 32, 64, (uint64_t)a.Cout * 64, 32,
                   (uint32_t)t.n, 9, CU_TENSOR_MAP_SWIZZLE_64B)) {
            set_error("cth_unet: tensor map encoding failed");
            return CTH_ERR_CUDA;
        }
        // persistent: at most one CTA per SM, each walking its share of the tiles
        const long tiles = (long)((a.W + TC_M - 1) / TC_M) * ((a.H + t.r - 1) / t.r) * (a.Cout / t.n);
        const long cap = n->max_ctas > 0 ? std::min(n->max_ctas, n->sms) : n->sms;
        const unsigned grd = (unsigned)std::min<long>(tiles, cap);
        ConvArgs ta = a;
        ta.wait_polls = n->wait_polls;
        ta.stall = n->stall;
#define CTH_TC_LAUNCH(NN, RR)                                                                    \
    if (t.n == NN && t.r == RR) {                                                                \
        k_conv3_tc<NN, RR><<<grd, TC_THREADS, TcShape<NN, RR>::kSmem, s>>>(ti, tw, ta, n->err);  \
        return CTH_OK;                                                                           \
    }
        CTH_TC_TILES(CTH_TC_LAUNCH)
#undef CTH_TC_LAUNCH
        set_error("cth_unet: no tcgen05 tile for this convolution");
        return CTH_ERR_ARG;
    }
    dim3 grd((a.W + TW - 1) / TW, (a.H + TH - 1) / TH, a.Cout / 32);
    k_conv3_fwd<<<grd, 128, 0, s>>>(a);
    return CTH_OK;
}

int conv_fwd(cth_unet* n, const Conv& c, cudaStream_t s) {
    ConvArgs a{};
    a.in = c.in.p; a.in_cs = c.in.cs; a.in_coff = c.in.coff; a.Cin = c.cin;
    a.w = n->wb + c.wb_off;
    a.wtc = n->wbt + c.wb_off;
    a.bias = n->prm + c.b_off;
    a.out = c.out.p; a.out_cs = c.out.cs; a.out_coff = c.out.coff; a.Cout = c.cout;
    a.H = c.H; a.W = c.W;
    a.relu = 1;
    return launch_conv(n, a, s);
}

int conv_bwd(cth_unet* n, const Conv& c, cudaStream_t s) {
    // weight and bias gradients
    WgradArgs w{};
    w.dy = c.dout.p; w.dy_cs = c.dout.cs; w.dy_coff = c.dout.coff; w.Cout = c.cout;
    w.in = c.in.p; w.in_cs = c.in.cs; w.in_coff = c.in.coff; w.Cin = c.cin;
    w.H = c.H; w.W = c.W;
    w.dw = n->grad + c.w_off;
    const int npatch = ((c.W + TW - 1) / TW) * ((c.H + TH - 1) / TH);
    const int tiles = (c.cout / 32) * (c.cin / 32);
    int ppc = (int)std::ceil((double)npatch * tiles / (n->sms * 4.0));
    ppc = std::max(1, std::min(ppc, npatch));
    w.patches_per_cta = ppc;
    dim3 gw((npatch + ppc - 1) / ppc, c.cout / 32, c.cin / 32);
    k_conv3_wgrad<<<gw, 288, 0, s>>>(w);
    const int npix = c.H * c.W;
    {
        const int lanes = 256 / (c.cout / 8);
        const int nb = std::max(1, std::min(2 * n->sms, (npix + lanes - 1) / lanes));
        k_bias_grad<<<nb, 256, 0, s>>>(c.dout.p, c.dout.cs, c.dout.coff, c.cout, npix, n->grad + c.b_off);
    }
    if (!c.din.p) return CTH_OK;
    ConvArgs a{};
    a.in = c.dout.p; a.in_cs = c.dout.cs; a.in_coff = c.dout.coff; a.Cin = c.cout;
    a.w = n->wt + c.wb_off;
    a.wtc = n->wtt + c.wb_off;
    a.bias = nullptr;
    a.out = c.din.p; a.out_cs = c.din.cs; a.out_coff = c.din.coff; a.Cout = c.cin;
    a.H = c.H; a.W = c.W;
    a.relu = 0;
    a.gate = c.out_gate_for_din;
    a.gate_cs = c.din.cs; a.gate_coff = c.din.coff;
    a.accumulate = c.din_accumulate;
    return launch_conv(n, a, s);
}

int forward(cth_unet* n, const float* in, cudaStream_t s) {
    const size_t npx = (size_t)n->H * n->W;
    n->launches += 2 + (long long)n->convs.size() + (long long)n->pools.size() + (long long)n->ups.size();
    k_pack<<<grid1(npx), 256, 0, s>>>(in, n->cin, (int)npx, n->cpad, n->x_in);
    const auto& C = n->convs;
    int up = 0;
    for (size_t k = 0; k < C.size(); k++) {
        const int rc = conv_fwd(n, C[k], s);
        if (rc != CTH_OK) return rc;
        if (k == 1 || k == 3 || k == 5) {
            const auto& p = n->pools[k / 2];
            k_pool2<<<grid1((size_t)p.Ho * p.Wo * p.C / 8), 256, 0, s>>>(p.src.p, p.src.cs, p.src.coff, p.C, p.Ho, p.Wo,
                                                                      p.dst, p.C);
        }
        if (k == 7 || k == 9 || k == 11) {
            const auto& u = n->ups[up++];
            k_up2<<<grid1((size_t)u.Hi * u.Wi * u.C / 8), 256, 0, s>>>(u.src, u.C, u.C, u.Hi, u.Wi, u.dst.p, u.dst.cs,
                                                                        u.dst.coff);
        }
    }
    const int B = n->base;
    k_head_fwd<<<grid1(npx), 256, 0, s>>>(n->y_last, B, (int)npx, n->prm + n->head_w,
                                                             n->prm + n->head_b, n->cout, n->out);
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

int backward(cth_unet* n, const float* dout, cudaStream_t s) {
    const size_t npx = (size_t)n->H * n->W;
    const int B = n->base;
    const unsigned nhb = std::max<unsigned>(1, std::min<unsigned>(4u * n->sms, (unsigned)((npx + 127) / 128)));
    k_head_bwd<<<nhb, 128, 0, s>>>(n->y_last, B, (int)npx, n->prm + n->head_w, n->cout,
                                                            dout, n->dy_last, n->grad + n->head_w,
                                                            n->grad + n->head_b);
    const auto& C = n->convs;
    // the decoder convs write the concatenation gradients whole; the pooling
    // gradients are then added into their skip channels
    for (int k = (int)C.size() - 1; k >= 0; k--) {
        const int rc = conv_bwd(n, C[k], s);
        if (rc != CTH_OK) return rc;
        if (k == 12 || k == 10 || k == 8) {
            const auto& u = n->ups[(k - 8) / 2];
            k_up2_bwd<<<grid1((size_t)u.Hi * u.Wi * u.C / 8), 256, 0, s>>>(u.ddst.p, u.ddst.cs, u.ddst.coff, u.C, u.Hi,
                                                                      u.Wi, u.dsrc, u.C);
        }
        if (k == 6 || k == 4 || k == 2) {
            const auto& p = n->pools[k / 2 - 1];
            const TensorRef dskip = n->convs[k - 1].dout;
            k_pool2_bwd<<<grid1((size_t)4 * p.Ho * p.Wo * p.C / 8), 256, 0, s>>>(p.ddst, p.C, p.C, p.Ho, p.Wo, dskip.p,
                                                                             dskip.cs, dskip.coff, p.src.p, p.src.cs,
                                                                             p.src.coff);
        }
    }
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

cth_unet* cth_unet_create(int H, int W, int cin, int cout, int base, int device) {
    if (H < 8 || W < 8 || H % 8 || W % 8 || cin < 1 || cin > 32 || cout < 1 || cout > 32 || base != 32) {
        set_error("cth_unet_create: H, W multiples of 8, 1 <= cin, cout <= 32, base 32");
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        set_error("cth_unet_create: cudaSetDevice failed");
        return nullptr;
    }
    cth_unet* n = new cth_unet();
    n->device = device;
    n->H = H; n->W = W; n->cin = cin; n->cout = cout; n->base = base;
    if (build(n) != CTH_OK) {
        cth_unet_destroy(n);
        return nullptr;
    }
    return n;
}

void cth_unet_destroy(cth_unet* n) {
    if (!n) return;
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    for (void* p : n->bufs) cudaFree(p);
    for (void* p : {(void*)n->prm, (void*)n->grad, (void*)n->adam_m, (void*)n->adam_v, (void*)n->wb, (void*)n->wt,
                    (void*)n->wbt, (void*)n->wtt,
                    (void*)n->out, (void*)n->dout, (void*)n->loss, (void*)n->cw, (void*)n->feat, (void*)n->err,
                    (void*)n->smooth, (void*)n->feat_mw})
        if (p) cudaFree(p);
    delete n;
}

long long cth_unet_nparams(const cth_unet* n) { return n ? (long long)n->nparam : -1; }

long long cth_unet_launch_count(const cth_unet* n) { return n ? n->launches : -1; }

int cth_unet_set_tensor_cores(cth_unet* n, int tcgen05) {
    if (!n) { set_error("cth_unet_set_tensor_cores: null network"); return CTH_ERR_ARG; }
    n->use_tc = tcgen05 != 0;
    return CTH_OK;
}

int cth_unet_set_smoothing(cth_unet* n, int passes) {
    if (!n || passes < 0 || passes > 64) {
        set_error("cth_unet_set_smoothing: passes in [0, 64]");
        return CTH_ERR_ARG;
    }
    n->smooth_passes = passes;
    return CTH_OK;
}

int cth_unet_check(cth_unet* n) {
    if (!n) { set_error("cth_unet_check: null network"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    CTH_CUDA(cudaDeviceSynchronize());
    int e = 0;
    CTH_CUDA(cudaMemcpy(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        // reported once: the flag is cleared for the following calls
        CTH_CUDA(cth::zero_fill(n->err, sizeof(int)));
        set_error("cth_unet: a tensor-core convolution gave up waiting (its output is not valid)");
        return CTH_ERR_CUDA;
    }
    return CTH_OK;
}

int cth_unet_set_grid_limit(cth_unet* n, int ctas) {
    if (!n || ctas < 0) {
        set_error("cth_unet_set_grid_limit: invalid arguments");
        return CTH_ERR_ARG;
    }
    n->max_ctas = ctas;
    return CTH_OK;
}

int cth_unet_set_wait_test(cth_unet* n, int stall, int polls) {
    if (!n || polls < 1) {
        set_error("cth_unet_set_wait_test: invalid arguments");
        return CTH_ERR_ARG;
    }
    n->stall = stall != 0;
    n->wait_polls = polls;
    return CTH_OK;
}

int cth_unet_set_params(cth_unet* n, const float* host, long long count) {
    if (!n || !host || count != (long long)n->nparam) { set_error("cth_unet_set_params: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    CTH_CUDA(cudaMemcpy(n->prm, host, n->nparam * sizeof(float), cudaMemcpyHostToDevice));
    CTH_CUDA(cth::zero_fill(n->adam_m, n->nparam * sizeof(float)));
    CTH_CUDA(cth::zero_fill(n->adam_v, n->nparam * sizeof(float)));
    int rc = sync_weights(n, 0);
    if (rc != CTH_OK) return rc;
    CTH_CUDA(cudaDeviceSynchronize());
    return CTH_OK;
}

int cth_unet_get_params(const cth_unet* n, float* host, long long count) {
    if (!n || !host || count != (long long)n->nparam) { set_error("cth_unet_get_params: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    CTH_CUDA(cudaDeviceSynchronize());
    CTH_CUDA(cudaMemcpy(host, n->prm, n->nparam * sizeof(float), cudaMemcpyDeviceToHost));
    return CTH_OK;
}

int cth_unet_get_grads(const cth_unet* n, float* host, long long count) {
    if (!n || !host || count != (long long)n->nparam) { set_error("cth_unet_get_grads: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    CTH_CUDA(cudaDeviceSynchronize());
    CTH_CUDA(cudaMemcpy(host, n->grad, n->nparam * sizeof(float), cudaMemcpyDeviceToHost));
    return CTH_OK;
}

int cth_unet_set_loss_weights(cth_unet* n, const float* w_host) {
    if (!n || !w_host) { set_error("cth_unet_set_loss_weights: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    CTH_CUDA(cudaMemcpy(n->cw, w_host, n->cout * sizeof(float), cudaMemcpyHostToDevice));
    return CTH_OK;
}

// forward pass of the FP32 NHWC input (H x W x cin, device); the FP32 NHWC
// output (H x W x cout) is copied to out (device) when out is not null
int cth_unet_forward(cth_unet* n, const float* in, float* out, void* stream) {
    if (!n || !in) { set_error("cth_unet_forward: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    cudaStream_t s = (cudaStream_t)stream;
    int rc = forward(n, in, s);
    if (rc != CTH_OK) return rc;
    if (out)
        CTH_CUDA(cudaMemcpyAsync(out, n->out, (size_t)n->H * n->W * n->cout * sizeof(float), cudaMemcpyDeviceToDevice, s));
    return CTH_OK;
}

// gradients of <dout, forward output> after cth_unet_forward (zeroed first)
int cth_unet_backward(cth_unet* n, const float* dout, void* stream) {
    if (!n || !dout) { set_error("cth_unet_backward: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    cudaStream_t s = (cudaStream_t)stream;
    CTH_CUDA(cudaMemsetAsync(n->grad, 0, n->nparam * sizeof(float), s));
    return backward(n, dout, s);
}

// one Adam step on the weighted masked MSE between the output and target
// (device FP32 NHWC, mask one value per pixel, msum = sum of the mask);
// step t >= 1 (bias correction); loss (host) receives the loss before the step
int cth_unet_train_step(cth_unet* n, const float* in, const float* target, const float* mask, double msum, float lr,
                        int t, void* stream, double* loss) {
    if (!n || !in || !target || !mask || !(msum > 0.0) || t < 1) {
        set_error("cth_unet_train_step: invalid arguments");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(n->device));
    cudaStream_t s = (cudaStream_t)stream;
    int rc = forward(n, in, s);
    if (rc != CTH_OK) return rc;
    const size_t npx = (size_t)n->H * n->W;
    CTH_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(double), s));
    k_mse<<<grid1(npx), 256, 0, s>>>(n->out, target, mask, (int)npx, n->cout, n->cw, 1.0 / msum, n->dout, n->loss);
    CTH_CUDA(cudaMemsetAsync(n->grad, 0, n->nparam * sizeof(float), s));
    rc = backward(n, n->dout, s);
    if (rc != CTH_OK) return rc;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)t)), c2 = 1.f / (1.f - std::pow(b2, (float)t));
    k_adam<<<grid1(n->nparam), 256, 0, s>>>(n->prm, n->grad, n->adam_m, n->adam_v, n->nparam, lr, b1, b2, 1e-8f, c1,
                                            c2);
    rc = sync_weights(n, s);
    if (rc != CTH_OK) return rc;
    if (loss) {
        CTH_CUDA(cudaMemcpyAsync(loss, n->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CTH_CUDA(cudaStreamSynchronize(s));
    }
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

// 2 cin + 2 cout values: input mean[cin], input std[cin], output mean[cout], output std[cout]
int cth_unet_set_stats(cth_unet* n, const float* stats) {
    if (!n || !stats) { set_error("cth_unet_set_stats: invalid arguments"); return CTH_ERR_ARG; }
    const int ci = n->cin, co = n->cout;
    for (int k = 0; k < ci; k++) {
        n->stats.in_mean[k] = stats[k];
        n->stats.in_std[k] = stats[ci + k] > 0.f ? stats[ci + k] : 1.f;
    }
    for (int k = 0; k < co; k++) {
        n->stats.out_mean[k] = stats[2 * ci + k];
        n->stats.out_std[k] = stats[2 * ci + co + k] > 0.f ? stats[2 * ci + co + k] : 1.f;
    }
    return CTH_OK;
}

// the network's input (H x W x 6, FP32, device) from a field store whose grid is
// at most H x W cells
int cth_unet_features(cth_unet* n, cth_fields* fs, float* out, void* stream) {
    if (!n || !fs || !out || n->cin != 6 || fs->g->ni > n->W || fs->g->nj > n->H) {
        set_error("cth_unet_features: invalid arguments (6 input channels, grid within the image)");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(n->device));
    const char* names[6] = {"rhoe", "nu_m", "Bx", "Br", "dphi_prev2", "dphi_prev"};
    const double* q[6];
    for (int k = 0; k < 6; k++) {
        q[k] = field_ptr(fs, names[k]);
        if (!q[k]) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npx = (size_t)n->H * n->W;
    k_features<<<grid1(npx), 256, 0, s>>>(q[0], q[1], q[2], q[3], q[4], q[5], fs->g->ni, fs->g->nj, fs->g->ld,
                                          n->H, n->W, n->stats, out);
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

// warm-start prediction: features -> network; "dphi_guess" = "dphi_prev" +
// output channel 2 (the initial guess of cth_solve_phi_pc with warm_start = 1)
int cth_unet_predict_dphi(cth_unet* n, cth_fields* fs, void* stream) {
    if (!n || !fs || n->cout < 3) { set_error("cth_unet_predict_dphi: invalid arguments"); return CTH_ERR_ARG; }
    CTH_CUDA(cudaSetDevice(n->device));
    const size_t npx = (size_t)n->H * n->W;
    if (!n->feat) CTH_CUDA(cudaMalloc(&n->feat, npx * 6 * sizeof(float)));
    int rc = cth_unet_features(n, fs, n->feat, stream);
    if (rc != CTH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = forward(n, n->feat, s);
    if (rc != CTH_OK) return rc;
    double* dst = field_ptr(fs, "dphi_guess");
    const double* prev = field_ptr(fs, "dphi_prev");
    if (!dst || !prev) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    const int ncell = fs->g->ni * fs->g->nj;
    const float* o = n->out;
    if (n->smooth_passes > 0) {
        if (!n->smooth) CTH_CUDA(cudaMalloc(&n->smooth, npx * n->cout * sizeof(float)));
        float* buf[2] = {n->out, n->smooth};
        for (int k = 0; k < n->smooth_passes; k++) {
            k_smooth5<<<grid1((size_t)ncell), 256, 0, s>>>(buf[k & 1], buf[(k + 1) & 1], n->cout, 2, fs->g->nj,
                                                           fs->g->ni, n->W);
        }
        o = buf[n->smooth_passes & 1];
        n->launches += n->smooth_passes;
    }
    k_unpack<<<grid1((size_t)ncell), 256, 0, s>>>(o, n->cout, 2, fs->g->ni, fs->g->nj, fs->g->ld, n->W,
                                                   n->stats.out_mean[2], n->stats.out_std[2], prev, dst);
    n->launches += 2;  // features, unpack
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

// the microwave network (9 input, 6 output channels): features from the store and
// the previous fields E3 (three interleaved complex planes of the store's layout)
int cth_unet_mw_features(cth_unet* n, cth_fields* fs, const double* E3, double escale, float* out, void* stream) {
    if (!n || !fs || !E3 || !out || n->cin != 9 || fs->g->ni > n->W || fs->g->nj > n->H) {
        set_error("cth_unet_mw_features: invalid arguments (9 input channels, grid within the image)");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(n->device));
    const char* names[4] = {"rhoe", "nu_m1", "Bx", "Br"};
    const double* q[4];
    for (int k = 0; k < 4; k++) {
        q[k] = field_ptr(fs, names[k]);
        if (!q[k]) { set_error("field allocation failed"); return CTH_ERR_ALLOC; }
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npx = (size_t)n->H * n->W;
    const size_t pl = (size_t)(fs->g->nj + 2) * fs->g->ld;
    k_mw_features<<<grid1(npx), 256, 0, s>>>(q[0], q[1], q[2], q[3], E3, escale, pl, fs->g->ni, fs->g->nj,
                                             fs->g->ld, n->H, n->W, n->stats, out);
    n->launches++;
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

// the microwave guess: features -> network -> Eguess = Eprev + predicted change
// (Eguess may not alias Eprev)
int cth_unet_mw_guess(cth_unet* n, cth_fields* fs, const double* Eprev, double jprev, double jnow, double* Eguess,
                      void* stream) {
    if (!n || !fs || !Eprev || !Eguess || Eprev == Eguess || n->cin != 9 || n->cout != 6 || !(jprev != 0.0) ||
        !std::isfinite(jprev) || !std::isfinite(jnow)) {
        set_error("cth_unet_mw_guess: invalid arguments (9 input, 6 output channels; distinct planes; finite, "
                  "nonzero excitations)");
        return CTH_ERR_ARG;
    }
    CTH_CUDA(cudaSetDevice(n->device));
    const size_t npx = (size_t)n->H * n->W;
    if (!n->feat_mw) CTH_CUDA(cudaMalloc(&n->feat_mw, npx * 9 * sizeof(float)));
    int rc = cth_unet_mw_features(n, fs, Eprev, 1.0 / jprev, n->feat_mw, stream);
    if (rc != CTH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = forward(n, n->feat_mw, s);
    if (rc != CTH_OK) return rc;
    const size_t pl = (size_t)(fs->g->nj + 2) * fs->g->ld;
    k_mw_unpack<<<grid1(3 * pl), 256, 0, s>>>(n->out, n->W, n->stats, Eprev, jnow / jprev, jnow, Eguess, pl,
                                              fs->g->ni, fs->g->nj, fs->g->ld);
    n->launches++;
    CTH_CUDA(cudaGetLastError());
    return CTH_OK;
}

}  // extern "C"
