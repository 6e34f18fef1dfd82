// unet.cu -- kernels of the learned warm start: a small convolutional U-Net in BF16 with
// FP32 accumulation (forward, data gradient, weight gradient) and its optimiser.
//
// Activations are NHWC bf16 tensors addressed through channel views (pixel stride
// `cs`, channel offset `co`), so a decoder's concatenated input is one buffer that the
// encoder writes into and the upsampler fills.  Convolutions are 3x3, "same" padding.
//
// conv3x3_fwd: implicit GEMM, M = pixels, N = output channels, K = 9 taps x Cin, on the
// BF16 tensor cores (mma.sync m16n8k16, FP32 accumulators), operands staged in shared
// memory by cp.async (zero-filled outside the image) and fed by ldmatrix.  A block
// computes 64 pixels x 64 channels with 4 warps of 32 x 32; K advances one
// (tap, 16-channel) slice per stage, double-buffered.  The data gradient is the same
// kernel on the flipped, transposed weights.
// conv3x3_wgrad: dW[co][tap][ci] = sum_p dY[p][co] X[p + tap][ci], M = co, N = (tap, ci),
// K = pixels, split over blocks and accumulated in FP32 with atomics.
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdlib>

#include "mm_internal.h"

namespace mm {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void ldm_x4(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldm_x4_t(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------- forward / data gradient
// out[p][co] = act(bias[co] + sum_{tap, ci} W[co][tap][ci] in[p + tap][ci])
// Cin % 16 == 0; W rows hold Cout_w >= Cout rows (extra rows ignored); accumulate: add to out.
#define FWD_BM 64
#define FWD_BN 64
#define FWD_PITCH 24  // bf16 per smem row (16 + 8: ldmatrix rows on distinct banks)

__global__ void __launch_bounds__(128) conv3x3_fwd_kernel(const bf16* __restrict__ in, int in_cs, int in_co, int Cin,
                                                          const bf16* __restrict__ W, const float* __restrict__ bias,
                                                          bf16* __restrict__ out, int out_cs, int out_co, int Cout,
                                                          int B, int H, int Wd, int relu) {
    __shared__ __align__(128) bf16 sA[2][FWD_BM * FWD_PITCH];
    __shared__ __align__(128) bf16 sB[2][FWD_BN * FWD_PITCH];
    const long long P = (long long)B * H * Wd;
    const long long p0 = (long long)blockIdx.x * FWD_BM;
    const int n0 = blockIdx.y * FWD_BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    // loader roles: row r (pixel or output channel), 16-byte half h
    const int lr = tid >> 1, lh = tid & 1;
    const long long pr = p0 + lr;
    int py = 0, px = 0, pb = 0;
    if (pr < P) {
        px = (int)(pr % Wd);
        const long long t = pr / Wd;
        py = (int)(t % H);
        pb = (int)(t / H);
    }
    const int nslices = Cin / 16;
    const int nk = 9 * nslices;
    auto load = [&](int stage, int kk) {
        const int tap = kk / nslices, cs = (kk % nslices) * 16;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        const int yy = py + dy, xx = px + dx;
        const bool ok = pr < P && yy >= 0 && yy < H && xx >= 0 && xx < Wd;
        const long long q = ok ? ((long long)pb * H + yy) * Wd + xx : 0;
        cp_async16(&sA[stage][lr * FWD_PITCH + lh * 8], in + q * in_cs + in_co + cs + lh * 8, ok);
        const int co = n0 + lr;
        const bool okb = co < Cout;
        cp_async16(&sB[stage][lr * FWD_PITCH + lh * 8],
                   W + ((long long)(okb ? co : 0) * 9 + tap) * Cin + cs + lh * 8, okb);
    };
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
    load(0, 0);
    cp_commit();
    for (int kk = 0; kk < nk; kk++) {
        const int st = kk & 1;
        if (kk + 1 < nk) load(st ^ 1, kk + 1);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        unsigned a[2][4], b[2][4];
#pragma unroll
        for (int i = 0; i < 2; i++)
            ldm_x4(a[i], &sA[st][(wm + i * 16 + (lane & 15)) * FWD_PITCH + (lane >> 4) * 8]);
#pragma unroll
        for (int j = 0; j < 2; j++)
            ldm_x4(b[j], &sB[st][(wn + j * 16 + (lane & 7) + ((lane >> 4) << 3)) * FWD_PITCH + ((lane >> 3) & 1) * 8]);
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i], b[j >> 1][(j & 1) * 2], b[j >> 1][(j & 1) * 2 + 1]);
        __syncthreads();
    }
    // epilogue
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int hr = 0; hr < 2; hr++) {
            const long long p = p0 + wm + i * 16 + g + hr * 8;
            if (p >= P) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int co = n0 + wn + j * 8 + t4 * 2;
                if (co >= Cout) continue;
                float v0 = acc[i][j][hr * 2], v1 = acc[i][j][hr * 2 + 1];
                if (bias) {
                    v0 += bias[co];
                    if (co + 1 < Cout) v1 += bias[co + 1];
                }
                if (relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                bf16* o = out + p * out_cs + out_co + co;
                if (co + 1 < Cout) {
                    *reinterpret_cast<__nv_bfloat162*>(o) = __floats2bfloat162_rn(v0, v1);
                } else {
                    o[0] = __float2bfloat16_rn(v0);
                }
            }
        }
}

// ---------------------------------------------------------------- weight gradient
// dW[co][tap][ci] += sum_{p in this block's pixels} dY[p][co] X[p + tap][ci]  (FP32)
#define WG_BM 64   // output channels
#define WG_BN 64   // (tap, ci) columns
#define WG_BK 32   // pixels per stage
#define WG_PA 72   // bf16 per smem row of A (64 + 8)
#define WG_PB 72

__global__ void __launch_bounds__(128) conv3x3_wgrad_kernel(const bf16* __restrict__ dy, int dy_cs, int dy_co, int Cout,
                                                            const bf16* __restrict__ x, int x_cs, int x_co, int Cin,
                                                            float* __restrict__ dW, int B, int H, int Wd,
                                                            int pix_per_block) {
    __shared__ __align__(128) bf16 sA[2][WG_BK * WG_PA];  // [pixel][co]
    __shared__ __align__(128) bf16 sB[2][WG_BK * WG_PB];  // [pixel][(tap, ci)]
    const int P = B * H * Wd;
    const int m0 = blockIdx.x * WG_BM;
    const int n0 = blockIdx.y * WG_BN;
    const int Ncols = 9 * Cin;
    const int pstart = blockIdx.z * pix_per_block;
    const int pend = pstart + pix_per_block < P ? pstart + pix_per_block : P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    auto load = [&](int stage, int pk) {
        // A: 32 pixels x 64 channels = 256 chunks of 8 channels; 2 per thread
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int c = tid + r * 128;
            const int row = c >> 3, ch = (c & 7) * 8;
            const int p = pk + row;
            const bool ok = p < pend && m0 + ch < Cout;
            cp_async16(&sA[stage][row * WG_PA + ch], dy + (long long)(ok ? p : 0) * dy_cs + dy_co + (ok ? m0 + ch : 0),
                       ok);
        }
        // B: 32 pixels x 64 (tap, ci) columns, 8 columns (one tap, 8 channels) per chunk
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int c = tid + r * 128;
            const int row = c >> 3, col = (c & 7) * 8;
            const int p = pk + row;
            const int n = n0 + col;
            bool ok = p < pend && n < Ncols;
            int q = 0, ci = 0;
            if (ok) {   // 32-bit index arithmetic (the host checks that the pixels fit)
                const int tap = n / Cin;
                ci = n - tap * Cin;
                const int tt = p / Wd, xx0 = p - tt * Wd;
                const int bb = tt / H, yy0 = tt - bb * H;
                const int yy = yy0 + tap / 3 - 1, xx = xx0 + tap % 3 - 1;
                ok = yy >= 0 && yy < H && xx >= 0 && xx < Wd;
                q = (bb * H + yy) * Wd + xx;
            }
            cp_async16(&sB[stage][row * WG_PB + col], x + (long long)(ok ? q : 0) * x_cs + x_co + (ok ? ci : 0), ok);
        }
    };
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
    const int nk = (pend - pstart + WG_BK - 1) / WG_BK;
    if (nk <= 0) return;
    load(0, pstart);
    cp_commit();
    for (int kk = 0; kk < nk; kk++) {
        const int st = (int)(kk & 1);
        if (kk + 1 < nk) load(st ^ 1, pstart + (kk + 1) * WG_BK);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < WG_BK; ks += 16) {
            unsigned a[2][4], b[2][4];
#pragma unroll
            for (int i = 0; i < 2; i++)
                ldm_x4_t(a[i], &sA[st][(ks + (lane & 7) + ((lane >> 4) << 3)) * WG_PA + wm + i * 16 +
                                       ((lane >> 3) & 1) * 8]);
#pragma unroll
            for (int j = 0; j < 2; j++)
                ldm_x4_t(b[j], &sB[st][(ks + (lane & 7) + (((lane >> 3) & 1) << 3)) * WG_PB + wn + j * 16 +
                                       (lane >> 4) * 8]);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    mma_bf16(acc[i][j], a[i], b[j >> 1][(j & 1) * 2], b[j >> 1][(j & 1) * 2 + 1]);
        }
        __syncthreads();
    }
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int hr = 0; hr < 2; hr++) {
            const int co = m0 + wm + i * 16 + g + hr * 8;
            if (co >= Cout) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int n = n0 + wn + j * 8 + t4 * 2;
                if (n < Ncols) atomicAdd(dW + (long long)co * Ncols + n, acc[i][j][hr * 2]);
                if (n + 1 < Ncols) atomicAdd(dW + (long long)co * Ncols + n + 1, acc[i][j][hr * 2 + 1]);
            }
        }
}

// ---------------------------------------------------------------- elementwise pieces
// 2x2 average pool: out (H/2 x W/2) <- in (H x W), channel views
// 2x2 average pooling, nearest upsampling and their gradients on NHWC views, 8 channels
// (16 bytes) per thread; the sums run in the same order as per channel.
__device__ __forceinline__ void ld8(const bf16* p, float v[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 f = __bfloat1622float2(h[k]);
        v[2 * k] = f.x;
        v[2 * k + 1] = f.y;
    }
}
__device__ __forceinline__ void st8(bf16* p, const float v[8]) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; k++) h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

__global__ void pool_fwd_kernel(const bf16* in, int in_cs, int in_co, bf16* out, int out_cs, int out_co, int C, int B,
                                int Ho, int Wo) {
    const int G = C >> 3;
    const long long n = (long long)B * Ho * Wo * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const long long p = e / G;
        const int x = (int)(p % Wo);
        const long long t = p / Wo;
        const int y = (int)(t % Ho), b = (int)(t / Ho);
        const int Wi = 2 * Wo, Hi = 2 * Ho;
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, v[8];
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                ld8(in + (((long long)b * Hi + 2 * y + i) * Wi + 2 * x + j) * in_cs + in_co + 8 * g, v);
#pragma unroll
                for (int k = 0; k < 8; k++) s[k] += v[k];
            }
#pragma unroll
        for (int k = 0; k < 8; k++) s[k] *= 0.25f;
        st8(out + p * out_cs + out_co + 8 * g, s);
    }
}
__global__ void pool_bwd_kernel(const bf16* dout, int do_cs, int do_co, bf16* din, int di_cs, int di_co, int C, int B,
                                int Ho, int Wo) {
    const int G = C >> 3;
    const long long n = (long long)B * (2 * Ho) * (2 * Wo) * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const long long p = e / G;
        const int Wi = 2 * Wo, Hi = 2 * Ho;
        const int x = (int)(p % Wi);
        const long long t = p / Wi;
        const int y = (int)(t % Hi), b = (int)(t / Hi);
        float gv[8], dv[8];
        ld8(dout + (((long long)b * Ho + y / 2) * Wo + x / 2) * do_cs + do_co + 8 * g, gv);
        bf16* d = din + p * di_cs + di_co + 8 * g;
        ld8(d, dv);
#pragma unroll
        for (int k = 0; k < 8; k++) dv[k] = dv[k] + 0.25f * gv[k];
        st8(d, dv);
    }
}
__global__ void up_fwd_kernel(const bf16* in, int in_cs, int in_co, bf16* out, int out_cs, int out_co, int C, int B,
                              int Hi, int Wi) {
    const int G = C >> 3;
    const long long n = (long long)B * (2 * Hi) * (2 * Wi) * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const long long p = e / G;
        const int Wo = 2 * Wi, Ho = 2 * Hi;
        const int x = (int)(p % Wo);
        const long long t = p / Wo;
        const int y = (int)(t % Ho), b = (int)(t / Ho);
        *reinterpret_cast<uint4*>(out + p * out_cs + out_co + 8 * g) =
            *reinterpret_cast<const uint4*>(in + (((long long)b * Hi + y / 2) * Wi + x / 2) * in_cs + in_co + 8 * g);
    }
}
__global__ void up_bwd_kernel(const bf16* dout, int do_cs, int do_co, bf16* din, int di_cs, int di_co, int C, int B,
                              int Hi, int Wi) {
    const int G = C >> 3;
    const long long n = (long long)B * Hi * Wi * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(e % G);
        const long long p = e / G;
        const int x = (int)(p % Wi);
        const long long t = p / Wi;
        const int y = (int)(t % Hi), b = (int)(t / Hi);
        const int Wo = 2 * Wi, Ho = 2 * Hi;
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, v[8];
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                ld8(dout + (((long long)b * Ho + 2 * y + i) * Wo + 2 * x + j) * do_cs + do_co + 8 * g, v);
#pragma unroll
                for (int k = 0; k < 8; k++) s[k] += v[k];
            }
        st8(din + p * di_cs + di_co + 8 * g, s);
    }
}
// dpre = dout * (out > 0) in place on the gradient view
__global__ void relu_bwd_kernel(const bf16* out, int o_cs, int o_co, bf16* d, int d_cs, int d_co, int C, long long P) {
    const long long n = P * C;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const long long p = e / C;
        if (!(__bfloat162float(out[p * o_cs + o_co + c]) > 0.f)) d[p * d_cs + d_co + c] = __float2bfloat16_rn(0.f);
    }
}
// db[c] += sum_p d[p][c]
// ReLU backward and bias gradient in one pass: each thread takes 8 consecutive channels
// of a pixel (16-byte loads; consecutive threads cover consecutive channels, then the
// next pixels), zeroes the gradient where the forward output was not positive (relu),
// keeps 8 register sums for its channels, and the block adds its per-channel sums to db.
__global__ void relu_bias_bwd_kernel(const bf16* __restrict__ out, int o_cs, int o_co, bf16* __restrict__ d, int d_cs,
                                     int d_co, int C, long long P, long long ppb, int relu, float* __restrict__ db) {
    __shared__ float acc[512];
    const int G = C / 8;                       // threads per pixel
    const int K = blockDim.x / G;              // pixels per block iteration
    const int g = threadIdx.x % G, r = threadIdx.x / G;
    for (int i = threadIdx.x; i < C; i += blockDim.x) acc[i] = 0.f;
    __syncthreads();
    const long long p0 = blockIdx.x * ppb, p1 = min(P, p0 + ppb);
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (r < K) {
        for (long long p = p0 + r; p < p1; p += K) {
            uint4* gp = reinterpret_cast<uint4*>(d + p * d_cs + d_co + 8 * g);
            uint4 gv = *gp;
            __nv_bfloat162* gh = reinterpret_cast<__nv_bfloat162*>(&gv);
            if (relu) {
                const uint4 ov = *reinterpret_cast<const uint4*>(out + p * o_cs + o_co + 8 * g);
                const __nv_bfloat162* oh = reinterpret_cast<const __nv_bfloat162*>(&ov);
                bool changed = false;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float2 of = __bfloat1622float2(oh[k]);
                    float2 gf = __bfloat1622float2(gh[k]);
                    if (!(of.x > 0.f)) { gf.x = 0.f; changed = true; }
                    if (!(of.y > 0.f)) { gf.y = 0.f; changed = true; }
                    gh[k] = __floats2bfloat162_rn(gf.x, gf.y);
                }
                if (changed) *gp = gv;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float2 gf = __bfloat1622float2(gh[k]);
                s[2 * k] += gf.x;
                s[2 * k + 1] += gf.y;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) atomicAdd(&acc[8 * g + k], s[k]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x) atomicAdd(db + i, acc[i]);
}

__global__ void bias_grad_kernel(const bf16* d, int d_cs, int d_co, int C, long long P, float* db) {
    const int c = blockIdx.y;
    float s = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        s += __bfloat162float(d[p * d_cs + d_co + c]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        atomicAdd(db + c, t);
    }
}
// masked mean-square error of the first 3 channels against a float target [P][3]:
// loss += sum mask |out - target|^2 / norm ; dout = 2 mask (out - target) / norm
__global__ void mse_kernel(const bf16* out, int o_cs, const float* target, const float* mask, long long P, float norm,
                           bf16* dout, int d_cs, float* loss) {
    float s = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        const float w = mask[p];
        for (int c = 0; c < 3; c++) {
            const float diff = __bfloat162float(out[p * o_cs + c]) - target[p * 3 + c];
            s += w * diff * diff;
            dout[p * d_cs + c] = __float2bfloat16_rn(2.f * w * diff / norm);
        }
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        atomicAdd(loss, t / norm);
    }
}
// Adam (Kingma & Ba) on FP32 master weights; refreshes the bf16 copy
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2, bf16* wb) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}
// Wt[ci][tap'][co] = W[co][8 - tap'][ci] for the data gradient (rows padded to Cin_t >= Cout,
// columns Coutp >= Cin)
__global__ void flip_kernel(const bf16* W, int Cout, int Cin, bf16* Wt, int Cin_t, int Cout_t) {
    const long long n = (long long)Cout_t * 9 * Cin_t;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(e % Cin_t);          // column: the original output channel
        const long long r = e / Cin_t;
        const int tap = (int)(r % 9), ci = (int)(r / 9);
        bf16 v = __float2bfloat16_rn(0.f);
        if (co < Cout && ci < Cin) v = W[((long long)co * 9 + (8 - tap)) * Cin + ci];
        Wt[e] = v;
    }
}
// float -> bf16 into a channel view; in [P][C] float
__global__ void to_bf16_kernel(const float* in, long long P, int C, bf16* out, int o_cs, int o_co) {
    const long long n = P * C;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const long long p = e / C;
        out[p * o_cs + o_co + c] = __float2bfloat16_rn(in[e]);
    }
}

// ---------------------------------------------------------------- C-ABI (host launchers)
static int grid1(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace mm

using namespace mm;

#define NN_CHECK()                                                                              \
    do {                                                                                        \
        cudaError_t e_ = cudaGetLastError();                                                    \
        if (e_ != cudaSuccess) return report_error(MM_ERR_CUDA, cudaGetErrorString(e_));        \
    } while (0)

extern "C" MM_API int mm_nn_conv3x3(const void* in, int in_cs, int in_co, int Cin, const void* W, const float* bias,
                                    void* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu,
                                    mm_stream st) {
    if (Cin % 16 || in_cs % 8 || in_co % 8 || Cout < 1 || B < 1 || H < 1 || Wd < 1 || (out_co & 1) || (out_cs & 1))
        return report_error(MM_ERR_ARG, "mm_nn_conv3x3: Cin, channel stride and offset must be multiples of 16/8/8");
    const long long P = (long long)B * H * Wd;
    dim3 grid((unsigned)((P + FWD_BM - 1) / FWD_BM), (unsigned)((Cout + FWD_BN - 1) / FWD_BN));
    conv3x3_fwd_kernel<<<grid, 128, 0, (cudaStream_t)st>>>((const bf16*)in, in_cs, in_co, Cin, (const bf16*)W, bias,
                                                           (bf16*)out, out_cs, out_co, Cout, B, H, Wd, relu);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_conv3x3_wgrad(const void* dy, int dy_cs, int dy_co, int Cout, const void* x, int x_cs,
                                          int x_co, int Cin, float* dW, int B, int H, int Wd, mm_stream st) {
    if (Cin % 8 || Cout % 8 || dy_cs % 8 || dy_co % 8 || x_cs % 8 || x_co % 8)
        return report_error(MM_ERR_ARG, "mm_nn_conv3x3_wgrad: channel counts, strides and offsets must be multiples of 8");
    if ((long long)B * H * Wd >= (1LL << 30)) return report_error(MM_ERR_ARG, "mm_nn_conv3x3_wgrad: too many pixels");
    const long long P = (long long)B * H * Wd;
    const int mt = (Cout + WG_BM - 1) / WG_BM, nt = (9 * Cin + WG_BN - 1) / WG_BN;
    // split the pixels so that about 4 waves of blocks cover the GPU
    long long splits = (148LL * 4 * 4 + mt * nt - 1) / (mt * nt);
    long long ppb = (P + splits - 1) / splits;
    ppb = ((ppb + WG_BK - 1) / WG_BK) * WG_BK;
    if (ppb < 4 * WG_BK) ppb = 4 * WG_BK;
    splits = (P + ppb - 1) / ppb;
    dim3 grid((unsigned)mt, (unsigned)nt, (unsigned)splits);
    conv3x3_wgrad_kernel<<<grid, 128, 0, (cudaStream_t)st>>>((const bf16*)dy, dy_cs, dy_co, Cout, (const bf16*)x, x_cs,
                                                             x_co, Cin, dW, B, H, Wd, (int)ppb);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_pool(const void* in, int in_cs, int in_co, void* out, int out_cs, int out_co, int C, int B,
                                 int Ho, int Wo, int backward, mm_stream st) {
    if (C % 8 || in_cs % 8 || in_co % 8 || out_cs % 8 || out_co % 8)
        return report_error(MM_ERR_ARG, "mm_nn_pool: channel counts, strides and offsets must be multiples of 8");
    const long long n = (long long)B * Ho * Wo * (C / 8) * (backward ? 4 : 1);
    if (backward)
        pool_bwd_kernel<<<grid1(n), 256, 0, (cudaStream_t)st>>>((const bf16*)in, in_cs, in_co, (bf16*)out, out_cs,
                                                                 out_co, C, B, Ho, Wo);
    else
        pool_fwd_kernel<<<grid1(n), 256, 0, (cudaStream_t)st>>>((const bf16*)in, in_cs, in_co, (bf16*)out, out_cs,
                                                                 out_co, C, B, Ho, Wo);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_upsample(const void* in, int in_cs, int in_co, void* out, int out_cs, int out_co, int C,
                                     int B, int Hi, int Wi, int backward, mm_stream st) {
    if (C % 8 || in_cs % 8 || in_co % 8 || out_cs % 8 || out_co % 8)
        return report_error(MM_ERR_ARG, "mm_nn_upsample: channel counts, strides and offsets must be multiples of 8");
    const long long n = (long long)B * Hi * Wi * (C / 8) * (backward ? 1 : 4);
    if (backward)
        up_bwd_kernel<<<grid1(n), 256, 0, (cudaStream_t)st>>>((const bf16*)in, in_cs, in_co, (bf16*)out, out_cs, out_co,
                                                               C, B, Hi, Wi);
    else
        up_fwd_kernel<<<grid1(n), 256, 0, (cudaStream_t)st>>>((const bf16*)in, in_cs, in_co, (bf16*)out, out_cs, out_co,
                                                               C, B, Hi, Wi);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_relu_bwd(const void* out, int o_cs, int o_co, void* d, int d_cs, int d_co, int C,
                                     long long P, mm_stream st) {
    relu_bwd_kernel<<<grid1(P * C), 256, 0, (cudaStream_t)st>>>((const bf16*)out, o_cs, o_co, (bf16*)d, d_cs, d_co, C, P);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_relu_bias_bwd(const void* out, int o_cs, int o_co, void* d, int d_cs, int d_co, int C,
                                          long long P, int relu, float* db, mm_stream st) {
    if (C < 8 || C > 512 || C % 8 || o_cs % 8 || o_co % 8 || d_cs % 8 || d_co % 8 || P < 0)
        return report_error(MM_ERR_ARG, "mm_nn_relu_bias_bwd: C in 8..512, channel counts, strides and offsets multiples of 8");
    const int G = C / 8;
    const int K = G >= 256 ? 1 : 256 / G;
    const long long blocks = 148LL * 4;
    long long ppb = (P + blocks - 1) / blocks;
    if (ppb < K) ppb = K;
    const long long nb = (P + ppb - 1) / ppb;
    if (nb > 0)
        relu_bias_bwd_kernel<<<(unsigned)nb, G * K, 0, (cudaStream_t)st>>>((const bf16*)out, o_cs, o_co, (bf16*)d, d_cs,
                                                                           d_co, C, P, ppb, relu, db);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_bias_grad(const void* d, int d_cs, int d_co, int C, long long P, float* db, mm_stream st) {
    long long b = (P + 255) / 256;
    if (b > 64) b = 64;
    bias_grad_kernel<<<dim3((unsigned)b, (unsigned)C), 256, 0, (cudaStream_t)st>>>((const bf16*)d, d_cs, d_co, C, P, db);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_mse(const void* out, int o_cs, const float* target, const float* mask, long long P,
                                float norm, void* dout, int d_cs, float* loss, mm_stream st) {
    mse_kernel<<<grid1(P), 256, 0, (cudaStream_t)st>>>((const bf16*)out, o_cs, target, mask, P, norm, (bf16*)dout, d_cs,
                                                       loss);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1,
                                 float b2, float eps, int t, void* wb, mm_stream st) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    adam_kernel<<<grid1(n), 256, 0, (cudaStream_t)st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, (bf16*)wb);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_flip(const void* W, int Cout, int Cin, void* Wt, int Cin_t, int Cout_t, mm_stream st) {
    flip_kernel<<<grid1((long long)Cout_t * 9 * Cin_t), 256, 0, (cudaStream_t)st>>>((const bf16*)W, Cout, Cin, (bf16*)Wt,
                                                                                      Cin_t, Cout_t);
    NN_CHECK();
    return MM_OK;
}

extern "C" MM_API int mm_nn_to_bf16(const float* in, long long P, int C, void* out, int o_cs, int o_co, mm_stream st) {
    to_bf16_kernel<<<grid1(P * C), 256, 0, (cudaStream_t)st>>>(in, P, C, (bf16*)out, o_cs, o_co);
    NN_CHECK();
    return MM_OK;
}

// ---------------------------------------------------------------- tcgen05 forward convolution
// The same implicit GEMM on the 5th-generation tensor cores: D[128 positions][N] in TMEM
// (FP32), A = positions x (tap, channel) and B = output channels x (tap, channel), both
// K-major bf16 in shared memory in the canonical no-swizzle layout (8-row x 16-byte core
// matrices).  One thread issues the nine tcgen05.mma (M 128, N, K 16) of a 16-channel
// slice; stages form a ring of 2-4 buffers filled by cp.async and released by a
// tcgen05.commit to the stage's mbarrier, so several slices load while the tensor core
// works.  Waits are bounded: a wait that runs out sets *err and the block frees its TMEM
// and returns.
namespace mm {

// Epilogue store of one pixel's 16 consecutive output channels c0 .. c0+15 (FP32 from
// TMEM): bias, ReLU, bf16.  With vec (the row start 16-byte aligned and all 16 channels
// present) two 16-byte stores, else bf16 pairs and a last single channel.
__device__ __forceinline__ void store16(const unsigned (&v)[16], bf16* row, int c0, int Cout,
                                        const float* __restrict__ bias, int relu, bool vec) {
    float f[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
        float a = __uint_as_float(v[e]);
        if (bias && c0 + e < Cout) a += bias[c0 + e];
        if (relu) a = fmaxf(a, 0.f);
        f[e] = a;
    }
    if (vec && c0 + 16 <= Cout) {
        unsigned w[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
            w[e] = *reinterpret_cast<unsigned*>(&h);
        }
        uint4* o = reinterpret_cast<uint4*>(row + c0);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
        return;
    }
#pragma unroll
    for (int e = 0; e < 16; e += 2) {
        const int co = c0 + e;
        if (co >= Cout) break;
        bf16* o = row + co;
        if (co + 1 < Cout) *reinterpret_cast<__nv_bfloat162*>(o) = __floats2bfloat162_rn(f[e], f[e + 1]);
        else o[0] = __float2bfloat16_rn(f[e]);
    }
}

// Iteration limit of the mbarrier waits of the tcgen05 kernels (mm_nn_set_wait_limit
// changes it, e.g. to 0 so that a test sees the time-out path; the clean-up wait for
// MMAs in flight always uses the default).
constexpr long long kWaitLimitDefault = 1LL << 26;
static long long g_wait_limit = kWaitLimitDefault;

__device__ __forceinline__ uint64_t umma_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, no swizzle
}

__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity, long long limit) {
    for (long long i = 0; i < limit; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity));
        if (ok) return true;
    }
    return false;
}

// Halo-band layout.  The tile runs over padded positions: image b, row y, column x sit
// at q = b (H+1)(W+1) + y (W+1) + x + 1, so every row starts with a zero column and every
// image ends with a zero row.  An output at q reads its tap (dy, dx) at q + dy (W+1) + dx,
// which is a zero pad whenever the tap leaves the image.  The 128 outputs q0 .. q0+127
// of a tile therefore read, for every tap, 128 consecutive positions of one band
// q0 - (W+2) .. q0 + 127 + (W+2): the A operand of tap (dy, dx) is the band's descriptor
// shifted by ((dy+1)(W+1) + dx+1) x 16 bytes.  A stage holds one 16-channel slice of the
// band (two 8-channel planes, K-direction stride = plane size, 8-position groups 128
// bytes apart) and the slice's weights for all nine taps; it is read from global memory
// once instead of once per tap.  Pad positions are computed and not stored.
constexpr int BAND_MAX = 128 + 2 * 257 + 2;  // widths up to 256

template <int N, int ST>
__global__ void __launch_bounds__(256) conv3x3_tc_kernel(const bf16* __restrict__ in, int in_cs, int in_co, int Cin,
                                                         const bf16* __restrict__ W, const float* __restrict__ bias,
                                                         bf16* __restrict__ out, int out_cs, int out_co, int Cout,
                                                         int B, int H, int Wd, int relu, int* err, int band,
                                                         int stage_bytes, long long limit) {
    constexpr int M = 128;
    constexpr int TCOLS = N < 32 ? 32 : N;         // TMEM columns (power of two >= 32)
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long mbar[ST];
    __shared__ unsigned tmem_base_sh;
    __shared__ int fail_sh;
    __shared__ int s_q[BAND_MAX];                  // band position -> input pixel, or -1
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Wp = Wd + 1;
    const long long img = (long long)(H + 1) * Wp;
    const long long total = (long long)B * img;
    const long long q0 = (long long)blockIdx.x * M;
    const int n0 = blockIdx.y * N;
    const int plane = band * 16;                   // bytes of one 8-channel plane of the band
    const bool vec = (out_cs % 8 == 0) && (out_co % 8 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    for (int i = tid; i < band; i += 256) {
        const long long q = q0 - (Wp + 1) + i;
        int pix = -1;
        if (q >= 0 && q < total) {
            const long long b = q / img, r = q - b * img;
            const int y = (int)(r / Wp), xp = (int)(r - (long long)y * Wp);
            if (y < H && xp > 0) pix = (int)(((long long)b * H + y) * Wd + xp - 1);
        }
        s_q[i] = pix;
    }
    if (tid == 0) {
        fail_sh = 0;
        for (int i = 0; i < ST; i++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[i])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "n"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const unsigned tmem = tmem_base_sh;
    const int nstages = Cin / 16;
    const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
    const long long LIMIT = limit;
    // core-matrix offset of (row r, k-half h) in a 16-channel weight block: K-adjacent core
    // matrices 128 bytes apart, 8-row groups 256 bytes apart
    auto core_off = [](int r, int h) { return ((r >> 3) * 2 + h) * 128 + (r & 7) * 16; };
    const int bwt = 2 * plane;                     // weights follow the band in a stage
    auto load_stage = [&](int s) {
        unsigned char* base = smem + (s % ST) * stage_bytes;
        const int cs = s * 16;
        // band: consecutive lanes take consecutive positions of one plane
        for (int c = tid; c < 2 * band; c += 256) {
            const int h = c >= band ? 1 : 0, i = c - h * band;
            const int pix = s_q[i];
            const bool ok = pix >= 0;
            cp_async16(base + h * plane + i * 16, in + (long long)(ok ? pix : 0) * in_cs + in_co + cs + h * 8, ok);
        }
        // weights of the nine taps
        for (int c = tid; c < 9 * 2 * N; c += 256) {
            const int tap = c / (2 * N), rem = c - tap * 2 * N;
            const int rr = rem >> 1, h = rem & 1;
            const int co = n0 + rr;
            const bool okb = co < Cout;
            cp_async16(base + bwt + tap * N * 32 + core_off(rr, h),
                       W + ((long long)(okb ? co : 0) * 9 + tap) * Cin + cs + h * 8, okb);
        }
    };
    for (int s = 0; s < ST - 1; s++) {
        if (s < nstages) load_stage(s);
        cp_commit();
    }
    int issued = 0;  // stages whose MMAs were issued and committed
    for (int s = 0; s < nstages; s++) {
        cp_wait<ST - 2>();  // this thread's copies of stage s have landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
        __syncthreads();
        if (fail_sh) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const unsigned base = smem_u32(smem + (s % ST) * stage_bytes);
#pragma unroll 1
            for (int tap = 0; tap < 9; tap++) {
                const unsigned off = (unsigned)(((tap / 3) * Wp + tap % 3) * 16);
                const uint64_t ad = umma_desc(base + off, (unsigned)plane, 128);
                const uint64_t bd = umma_desc(base + bwt + tap * N * 32, 128, 256);
                const unsigned acc = (s > 0 || tap > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&mbar[s % ST])));
        }
        issued = s + 1;
        // refill the buffer of stage s-1 with stage s+ST-1 once the MMAs of s-1 are done
        const int nx = s + ST - 1;
        if (nx < nstages) {
            if (s >= 1 && !mbar_wait(smem_u32(&mbar[(s - 1) % ST]), ((s - 1) / ST) & 1, LIMIT)) {
                if (lane == 0) atomicExch(&fail_sh, 1);
            } else {
                load_stage(nx);
            }
        }
        cp_commit();
    }
    cp_wait<0>();
    __syncthreads();
    // the last commit covers every MMA of the block; a block that gave up waits (bounded,
    // with the default limit) for the MMAs it has in flight before its TMEM is freed
    if (issued > 0) {
        const int last = issued - 1;
        const bool ok = !fail_sh && mbar_wait(smem_u32(&mbar[last % ST]), (last / ST) & 1, LIMIT);
        if (!ok) {
            if (lane == 0) atomicExch(&fail_sh, 1);
            mbar_wait(smem_u32(&mbar[last % ST]), (last / ST) & 1, kWaitLimitDefault);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (tile rows) and the column
    // half w / 4 (N = 16: warps 0-3 take all columns); 16 columns per load
    constexpr int CW = N >= 32 ? N / 2 : N;
    const int quad = warp & 3, chalf = warp >> 2;
    if (!fail_sh && chalf * CW < N) {
        // this lane's output pixel (pad positions are not stored)
        const int pix = s_q[quad * 32 + lane + Wp + 1];
#pragma unroll
        for (int c0 = chalf * CW; c0 < chalf * CW + CW; c0 += 16) {
            unsigned v[16];
            const unsigned ta = tmem + ((unsigned)(quad * 32) << 16) + (unsigned)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];\n"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
            if (pix >= 0) store16(v, out + (long long)pix * out_cs + out_co, n0 + c0, Cout, bias, relu, vec);
        }
    } else if (fail_sh && tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(TCOLS));
    }
}

// Stages of the ring: as many (2..4) as fit in 110 KB, so that two blocks share an SM.
template <int N, int ST>
static cudaError_t launch_conv_tc_st(const bf16* in, int in_cs, int in_co, int Cin, const bf16* W, const float* bias,
                                     bf16* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu,
                                     int* err, cudaStream_t st, int band, int stage_bytes) {
    const int smem = ST * stage_bytes;
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<N, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long positions = (long long)B * (H + 1) * (Wd + 1);
    dim3 grid((unsigned)((positions + 127) / 128), (unsigned)((Cout + N - 1) / N));
    conv3x3_tc_kernel<N, ST><<<grid, 256, smem, st>>>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H,
                                                      Wd, relu, err, band, stage_bytes, g_wait_limit);
    return cudaGetLastError();
}

template <int N>
static cudaError_t launch_conv_tc(const bf16* in, int in_cs, int in_co, int Cin, const bf16* W, const float* bias,
                                  bf16* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu, int* err,
                                  cudaStream_t st) {
    const int band = 128 + 2 * (Wd + 1) + 2;
    const int stage_bytes = ((2 * band * 16 + 9 * N * 32) + 127) / 128 * 128;
    const int fit = (110 * 1024) / stage_bytes;
    if (fit >= 4)
        return launch_conv_tc_st<N, 4>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu, err,
                                       st, band, stage_bytes);
    if (fit == 3)
        return launch_conv_tc_st<N, 3>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu, err,
                                       st, band, stage_bytes);
    return launch_conv_tc_st<N, 2>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu, err, st,
                                   band, stage_bytes);
}

// ---------------------------------------------------------------- tcgen05 convolution, persistent
// The same halo-band implicit GEMM as conv3x3_tc_kernel, as a persistent, warp-specialised
// kernel: each block walks tiles blockIdx.x, + gridDim.x, ... with
//   warps 0-7  loading (cp.async) the band slice and weights of each (tile, stage) into a
//              ring of ST stages; a loader thread signals a stage on its `full` mbarrier
//              once its own copies have landed (waited lazily, ST-1 stages behind, then
//              a proxy fence for the tensor core's reads);
//   warp 8     one thread issuing the nine MMAs of every stage into one of two TMEM
//              accumulators (tile parity) and releasing the stage (`empty`, by
//              tcgen05.commit) and the finished accumulator (`accfull`);
//   warps 9-12 draining an accumulator (TMEM lane quarter = warp % 4) to the output
//              while the next tile accumulates in the other one, then `accempty`.
// So loads, MMAs and the epilogue of consecutive tiles overlap, and the per-block set-up
// (barriers, TMEM allocation) happens once per SM slot instead of once per tile.  Every
// wait is bounded; a block that runs out sets *err and all its roles stop.
constexpr int TCP_LW = 8;                          // loader warps (0 .. TCP_LW-1)
constexpr int TCP_LOAD_THREADS = 32 * TCP_LW;
constexpr int TCP_THREADS = 32 * (TCP_LW + 1 + 4);   // + the MMA warp + four epilogue warps

__device__ __forceinline__ void mbar_init(unsigned long long* b, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(b)) : "memory");
}

template <int N, int ST>
__global__ void __launch_bounds__(TCP_THREADS, 1) conv3x3_tcp_kernel(
    const bf16* __restrict__ in, int in_cs, int in_co, int Cin, const bf16* __restrict__ W,
    const float* __restrict__ bias, bf16* __restrict__ out, int out_cs, int out_co, int Cout, int B, int H, int Wd,
    int relu, int* err, int band, int stage_bytes, long long limit, int ntiles) {
    constexpr int M = 128;
    constexpr int TCOLS = N < 32 ? 32 : N;
    constexpr int ACOLS = 2 * TCOLS;               // two accumulators
    constexpr int D = ST - 1;                      // stages whose loads are awaited lazily
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long full[ST], empty[ST], accfull[2], accempty[2];
    __shared__ unsigned tmem_base_sh;
    __shared__ int fail_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Wp = Wd + 1;
    const unsigned img = (unsigned)(H + 1) * (unsigned)Wp;
    const long long total = (long long)B * img;
    const int n0 = blockIdx.y * N;
    const int plane = band * 16;
    const int bwt = 2 * plane;
    const int nstages = Cin / 16;
    const bool vec = (out_cs % 8 == 0) && (out_co % 8 == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
    const int nt = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    if (tid == 0) {
        fail_sh = 0;
        for (int i = 0; i < ST; i++) {
            mbar_init(&full[i], TCP_LOAD_THREADS);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&accfull[i], 1);
            mbar_init(&accempty[i], 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == TCP_LW) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "n"(ACOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const unsigned tmem = tmem_base_sh;
    const long long LIMIT = limit;
    volatile int* failp = &fail_sh;
    // padded position -> input pixel, or -1 (pad column, pad row, outside the batch)
    auto pix_of = [&](long long q) -> int {
        if (q < 0 || q >= total) return -1;
        const unsigned uq = (unsigned)q;
        const unsigned b = uq / img, r = uq - b * img;
        const unsigned y = r / (unsigned)Wp, xp = r - y * (unsigned)Wp;
        return (y < (unsigned)H && xp > 0u) ? (int)((b * (unsigned)H + y) * (unsigned)Wd + xp - 1u) : -1;
    };
    auto core_off = [](int r, int h) { return ((r >> 3) * 2 + h) * 128 + (r & 7) * 16; };
    int last_commit_slot = -1, last_commit_parity = 0;  // MMA thread: its last release of a stage
    if (warp < TCP_LW) {
        // ---- loaders
        int g = 0;
        bool ok = true;
        for (int j = 0; j < nt && ok; j++) {
            const long long q0 = (long long)((int)blockIdx.x + j * (int)gridDim.x) * M;
            for (int s = 0; s < nstages; s++, g++) {
                const int slot = g % ST;
                if (g >= ST && !mbar_wait(smem_u32(&empty[slot]), ((g / ST) - 1) & 1, LIMIT)) {
                    atomicExch(&fail_sh, 1);
                    ok = false;
                    break;
                }
                if (*failp) { ok = false; break; }
                unsigned char* base = smem + slot * stage_bytes;
                const int cs = s * 16;
                for (int c = tid; c < 2 * band; c += TCP_LOAD_THREADS) {
                    const int h = c >= band ? 1 : 0, i = c - h * band;
                    const int pix = pix_of(q0 - (Wp + 1) + i);
                    cp_async16(base + h * plane + i * 16, in + (long long)(pix >= 0 ? pix : 0) * in_cs + in_co + cs + h * 8,
                               pix >= 0);
                }
                for (int c = tid; c < 9 * 2 * N; c += TCP_LOAD_THREADS) {
                    const int tap = c / (2 * N), rem = c - tap * 2 * N;
                    const int rr = rem >> 1, h = rem & 1;
                    const int co = n0 + rr;
                    const bool okb = co < Cout;
                    cp_async16(base + bwt + tap * N * 32 + core_off(rr, h),
                               W + ((long long)(okb ? co : 0) * 9 + tap) * Cin + cs + h * 8, okb);
                }
                cp_commit();
                if (g >= D) {  // this thread's copies of stage g - D have landed
                    cp_wait<D>();
                    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                    mbar_arrive(&full[(g - D) % ST]);
                }
            }
        }
        // the stages not yet signalled
        cp_wait<0>();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if (ok)
            for (int k = (g - D > 0 ? g - D : 0); k < g; k++) mbar_arrive(&full[k % ST]);
    } else if (warp == TCP_LW) {
        // ---- MMA issuer
        if (lane == 0) {
            const unsigned idesc =
                (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
            int g = 0;
            bool ok = true;
            for (int j = 0; j < nt && ok; j++) {
                const int acc = j & 1;
                if (j >= 2 && !mbar_wait(smem_u32(&accempty[acc]), ((j >> 1) - 1) & 1, LIMIT)) {
                    atomicExch(&fail_sh, 1);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                const unsigned dtm = tmem + (unsigned)(acc * TCOLS);
                for (int s = 0; s < nstages; s++, g++) {
                    const int slot = g % ST;
                    if (*failp || !mbar_wait(smem_u32(&full[slot]), (g / ST) & 1, LIMIT)) {
                        atomicExch(&fail_sh, 1);
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
                    const unsigned base = smem_u32(smem + slot * stage_bytes);
#pragma unroll 1
                    for (int tap = 0; tap < 9; tap++) {
                        const unsigned off = (unsigned)(((tap / 3) * Wp + tap % 3) * 16);
                        const uint64_t ad = umma_desc(base + off, (unsigned)plane, 128);
                        const uint64_t bd = umma_desc(base + bwt + tap * N * 32, 128, 256);
                        const unsigned accf = (s > 0 || tap > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtm),
                            "l"(ad), "l"(bd), "r"(idesc), "r"(accf));
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                            smem_u32(&empty[slot])));
                    last_commit_slot = slot;
                    last_commit_parity = (g / ST) & 1;
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                    smem_u32(&accfull[acc])));
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: TMEM lane quarter of this warp = its rows of the tile
        const int quad = warp & 3;
        for (int j = 0; j < nt; j++) {
            const int acc = j & 1;
            if (*failp || !mbar_wait(smem_u32(&accfull[acc]), (j >> 1) & 1, LIMIT)) {
                atomicExch(&fail_sh, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const long long q0 = (long long)((int)blockIdx.x + j * (int)gridDim.x) * M;
            const int pix = pix_of(q0 + quad * 32 + lane);
#pragma unroll 1
            for (int c0 = 0; c0 < N; c0 += 16) {
                unsigned v[16];
                const unsigned ta = tmem + ((unsigned)(quad * 32) << 16) + (unsigned)(acc * TCOLS + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
                if (pix >= 0) store16(v, out + (long long)pix * out_cs + out_co, n0 + c0, Cout, bias, relu, vec);
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
            mbar_arrive(&accempty[acc]);
        }
    }
    __syncthreads();
    // a block that gave up waits (bounded, default limit) for the MMAs it has in flight
    // before its TMEM is freed
    if (warp == TCP_LW && lane == 0 && *failp && last_commit_slot >= 0)
        mbar_wait(smem_u32(&empty[last_commit_slot]), last_commit_parity, kWaitLimitDefault);
    if (tid == 0 && *failp) atomicExch(err, 1);
    __syncthreads();
    if (warp == TCP_LW) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(ACOLS));
    }
}

template <int N, int ST>
static cudaError_t launch_conv_tcp_st(const bf16* in, int in_cs, int in_co, int Cin, const bf16* W, const float* bias,
                                      bf16* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu,
                                      int* err, cudaStream_t st, int band, int stage_bytes) {
    const int smem = ST * stage_bytes;
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tcp_kernel<N, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long positions = (long long)B * (H + 1) * (Wd + 1);
    const int ntiles = (int)((positions + 127) / 128);
    constexpr int ACOLS = 2 * (N < 32 ? 32 : N);
    int bps = (227 * 1024) / (smem + 2048);
    if (bps > 512 / ACOLS) bps = 512 / ACOLS;
    if (bps > 2) bps = 2;
    if (bps < 1) bps = 1;
    const int ny = (Cout + N - 1) / N;
    int gx = (148 * bps + ny - 1) / ny;
    if (gx > ntiles) gx = ntiles;
    conv3x3_tcp_kernel<N, ST><<<dim3((unsigned)gx, (unsigned)ny), TCP_THREADS, smem, st>>>(
        in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu, err, band, stage_bytes,
        g_wait_limit, ntiles);
    return cudaGetLastError();
}

// Stages of the ring: as many (2..4) as fit in 110 KB, so that two blocks share an SM.
template <int N>
static cudaError_t launch_conv_tcp(const bf16* in, int in_cs, int in_co, int Cin, const bf16* W, const float* bias,
                                   bf16* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu,
                                   int* err, cudaStream_t st) {
    const int band = 128 + 2 * (Wd + 1) + 2;
    const int stage_bytes = ((2 * band * 16 + 9 * N * 32) + 127) / 128 * 128;
    const int fit = (110 * 1024) / stage_bytes;
    if (fit >= 4)
        return launch_conv_tcp_st<N, 4>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu,
                                        err, st, band, stage_bytes);
    if (fit == 3)
        return launch_conv_tcp_st<N, 3>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu,
                                        err, st, band, stage_bytes);
    return launch_conv_tcp_st<N, 2>(in, in_cs, in_co, Cin, W, bias, out, out_cs, out_co, Cout, B, H, Wd, relu, err,
                                    st, band, stage_bytes);
}

// The kernel of mm_nn_conv3x3_tc: the one-tile-per-block halo-band kernel (default), or
// the persistent warp-specialised one (mm_nn_set_conv_kernel(1), or MM_NN_CONV=persistent
// in the environment).  Measured per layer of the network at batch 256, the persistent
// kernel is ahead only on the 16x16 layers with 128 output channels (d2a 161 vs 169 us)
// and behind on the 64x64 ones (d0a 441 vs 292 us): its 128 loader threads per block
// bring in less of the band at a time than the 256 of the other kernel.
static int g_conv_kind = -1;
static bool conv_persistent() {
    if (g_conv_kind < 0) {
        const char* e = getenv("MM_NN_CONV");
        g_conv_kind = (e && e[0] == 'p') ? 1 : 0;
    }
    return g_conv_kind == 1;
}

// ---------------------------------------------------------------- tcgen05 weight gradient
// dW_tap[co][ci] = sum_q dY[q][co] X[q + off(tap)][ci] over the padded positions q of the
// halo-band layout (pads carry zero dY and zero X): nine GEMMs with K = positions, one
// TMEM accumulator each (M = 128 output channels, N = 32 input channels; 9 x 32 of the 512
// columns).  Both operands stay pixel-major as loaded, i.e. MN-major in the tcgen05
// sense: a plane per 8 channels holds 16 bytes per position, 8 consecutive positions
// form a core matrix (K-direction stride 128 bytes), planes are the MN-direction
// stride.  The X operand of tap (dy, dx) is the stage's band shifted along K by
// ((dy+1)(W+1) + dx+1) positions, a 16-byte-aligned descriptor offset.  Blocks split
// the positions; each adds its nine 128 x 32 partial sums to dW with FP32 atomics.
constexpr int WGT_KC = 64;  // positions per stage

__device__ __forceinline__ int band_pixel(int q, int total, int img, int Wp, int H, int Wd) {
    if (q < 0 || q >= total) return -1;
    const int b = q / img, r = q - b * img;
    const int y = r / Wp, xp = r - y * Wp;
    return (y < H && xp > 0) ? (b * H + y) * Wd + xp - 1 : -1;
}

constexpr int WGT_BAND_MAX = WGT_KC + 2 * 257 + 2;  // widths up to 256

template <int ST, int TG>
__global__ void __launch_bounds__(256) conv3x3_wgrad_tc_kernel(const bf16* __restrict__ dy, int dy_cs, int dy_co,
                                                               int Cout, const bf16* __restrict__ x, int x_cs,
                                                               int x_co, int Cin, float* __restrict__ dW, int B,
                                                               int H, int Wd, int* err, int band, int stage_bytes,
                                                               int per_block, long long limit) {
    constexpr int M = 128, N = 32, KC = WGT_KC;
    constexpr int TCOLS = TG * N > 256 ? 512 : (TG * N > 128 ? 256 : (TG * N > 64 ? 128 : 64));
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long mbar[ST];
    __shared__ unsigned tmem_base_sh;
    __shared__ int fail_sh;
    __shared__ int s_pix[2][WGT_BAND_MAX];         // band position -> pixel (or -1), two stages
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Wp = Wd + 1;
    const int img = (H + 1) * Wp;
    const int total = B * img;
    const int q_begin = blockIdx.x * per_block;
    const int q_end = q_begin + per_block < total ? q_begin + per_block : total;
    // blockIdx.y: input-channel tile and group of TG taps (taps tap0 .. tap0 + TG - 1)
    const int ngroups = 9 / TG;
    const int tap0 = (blockIdx.y % ngroups) * TG;
    const int ci0 = (blockIdx.y / ngroups) * N, co0 = blockIdx.z * M;
    // channel planes that exist: the others are never loaded, and the D rows / columns
    // they would feed are never stored
    const int ga = min(16, (Cout - co0 + 7) / 8), gb = min(4, (Cin - ci0 + 7) / 8);
    constexpr int PLANE_A = KC * 16;                // bytes per 8-channel plane of dY
    const int plane_b = band * 16;                  // bytes per 8-channel plane of the X band
    const int a_bytes = 16 * PLANE_A;               // 16 planes = 128 output channels
    if (tid == 0) {
        fail_sh = 0;
        for (int i = 0; i < ST; i++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[i])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "n"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const unsigned tmem = tmem_base_sh;
    const int nstages = q_end > q_begin ? (q_end - q_begin + KC - 1) / KC : 0;
    // BF16 A and B, F32 D, both operands MN-major (transpose bits 15 and 16)
    const unsigned idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((unsigned)(N >> 3) << 17) |
                           ((unsigned)(M >> 4) << 24);
    const long long LIMIT = limit;
    // the band of stage s: positions q0 - (W+2) .. q0 + KC + W, q0 = q_begin + s KC
    auto fill_pix = [&](int s) {
        const int qb = q_begin + s * KC - (Wp + 1);
        for (int i = tid; i < band; i += 256) s_pix[s & 1][i] = band_pixel(qb + i, total, img, Wp, H, Wd);
    };
    auto load_stage = [&](int s) {
        unsigned char* base = smem + (s % ST) * stage_bytes;
        const int q0 = q_begin + s * KC;
        const int* pixs = s_pix[s & 1];
        // dY rows of positions q0 .. q0+KC-1 (band entries W+2 ..): zero past this block's range
        for (int c = tid; c < ga * KC; c += 256) {
            const int g = c / KC, i = c - g * KC;
            const int pix = (q0 + i < q_end) ? pixs[Wp + 1 + i] : -1;
            const bool ok = pix >= 0;
            cp_async16(base + g * PLANE_A + i * 16, dy + (long long)(ok ? pix : 0) * dy_cs + dy_co + co0 + g * 8, ok);
        }
        unsigned char* bb = base + a_bytes;
        for (int c = tid; c < gb * band; c += 256) {
            const int g = c / band, i = c - g * band;
            const int pix = pixs[i];
            const bool ok = pix >= 0;
            cp_async16(bb + g * plane_b + i * 16, x + (long long)(ok ? pix : 0) * x_cs + x_co + ci0 + g * 8, ok);
        }
    };
    for (int s = 0; s < ST - 1; s++) {
        if (s < nstages) {
            fill_pix(s);
            __syncthreads();
            load_stage(s);
        }
        cp_commit();
    }
    int issued = 0;
    for (int s = 0; s < nstages; s++) {
        cp_wait<ST - 2>();
        asm volatile("fence.proxy.async.shared::cta;\n" ::);
        __syncthreads();
        if (fail_sh) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const unsigned base = smem_u32(smem + (s % ST) * stage_bytes);
#pragma unroll 1
            for (int tg = 0; tg < TG; tg++) {
                const int tap = tap0 + tg;
                const unsigned off = (unsigned)((tap / 3) * Wp + tap % 3);
#pragma unroll 1
                for (int kk = 0; kk < KC / 16; kk++) {
                    const uint64_t ad = umma_desc(base + kk * 16 * 16, 128, PLANE_A);
                    const uint64_t bd = umma_desc(base + a_bytes + (kk * 16 + off) * 16, 128, (unsigned)plane_b);
                    const unsigned acc = (s > 0 || kk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem + tg * N),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&mbar[s % ST])));
        }
        issued = s + 1;
        const int nx = s + ST - 1;
        if (nx < nstages) {
            if (s >= 1 && !mbar_wait(smem_u32(&mbar[(s - 1) % ST]), ((s - 1) / ST) & 1, LIMIT)) {
                if (lane == 0) atomicExch(&fail_sh, 1);
            }
            fill_pix(nx);
            __syncthreads();
            if (!fail_sh) load_stage(nx);
        }
        cp_commit();
    }
    cp_wait<0>();
    __syncthreads();
    // every MMA done before the TMEM is freed (see the forward kernel)
    if (issued > 0) {
        const int last = issued - 1;
        const bool ok = !fail_sh && mbar_wait(smem_u32(&mbar[last % ST]), (last / ST) & 1, LIMIT);
        if (!ok) {
            if (lane == 0) atomicExch(&fail_sh, 1);
            mbar_wait(smem_u32(&mbar[last % ST]), (last / ST) & 1, kWaitLimitDefault);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (output channels); warps 0-3
    // take the first (TG+1)/2 taps of the block, warps 4-7 the others
    const int quad = warp & 3, half = warp >> 2;
    constexpr int TH = (TG + 1) / 2;
    if (!fail_sh && issued > 0) {
        const int co = co0 + quad * 32 + lane;
        for (int tg = half * TH; tg < (half ? TG : TH); tg++) {
            const int tap = tap0 + tg;
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                if (ci0 + c0 >= Cin) break;   // warp-uniform
                unsigned v[16];
                const unsigned ta = tmem + ((unsigned)(quad * 32) << 16) + (unsigned)(tg * N + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
                if (co < Cout) {
                    float* d = dW + ((long long)co * 9 + tap) * Cin + ci0 + c0;
#pragma unroll
                    for (int e = 0; e < 16; e++)
                        if (ci0 + c0 + e < Cin) atomicAdd(d + e, __uint_as_float(v[e]));
                }
            }
        }
    } else if (fail_sh && tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(TCOLS));
    }
}

// TG taps per block: 9 (one block per SM, all 512 TMEM columns) or 3 (three tap groups
// as separate blocks, 128 columns each, up to four blocks per SM).
template <int ST, int TG>
static cudaError_t launch_wgrad_tc_st(const bf16* dy, int dy_cs, int dy_co, int Cout, const bf16* x, int x_cs,
                                      int x_co, int Cin, float* dW, int B, int H, int Wd, int* err, int band,
                                      int stage_bytes, cudaStream_t st) {
    // with all 512 TMEM columns in one block, at least 116 KB of shared memory keeps a
    // second block off the SM, so no allocation ever waits for another block; with 128
    // columns, four blocks fit the TMEM and shared memory is limited to a quarter
    const int smem = TG == 9 ? (ST * stage_bytes > 116 * 1024 ? ST * stage_bytes : 116 * 1024)
                             : (ST * stage_bytes > 56 * 1024 ? ST * stage_bytes : 56 * 1024);
    cudaError_t e =
        cudaFuncSetAttribute(conv3x3_wgrad_tc_kernel<ST, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long long total = (long long)B * (H + 1) * (Wd + 1);
    const int ct = (Cin + 31) / 32, mt = (Cout + 127) / 128;
    const int ng = 9 / TG;
    // about two (TG = 9) or eight (TG = 3) blocks' worth of work per SM, whole stages per block
    long long chunks = ((TG == 9 ? 2LL : 8LL) * 148 + (long long)ct * mt * ng - 1) / ((long long)ct * mt * ng);
    long long per = (total + chunks - 1) / chunks;
    per = (per + WGT_KC - 1) / WGT_KC * WGT_KC;
    chunks = (total + per - 1) / per;
    dim3 grid((unsigned)chunks, (unsigned)(ct * ng), (unsigned)mt);
    conv3x3_wgrad_tc_kernel<ST, TG><<<grid, 256, smem, st>>>(dy, dy_cs, dy_co, Cout, x, x_cs, x_co, Cin, dW, B, H, Wd,
                                                             err, band, stage_bytes, (int)per, g_wait_limit);
    return cudaGetLastError();
}

static int g_wgrad_tg = -1;  // taps per block of the tcgen05 weight gradient: 9 or 3
static int wgrad_taps() {
    if (g_wgrad_tg < 0) {
        const char* e = getenv("MM_NN_WGRAD_TAPS");
        g_wgrad_tg = (e && e[0] == '9') ? 9 : 3;
    }
    return g_wgrad_tg;
}

}  // namespace mm

extern "C" MM_API int mm_nn_set_wait_limit(long long iterations) {
    g_wait_limit = iterations < 0 ? kWaitLimitDefault : iterations;
    return MM_OK;
}

// tcgen05 variant of mm_nn_conv3x3_wgrad (dW accumulated, so zero it first; plus a device
// error flag that a timed-out wait sets).
extern "C" MM_API int mm_nn_conv3x3_wgrad_tc(const void* dy, int dy_cs, int dy_co, int Cout, const void* x, int x_cs,
                                             int x_co, int Cin, float* dW, int B, int H, int Wd, int* err,
                                             mm_stream st) {
    if (Cin % 8 || Cout % 8 || dy_cs % 8 || dy_co % 8 || x_cs % 8 || x_co % 8 || Wd < 1 || Wd > 256 || H < 1 ||
        B < 1 || !err || (long long)B * (H + 1) * (Wd + 1) >= (1LL << 30))
        return report_error(MM_ERR_ARG, "mm_nn_conv3x3_wgrad_tc: bad argument");
    const int band = WGT_KC + 2 * (Wd + 1) + 2;
    const int stage_bytes = ((16 * WGT_KC * 16 + 4 * band * 16) + 127) / 128 * 128;
    cudaError_t e;
    const bf16 *dyb = (const bf16*)dy, *xb = (const bf16*)x;
    cudaStream_t s = (cudaStream_t)st;
    if (wgrad_taps() == 9) {
        const int fit = (200 * 1024) / stage_bytes;
        if (fit >= 4)
            e = launch_wgrad_tc_st<4, 9>(dyb, dy_cs, dy_co, Cout, xb, x_cs, x_co, Cin, dW, B, H, Wd, err, band, stage_bytes, s);
        else if (fit == 3)
            e = launch_wgrad_tc_st<3, 9>(dyb, dy_cs, dy_co, Cout, xb, x_cs, x_co, Cin, dW, B, H, Wd, err, band, stage_bytes, s);
        else
            e = launch_wgrad_tc_st<2, 9>(dyb, dy_cs, dy_co, Cout, xb, x_cs, x_co, Cin, dW, B, H, Wd, err, band, stage_bytes, s);
    } else {
        const int fit = (56 * 1024) / stage_bytes;
        if (fit >= 3)
            e = launch_wgrad_tc_st<3, 3>(dyb, dy_cs, dy_co, Cout, xb, x_cs, x_co, Cin, dW, B, H, Wd, err, band, stage_bytes, s);
        else
            e = launch_wgrad_tc_st<2, 3>(dyb, dy_cs, dy_co, Cout, xb, x_cs, x_co, Cin, dW, B, H, Wd, err, band, stage_bytes, s);
    }
    if (e != cudaSuccess) return report_error(MM_ERR_CUDA, cudaGetErrorString(e));
    return MM_OK;
}

extern "C" MM_API int mm_nn_set_conv_kernel(int persistent) {
    if (persistent != 0 && persistent != 1) return report_error(MM_ERR_ARG, "mm_nn_set_conv_kernel: 0 or 1");
    g_conv_kind = persistent;
    return MM_OK;
}

// tcgen05 variant of mm_nn_conv3x3 (same arguments plus a device error flag that a
// timed-out wait sets); N tile = 16..128 chosen from Cout.
extern "C" MM_API int mm_nn_conv3x3_tc(const void* in, int in_cs, int in_co, int Cin, const void* W, const float* bias,
                                       void* out, int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu,
                                       int* err, mm_stream st) {
    if (Cin % 16 || in_cs % 8 || in_co % 8 || Cout < 1 || B < 1 || H < 1 || Wd < 1 || Wd > 256 || (out_co & 1) ||
        (out_cs & 1) || !err)
        return report_error(MM_ERR_ARG, "mm_nn_conv3x3_tc: bad argument");
    cudaError_t e;
    const bf16* i = (const bf16*)in;
    const bf16* w = (const bf16*)W;
    bf16* o = (bf16*)out;
    cudaStream_t s = (cudaStream_t)st;
    const bool pers = conv_persistent() && (long long)B * (H + 1) * (Wd + 1) < (1LL << 31);
    if (pers) {
        if (Cout <= 16) e = launch_conv_tcp<16>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
        else if (Cout <= 32) e = launch_conv_tcp<32>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
        else if (Cout <= 64) e = launch_conv_tcp<64>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
        else e = launch_conv_tcp<128>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
    } else if (Cout <= 16) e = launch_conv_tc<16>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
    else if (Cout <= 32) e = launch_conv_tc<32>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
    else if (Cout <= 64) e = launch_conv_tc<64>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
    else e = launch_conv_tc<128>(i, in_cs, in_co, Cin, w, bias, o, out_cs, out_co, Cout, B, H, Wd, relu, err, s);
    if (e != cudaSuccess) return report_error(MM_ERR_CUDA, cudaGetErrorString(e));
    return MM_OK;
}

// ---------------------------------------------------------------- input features
// feats[q][p][0..15] (bf16) of relaxation problem q: mask, Ms/1e6, Aex/1e-11, Ku/1e5,
// axis x, axis y (all times the mask), B_x/0.05 T, B_y/0.05 T, 1, zeros; from the masks
// [nq][P] and a parameter table prm[q][8] = (Ms, Aex, Ku, ux, uy, Bx, By, 0).
namespace mm {
__global__ void features_kernel(const float* masks, const float* prm, long long nq, int P, bf16* out) {
    const long long n = nq * P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long q = e / P;
        const float m = masks[e];
        const float* pr = prm + q * 8;
        float f[16] = {m, m * pr[0] / 1e6f, m * pr[1] / 1e-11f, m * pr[2] / 1e5f, m * pr[3], m * pr[4], pr[5] / 0.05f,
                       pr[6] / 0.05f, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + e * 16);
#pragma unroll
        for (int c = 0; c < 8; c++) o[c] = __floats2bfloat162_rn(f[2 * c], f[2 * c + 1]);
    }
}
}  // namespace mm

extern "C" MM_API int mm_nn_features(const float* masks, const float* prm, long long nq, int P, void* out,
                                     mm_stream st) {
    features_kernel<<<grid1(nq * P), 256, 0, (cudaStream_t)st>>>(masks, prm, nq, P, (bf16*)out);
    NN_CHECK();
    return MM_OK;
}

// ---------------------------------------------------------------- output -> initial states
// state[q][c][p] (internal SoA: c = 0,1,2 = m_z, m_y, m_x) = mask * normalised first three
// output channels (user order m_x, m_y, m_z) of problem q; a zero vector stays zero.
namespace mm {
__global__ void output_state_kernel(const bf16* out, int out_cs, const float* masks, long long nq, int P,
                                    float* state) {
    const long long n = nq * P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long q = e / P;
        const int p = (int)(e - q * P);
        const bf16* o = out + e * out_cs;
        const float x = __bfloat162float(o[0]), y = __bfloat162float(o[1]), z = __bfloat162float(o[2]);
        const float r = sqrtf(x * x + y * y + z * z);
        const float s = (r > 0.f ? 1.f / r : 0.f) * masks[e];
        float* d = state + q * 3LL * P + p;
        d[0] = z * s;
        d[P] = y * s;
        d[2LL * P] = x * s;
    }
}
}  // namespace mm

extern "C" MM_API int mm_nn_output_state(const void* out, int out_cs, const float* masks, long long nq, int P,
                                         float* state, mm_stream st) {
    if (out_cs < 3 || nq < 0 || P < 1) return report_error(MM_ERR_ARG, "mm_nn_output_state: bad argument");
    output_state_kernel<<<grid1(nq * P), 256, 0, (cudaStream_t)st>>>((const bf16*)out, out_cs, masks, nq, P, state);
    NN_CHECK();
    return MM_OK;
}
