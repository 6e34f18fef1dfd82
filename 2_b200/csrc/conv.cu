// conv.cu -- FFT convolution passes of the demag field.
//
// Replaces MaxwellPlan.update (src/mumax/modules/maxwell_convolution.go:272-309): the
// reference zero-pads each component into a full-size buffer (fftplanX.go:80-97),
// runs cuFFT R2C over the whole padded volume, accumulates up to nine cmadd passes
// (add.cu:202-221) and runs three C2R transforms plus crops.  Here the padded half is
// never stored: the row pass reads only the N2 real inputs, the column passes read
// and write only the non-zero rows, and the symmetric 3x3 kernel multiply happens in
// registers between the forward and inverse transforms of the innermost column pass.
//
//   pass  2-D film (N0 == 1)                 3-D (N0 > 1)
//   1     x rows  R2C  (xfwd)                x rows R2C   (xfwd)
//   2     y cols  fwd * K inv (colmul)       y cols fwd   (colfft)
//   3     x rows  C2R + epilogue (rhs.cu)    z cols fwd * K inv (colmul)
//   4                                        y cols inv   (colfft)
//   5                                        x rows C2R + epilogue (rhs.cu)
#include <cstdio>

#include "fft.cuh"
#include "mm_internal.h"

namespace mm {
using namespace mmfft;

__device__ __forceinline__ bool conv_skip(const DevCtl* ctl, int skip_retry) {
    return ctl && (ctl->done || (skip_retry && ctl->tries > 0));
}

// ---------------------------------------------------------------- R2C row pass
// rows: r = (c*Z + z)*Y + y over C components; input row r starts at in + r*in_pitch
// (reals, n_in of them; the rest of the length-2M row is zero);
// output row (c, z, y) goes to out + ((c*Z + z)*Yout + y)*hp (h = M+1 complex).
// mask (optional): input multiplied by mask[(z*Y + y)*in_pitch + x] (same for all c).
template <int M, typename V, typename S>
__global__ void __launch_bounds__(256) xfwd_kernel(const S* __restrict__ in_fixed, PP in_pp, const float* __restrict__ mask,
                                                   V* __restrict__ out, int nrows, int Z, int Y, int Yout,
                                                   int in_pitch, int n_in, int hp, const DevCtl* ctl, int skip_retry) {
    if (conv_skip(ctl, skip_retry)) return;
    const S* in = in_fixed ? in_fixed : reinterpret_cast<const S*>(in_pp.get(ctl ? ctl->cur : 0));
    constexpr int TPL = tpl(M);
    constexpr int LL = line_len(M);
    extern __shared__ unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int rpb = blockDim.x / TPL;
    const int lr = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    const int row = blockIdx.x * rpb + lr;
    const bool active = (row < nrows) && (lr < rpb);
    V* x = sm + lr * LL;
    if (active) {
        const S* src = in + (long long)row * in_pitch;
        const int zy = row % (Z * Y);
        const float* msk = mask ? mask + (long long)zy * in_pitch : nullptr;
        for (int e = t; e < M; e += TPL) {
            S a = 0, b = 0;
            if (2 * e < n_in) a = src[2 * e] * (msk ? (S)msk[2 * e] : (S)1);
            if (2 * e + 1 < n_in) b = src[2 * e + 1] * (msk ? (S)msk[2 * e + 1] : (S)1);
            x[padx(e)] = mkv(a, b);
        }
    }
    __syncthreads();
    fft_line<M, -1, V>(x, t, active);
    if (active) {
        // X[k] = E[k] + W^k O[k], E = (Z[k] + conj Z[M-k])/2, O = (Z[k] - conj Z[M-k])/(2i)
        const int c = row / (Z * Y);
        const int zy = row % (Z * Y);
        const int z = zy / Y, y = zy % Y;
        V* dst = out + ((long long)(c * Z + z) * Yout + y) * hp;
        typedef typename Scalar<V>::T T;
        for (int k = t; k <= M / 2; k += TPL) {
            V zk = x[padx(k % M)];
            V zm = x[padx((M - k) % M)];
            V e = cscale(cadd(zk, cconj(zm)), (T)0.5);
            V o = cscale(csub(zk, cconj(zm)), (T)0.5);
            o = mkv(o.y, -o.x);  // divide by i
            V w = Tw<-1, V>::get(k, 2 * M);
            V wo = cmul(w, o);
            dst[k] = cadd(e, wo);
            if (k != M - k) {
                // X[M-k] = conj(E[k]) - conj(W^k O[k]) ... computed directly:
                // E[M-k] = conj(E[k]), O[M-k] = conj(O[k]), W^(M-k) = -conj(W^k)
                V em = cconj(e);
                V om = cconj(o);
                V wm = mkv(-w.x, w.y);
                dst[M - k] = cadd(em, cmul(wm, om));
            }
        }
    }
}

// ---------------------------------------------------------------- generic column pass
// One component per line.  Block b covers outer index o = b / ntiles and the kx tile
// (b % ntiles)*TC ... +TC.  Line element e of column kx sits at
//   base + o*outer_stride + e*line_stride + kx.
// Reads elements e < n_in (rest zero), writes elements e < n_out.
template <int L, int SIGN, typename V>
__global__ void colfft_kernel(V* __restrict__ S, int ncols, int TC, long long outer_stride, long long line_stride,
                              int n_in, int n_out, const DevCtl* ctl, int skip_retry) {
    if (conv_skip(ctl, skip_retry)) return;
    constexpr int TPL = tpl(L);
    constexpr int LL = line_len(L);
    extern __shared__ unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    V* base = S + (long long)o * outer_stride + kx0;
    const int nthr = blockDim.x;
    for (int i = threadIdx.x; i < L * TC; i += nthr) {
        int e = i / TC, col = i % TC;
        V v = mkv((typename Scalar<V>::T)0, (typename Scalar<V>::T)0);
        if (e < n_in && kx0 + col < ncols) v = base[(long long)e * line_stride + col];
        sm[col * LL + padx(e)] = v;
    }
    __syncthreads();
    const int col = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    fft_line<L, SIGN, V>(sm + col * LL, t, col < TC);
    for (int i = threadIdx.x; i < n_out * TC; i += nthr) {
        int e = i / TC, c2 = i % TC;
        if (kx0 + c2 < ncols) base[(long long)e * line_stride + c2] = sm[c2 * LL + padx(e)];
    }
}

// ---------------------------------------------------------------- multiply pass
// Three components per column: forward transform, H_d = sum_s Khat_sd M_s (symmetric,
// real), inverse transform.  kaxis = 0: the line runs along z (ky = outer index);
// kaxis = 1: the line runs along y (kz = 0, 2-D films).
__device__ __forceinline__ void kernel_at(const KernelView& K, int kz, int ky, int kx, float out[6]) {
    float sz = 1.f, sy = 1.f;
    if (kz > K.L0 / 2) { kz = K.L0 - kz; sz = -1.f; }
    if (ky > K.L1 / 2) { ky = K.L1 - ky; sy = -1.f; }
    const long long cs = (long long)K.kd0 * K.kd1 * K.kd2;
    const long long idx = ((long long)kz * K.kd1 + ky) * K.kd2 + kx;
    // real-space K_sd is odd along axes s and d (s != d), so its transform flips sign
    // under k -> L-k along those axes; diagonal components are even.
    const float sg[6] = {1.f, 1.f, 1.f, sy, sz, sz * sy};
#pragma unroll
    for (int q = 0; q < 6; q++) out[q] = K.nz[q] ? sg[q] * __ldg(K.k + q * cs + idx) : 0.f;
}

template <int L>
__global__ void colmul_kernel(float2* __restrict__ S, KernelView K, int ncols, int TC, long long comp_stride,
                              long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                              const DevCtl* ctl, int skip_retry) {
    if (conv_skip(ctl, skip_retry)) return;
    constexpr int TPL = tpl(L);
    constexpr int LL = line_len(L);
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    float2* base = S + (long long)o * outer_stride + kx0;
    const int nthr = blockDim.x;
    for (int i = threadIdx.x; i < 3 * L * TC; i += nthr) {
        int c = i / (L * TC), r = i % (L * TC);
        int e = r / TC, col = r % TC;
        float2 v = make_float2(0.f, 0.f);
        if (e < n_in && kx0 + col < ncols) v = base[c * comp_stride + (long long)e * line_stride + col];
        sm[(c * TC + col) * LL + padx(e)] = v;
    }
    __syncthreads();
    const int col = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    const bool act = col < TC;
#pragma unroll 1
    for (int c = 0; c < 3; c++) fft_line<L, -1, float2>(sm + (c * TC + (act ? col : 0)) * LL, t, act);
    for (int i = threadIdx.x; i < L * TC; i += nthr) {
        int e = i / TC, c2 = i % TC;
        int kx = kx0 + c2;
        if (kx >= ncols) continue;
        float kk[6];
        if (kaxis == 0) kernel_at(K, e, o, kx, kk);
        else kernel_at(K, 0, e, kx, kk);
        float2 m0 = sm[(0 * TC + c2) * LL + padx(e)];
        float2 m1 = sm[(1 * TC + c2) * LL + padx(e)];
        float2 m2 = sm[(2 * TC + c2) * LL + padx(e)];
        // q: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy
        float2 h0 = make_float2(kk[0] * m0.x + kk[5] * m1.x + kk[4] * m2.x, kk[0] * m0.y + kk[5] * m1.y + kk[4] * m2.y);
        float2 h1 = make_float2(kk[5] * m0.x + kk[1] * m1.x + kk[3] * m2.x, kk[5] * m0.y + kk[1] * m1.y + kk[3] * m2.y);
        float2 h2 = make_float2(kk[4] * m0.x + kk[3] * m1.x + kk[2] * m2.x, kk[4] * m0.y + kk[3] * m1.y + kk[2] * m2.y);
        sm[(0 * TC + c2) * LL + padx(e)] = make_float2(h0.x * scale, h0.y * scale);
        sm[(1 * TC + c2) * LL + padx(e)] = make_float2(h1.x * scale, h1.y * scale);
        sm[(2 * TC + c2) * LL + padx(e)] = make_float2(h2.x * scale, h2.y * scale);
    }
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < 3; c++) fft_line<L, +1, float2>(sm + (c * TC + (act ? col : 0)) * LL, t, act);
    for (int i = threadIdx.x; i < 3 * n_in * TC; i += nthr) {
        int c = i / (n_in * TC), r = i % (n_in * TC);
        int e = r / TC, c2 = r % TC;
        if (kx0 + c2 < ncols) base[c * comp_stride + (long long)e * line_stride + c2] = sm[(c * TC + c2) * LL + padx(e)];
    }
}

// ---------------------------------------------------------------- launch helpers
static int g_max_smem = 0;
static int max_smem() {
    if (!g_max_smem) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (g_max_smem <= 0) g_max_smem = 48 * 1024;
    }
    return g_max_smem;
}

template <typename KT> static cudaError_t set_smem(KT kern, size_t bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

#define MM_FOR_POW2(X) X(1) X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

template <int M, typename V, typename S>
static cudaError_t launch_xfwd_t(const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                                 int in_pitch, int n_in, int hp, const DevCtl* ctl, int skip_retry, cudaStream_t st) {
    constexpr int TPL = tpl(M);
    int rpb = TPL >= 256 ? 1 : 256 / TPL;
    size_t smem = (size_t)rpb * line_len(M) * sizeof(V);
    while (smem > (size_t)max_smem() && rpb > 1) { rpb /= 2; smem = (size_t)rpb * line_len(M) * sizeof(V); }
    cudaError_t e = set_smem(xfwd_kernel<M, V, S>, smem);
    if (e != cudaSuccess) return e;
    int blocks = (nrows + rpb - 1) / rpb;
    xfwd_kernel<M, V, S><<<blocks, rpb * TPL, smem, st>>>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, ctl,
                                                          skip_retry);
    return cudaGetLastError();
}

template <typename V, typename S>
cudaError_t launch_xfwd(int M, const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                        int in_pitch, int n_in, int hp, const DevCtl* ctl, int skip_retry, cudaStream_t st) {
    switch (M) {
#define X(m) case m: return launch_xfwd_t<m, V, S>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, ctl, skip_retry, st);
        MM_FOR_POW2(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

// Picks the column tile width: as many columns as fit the shared-memory budget,
// up to 32 (256 B contiguous per row segment), at most 1024 threads.
static int pick_tc(int L, int ncomp, size_t vsize, int ncols) {
    int TC = 32;
    const size_t budget = 100 * 1024;
    while (TC > 1 && ((size_t)ncomp * TC * mmfft::line_len(L) * vsize > budget || TC * mmfft::tpl(L) > 1024)) TC /= 2;
    while (TC > 1 && TC / 2 >= ncols) TC /= 2;
    return TC;
}

template <int L, int SIGN, typename V>
static cudaError_t launch_colfft_t(V* S, int ncols, int nouter, long long outer_stride, long long line_stride,
                                   int n_in, int n_out, const DevCtl* ctl, int skip_retry, cudaStream_t st) {
    int TC = pick_tc(L, 1, sizeof(V), ncols);
    size_t smem = (size_t)TC * line_len(L) * sizeof(V);
    cudaError_t e = set_smem(colfft_kernel<L, SIGN, V>, smem);
    if (e != cudaSuccess) return e;
    int ntiles = (ncols + TC - 1) / TC;
    int threads = TC * tpl(L);
    if (threads < 32) threads = 32;
    colfft_kernel<L, SIGN, V><<<nouter * ntiles, threads, smem, st>>>(S, ncols, TC, outer_stride, line_stride, n_in,
                                                                      n_out, ctl, skip_retry);
    return cudaGetLastError();
}

template <typename V>
cudaError_t launch_colfft(int L, int sign, V* S, int ncols, int nouter, long long outer_stride,
                          long long line_stride, int n_in, int n_out, const DevCtl* ctl, int skip_retry,
                          cudaStream_t st) {
    if (sign < 0) {
        switch (L) {
#define X(l) case l: return launch_colfft_t<l, -1, V>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, ctl, skip_retry, st);
            MM_FOR_POW2(X)
#undef X
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (L) {
#define X(l) case l: return launch_colfft_t<l, 1, V>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, ctl, skip_retry, st);
            MM_FOR_POW2(X)
#undef X
            default: return cudaErrorInvalidValue;
        }
    }
}

template <int L>
static cudaError_t launch_colmul_t(float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                                   long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                                   const DevCtl* ctl, int skip_retry, cudaStream_t st) {
    int TC = pick_tc(L, 3, sizeof(float2), ncols);
    size_t smem = (size_t)3 * TC * line_len(L) * sizeof(float2);
    cudaError_t e = set_smem(colmul_kernel<L>, smem);
    if (e != cudaSuccess) return e;
    int ntiles = (ncols + TC - 1) / TC;
    int threads = TC * tpl(L);
    if (threads < 32) threads = 32;
    colmul_kernel<L><<<nouter * ntiles, threads, smem, st>>>(S, K, ncols, TC, comp_stride, outer_stride, line_stride,
                                                            n_in, kaxis, scale, ctl, skip_retry);
    return cudaGetLastError();
}

cudaError_t launch_colmul(int L, float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                          long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                          const DevCtl* ctl, int skip_retry, cudaStream_t st) {
    switch (L) {
#define X(l) case l: return launch_colmul_t<l>(S, K, ncols, nouter, comp_stride, outer_stride, line_stride, n_in, kaxis, scale, ctl, skip_retry, st);
        MM_FOR_POW2(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_xfwd<float2, float>(int, const float*, PP, const float*, float2*, int, int, int, int, int,
                                                int, int, const DevCtl*, int, cudaStream_t);
template cudaError_t launch_xfwd<double2, double>(int, const double*, PP, const float*, double2*, int, int, int, int,
                                                  int, int, int, const DevCtl*, int, cudaStream_t);
template cudaError_t launch_colfft<float2>(int, int, float2*, int, int, long long, long long, int, int, const DevCtl*,
                                           int, cudaStream_t);
template cudaError_t launch_colfft<double2>(int, int, double2*, int, int, long long, long long, int, int,
                                            const DevCtl*, int, cudaStream_t);

}  // namespace mm
