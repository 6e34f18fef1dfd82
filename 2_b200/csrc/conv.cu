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
//
// Column passes work on tiles of TC adjacent kx columns (TC a compile-time function
// of the line length), so every global access moves TC*8 contiguous bytes.
#include <cstdio>

#include "fft.cuh"
#include "fft4.cuh"
#include "mm_internal.h"
#include "kernel_view.cuh"
#include "pdl.cuh"

namespace mm {
using namespace mmfft;


// ---------------------------------------------------------------- R2C row pass
// rows (per simulation): r = (c*Z + z)*Y + y over C components; input row r starts at in + r*in_pitch
// (reals, n_in of them; the rest of the length-2M row is zero);
// output row (c, z, y) goes to out + ((c*Z + z)*Yout + y)*hp (h = M+1 complex).
// mask (optional): input multiplied by mask[(z*Y + y)*in_pitch + x] (same for all c).
template <int M, typename V, typename S>
__global__ void __launch_bounds__(256) xfwd_kernel(const S* __restrict__ in_fixed, PP in_pp, const float* __restrict__ mask,
                                                   V* __restrict__ out, int nrows, int Z, int Y, int Yout,
                                                   int in_pitch, int n_in, int hp, const float2* __restrict__ tw,
                                                   const DevCtl* ctl, int skip_retry, long long in_bstride,
                                                   long long out_bstride, long long mask_bstride) {
    const int sim = blockIdx.y;
    if (ctl) ctl += sim;
    if (conv_skip(ctl, skip_retry)) return;
    const S* in = (in_fixed ? in_fixed : reinterpret_cast<const S*>(in_pp.get(ctl ? ctl->cur : 0))) + sim * in_bstride;
    out += sim * out_bstride;
    if (mask) mask += sim * mask_bstride;
    constexpr int TPL = tpl(M);
    constexpr int LL = line_len(M);
    constexpr int RPB = TPL >= 256 ? 1 : 256 / TPL;
    extern __shared__ unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int lr = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    const int row = blockIdx.x * RPB + lr;
    const bool active = (row < nrows) && (lr < RPB);
    V* x = sm + (lr < RPB ? lr : 0) * LL;
    typedef typename Scalar<V>::T T;
    if (active) {
        const S* src = in + (long long)row * in_pitch;
        const int zy = row % (Z * Y);
        const float* msk = mask ? mask + (long long)zy * in_pitch : nullptr;
        const bool pairs = ((in_pitch & 1) == 0) && ((n_in & 1) == 0);
        if (pairs) {
            // two reals per load: z[e] = x[2e] + i x[2e+1]
            const int ne = n_in >> 1;
#pragma unroll 4
            for (int e = t; e < M; e += TPL) {
                V v = mkv((T)0, (T)0);
                if (e < ne) {
                    if constexpr (sizeof(S) == 4) {
                        float2 a = __ldg(reinterpret_cast<const float2*>(src) + e);
                        if (msk) {
                            float2 mm = __ldg(reinterpret_cast<const float2*>(msk) + e);
                            a.x *= mm.x;
                            a.y *= mm.y;
                        }
                        v = mkv((T)a.x, (T)a.y);
                    } else {
                        v = mkv((T)src[2 * e], (T)src[2 * e + 1]);
                    }
                }
                x[padx(e)] = v;
            }
        } else {
            for (int e = t; e < M; e += TPL) {
                S a = 0, b = 0;
                if (2 * e < n_in) a = src[2 * e] * (msk ? (S)msk[2 * e] : (S)1);
                if (2 * e + 1 < n_in) b = src[2 * e + 1] * (msk ? (S)msk[2 * e + 1] : (S)1);
                x[padx(e)] = mkv((T)a, (T)b);
            }
        }
    }
    __syncthreads();
    fft_line<M, -1, V>(x, t, active, tw);
    if (active) {
        // X[k] = E[k] + W^k O[k], E = (Z[k] + conj Z[M-k])/2, O = (Z[k] - conj Z[M-k])/(2i)
        const int c = row / (Z * Y);
        const int zy = row % (Z * Y);
        const int z = zy / Y, y = zy % Y;
        V* dst = out + ((long long)(c * Z + z) * Yout + y) * hp;
        for (int k = t; k <= M / 2; k += TPL) {
            V zk = x[padx(k & (M - 1))];
            V zm = x[padx((M - k) & (M - 1))];
            V e = cscale(cadd(zk, cconj(zm)), (T)0.5);
            V o = cscale(csub(zk, cconj(zm)), (T)0.5);
            o = mkv(o.y, -o.x);  // divide by i
            V w = TwSrc<-1, V>::get(tw, k, 2 * M);
            dst[k] = cadd(e, cmul(w, o));
            if (k != M - k) {
                // E[M-k] = conj E[k], O[M-k] = conj O[k], W^(M-k) = -conj W^k
                V wm = mkv(-w.x, w.y);
                dst[M - k] = cadd(cconj(e), cmul(wm, cconj(o)));
            }
        }
    }
}

// ---------------------------------------------------------------- column tiles
// Tile width: up to 32 columns, as many as fit 56 KB of shared memory and 1024 threads.
__host__ __device__ constexpr int col_tile(int L, int ncomp, int vsize) {
    int tc = 32;
    while (tc > 1 && (ncomp * tc * line_len(L) * vsize > 56 * 1024 || tc * tpl(L) > 1024)) tc /= 2;
    return tc;
}

// Copies rows e < n of the tile's columns (base + e*line_stride + col) into shared
// memory lines sm[(cline + col)*LL + padx(e)], zero-filling e in [n, L) if `zero`.
template <int L, int TC, typename V>
__device__ __forceinline__ void tile_load(V* sm, const V* __restrict__ base, long long line_stride, int n, int ncols_here,
                                          int cline, bool zero) {
    constexpr int LL = line_len(L);
    const int nthr = blockDim.x;
    bool done_vec = false;
    if constexpr (TC >= 2 && sizeof(V) == 8) {
        if (ncols_here == TC) {
            constexpr int TP = TC / 2;  // two columns per 16-byte access
            for (int i = threadIdx.x; i < n * TP; i += nthr) {
                const int e = i / TP, cp = (i % TP) * 2;
                float4 v = __ldg(reinterpret_cast<const float4*>(base + e * line_stride + cp));
                sm[(cline + cp) * LL + padx(e)] = make_float2(v.x, v.y);
                sm[(cline + cp + 1) * LL + padx(e)] = make_float2(v.z, v.w);
            }
            done_vec = true;
        }
    }
    if (!done_vec) {
        for (int i = threadIdx.x; i < n * TC; i += nthr) {
            const int e = i / TC, col = i % TC;
            V v = mkv((typename Scalar<V>::T)0, (typename Scalar<V>::T)0);
            if (col < ncols_here) v = base[e * line_stride + col];
            sm[(cline + col) * LL + padx(e)] = v;
        }
    }
    if (zero) {
        for (int i = threadIdx.x; i < (L - n) * TC; i += nthr) {
            const int e = n + i / TC, col = i % TC;
            sm[(cline + col) * LL + padx(e)] = mkv((typename Scalar<V>::T)0, (typename Scalar<V>::T)0);
        }
    }
}

template <int L, int TC, typename V>
__device__ __forceinline__ void tile_store(const V* sm, V* __restrict__ base, long long line_stride, int n, int ncols_here,
                                           int cline) {
    constexpr int LL = line_len(L);
    const int nthr = blockDim.x;
    bool done_vec = false;
    if constexpr (TC >= 2 && sizeof(V) == 8) {
        if (ncols_here == TC) {
            constexpr int TP = TC / 2;
            for (int i = threadIdx.x; i < n * TP; i += nthr) {
                const int e = i / TP, cp = (i % TP) * 2;
                V a = sm[(cline + cp) * LL + padx(e)];
                V b = sm[(cline + cp + 1) * LL + padx(e)];
                *reinterpret_cast<float4*>(base + e * line_stride + cp) = make_float4(a.x, a.y, b.x, b.y);
            }
            done_vec = true;
        }
    }
    if (!done_vec) {
        for (int i = threadIdx.x; i < n * TC; i += nthr) {
            const int e = i / TC, col = i % TC;
            if (col < ncols_here) base[e * line_stride + col] = sm[(cline + col) * LL + padx(e)];
        }
    }
}

// ---------------------------------------------------------------- generic column pass
// One component per line.  Block b covers outer index o = b / ntiles and the kx tile
// (b % ntiles)*TC ... +TC.  Line element e of column kx sits at
//   base + o*outer_stride + e*line_stride + kx.
// Reads elements e < n_in (rest zero), writes elements e < n_out.
template <int L, int SIGN, typename V>
__global__ void colfft_kernel(V* __restrict__ S, int ncols, long long outer_stride, long long line_stride, int n_in,
                              int n_out, const float2* __restrict__ tw, const DevCtl* ctl, int skip_retry,
                              long long sim_stride) {
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    constexpr int TC = col_tile(L, 1, sizeof(V));
    constexpr int TPL = tpl(L);
    constexpr int LL = line_len(L);
    extern __shared__ unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    const int nh = min(TC, ncols - kx0);
    V* base = S + (long long)o * outer_stride + kx0;
    tile_load<L, TC, V>(sm, base, line_stride, n_in, nh, 0, true);
    __syncthreads();
    const int col = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    fft_line<L, SIGN, V>(sm + (col < TC ? col : 0) * LL, t, col < TC, tw);
    tile_store<L, TC, V>(sm, base, line_stride, n_out, nh, 0);
}

// ---------------------------------------------------------------- multiply pass
// Three components per column: forward transform, H_d = sum_s Khat_sd M_s (symmetric,
// real), inverse transform.  kaxis = 0: the line runs along z (ky = outer index);
// kaxis = 1: the line runs along y (kz = 0, 2-D films).
template <int L>
__global__ void colmul_kernel(float2* __restrict__ S, KernelView K, int ncols, long long comp_stride,
                              long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                              const float2* __restrict__ tw, const DevCtl* ctl, int skip_retry, long long sim_stride,
                              const float* __restrict__ sim_scale) {
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    if (sim_scale) scale = sim_scale[blockIdx.y];
    constexpr int TC = col_tile(L, 3, 8);
    constexpr int TPL = tpl(L);
    constexpr int LL = line_len(L);
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    const int nh = min(TC, ncols - kx0);
    float2* base = S + (long long)o * outer_stride + kx0;
#pragma unroll 1
    for (int c = 0; c < 3; c++) tile_load<L, TC, float2>(sm, base + c * comp_stride, line_stride, n_in, nh, c * TC, true);
    __syncthreads();
    const int col = threadIdx.x / TPL;
    const int t = threadIdx.x % TPL;
    const bool act = col < TC;
#pragma unroll 1
    for (int c = 0; c < 3; c++) fft_line<L, -1, float2>(sm + (c * TC + (act ? col : 0)) * LL, t, act, tw);
    for (int i = threadIdx.x; i < L * TC; i += blockDim.x) {
        const int e = i / TC, c2 = i % TC;
        const int kx = kx0 + c2;
        if (c2 >= nh) continue;
        float kk[6];
        if (kaxis == 0) kernel_at(K, e, o, kx, kk);
        else kernel_at(K, 0, e, kx, kk);
        const int p = padx(e);
        float2 m0 = sm[(0 * TC + c2) * LL + p];
        float2 m1 = sm[(1 * TC + c2) * LL + p];
        float2 m2 = sm[(2 * TC + c2) * LL + p];
        // q: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy
        sm[(0 * TC + c2) * LL + p] = make_float2(scale * (kk[0] * m0.x + kk[5] * m1.x + kk[4] * m2.x),
                                                 scale * (kk[0] * m0.y + kk[5] * m1.y + kk[4] * m2.y));
        sm[(1 * TC + c2) * LL + p] = make_float2(scale * (kk[5] * m0.x + kk[1] * m1.x + kk[3] * m2.x),
                                                 scale * (kk[5] * m0.y + kk[1] * m1.y + kk[3] * m2.y));
        sm[(2 * TC + c2) * LL + p] = make_float2(scale * (kk[4] * m0.x + kk[3] * m1.x + kk[2] * m2.x),
                                                 scale * (kk[4] * m0.y + kk[3] * m1.y + kk[2] * m2.y));
    }
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < 3; c++) fft_line<L, +1, float2>(sm + (c * TC + (act ? col : 0)) * LL, t, act, tw);
#pragma unroll 1
    for (int c = 0; c < 3; c++) tile_store<L, TC, float2>(sm, base + c * comp_stride, line_stride, n_in, nh, c * TC);
}

// ---------------------------------------------------------------- register z-multiply
// The 3-D z pass without shared memory.  With the z direction zero-padded to
// L0 = 2P (P = N0 non-zero planes), the forward transform splits into its even and odd
// outputs, X[2k'] = DFT_P(x)[k'] and X[2k'+1] = DFT_P(x[z] W_{2P}^z)[k'], and the inverse
// likewise; so a lane pair takes one (ky, kx) column, each lane one parity, and every
// transform is a length-P DFT held in registers.  The two halves of the inverse are
// summed with one shuffle.  Replaces the z column FFT + multiply + inverse of colmul.

// exp(SIGN 2 pi i z / (2P)) from the FP32 table
template <int SIGN>
__device__ __forceinline__ float2 wtab(const float2* __restrict__ tw, int num, int den) {
    return TwSrc<SIGN, float2>::get(tw, num, den);
}

template <int P, bool BATCH>
__global__ void __launch_bounds__(128) zmul_reg_kernel(float2* __restrict__ S, KernelView K, int L1, int h, int hp,
                                                       long long comp_stride, long long zstride, float scale,
                                                       const float2* __restrict__ tw, const DevCtl* ctl,
                                                       int skip_retry, long long sim_stride,
                                                       const float* __restrict__ sim_scale) {
    pdl_begin();
    if (BATCH) {
        if (ctl) ctl += blockIdx.y;
        S += blockIdx.y * sim_stride;
        if (sim_scale) scale = sim_scale[blockIdx.y];
    }
    if (conv_skip(ctl, skip_retry)) return;
    const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s = (int)(gt & 1);
    const long long colg = gt >> 1;
    const bool active = colg < (long long)L1 * h;
    const int ky = active ? (int)(colg / h) : 0;
    const int kx = active ? (int)(colg % h) : 0;
    float2* base = S + (long long)ky * hp + kx;
    float2 x[3][P];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int z = 0; z < P; z++)
            x[c][z] = active ? base[c * comp_stride + z * zstride] : make_float2(0.f, 0.f);
    // odd outputs: pre-multiply by W_{2P}^z (forward)
    if (s) {
#pragma unroll
        for (int z = 1; z < P; z++) {
            const float2 w = wtab<-1>(tw, z, 2 * P);
#pragma unroll
            for (int c = 0; c < 3; c++) x[c][z] = cmul(x[c][z], w);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) RDft<P, -1>::run(x[c]);
    // multiply: x[c][k'] holds X_c[kz], kz = 2k' + s
    const int kyy = (ky > (K.L1 >> 1)) ? K.L1 - ky : ky;
    const float sy = (ky > (K.L1 >> 1)) ? -1.f : 1.f;
    const int cs = K.kd0 * K.kd1 * K.kd2;
#pragma unroll
    for (int k = 0; k < P; k++) {
        int kz = 2 * k + s;
        float sz = 1.f;
        if (kz > P) { kz = 2 * P - kz; sz = -1.f; }
        const int idx = (kz * K.kd1 + kyy) * K.kd2 + kx;
        const float kxx = __ldg(K.k + idx);
        const float kyy_ = __ldg(K.k + cs + idx);
        const float kzz = __ldg(K.k + 2 * cs + idx);
        const float kyz = K.nz[3] ? sy * __ldg(K.k + 3 * cs + idx) : 0.f;
        const float kxz = K.nz[4] ? sz * __ldg(K.k + 4 * cs + idx) : 0.f;
        const float kxy = K.nz[5] ? sz * sy * __ldg(K.k + 5 * cs + idx) : 0.f;
        const float2 m0 = x[0][k], m1 = x[1][k], m2 = x[2][k];
        x[0][k] = make_float2(scale * (kxx * m0.x + kxy * m1.x + kxz * m2.x), scale * (kxx * m0.y + kxy * m1.y + kxz * m2.y));
        x[1][k] = make_float2(scale * (kxy * m0.x + kyy_ * m1.x + kyz * m2.x), scale * (kxy * m0.y + kyy_ * m1.y + kyz * m2.y));
        x[2][k] = make_float2(scale * (kxz * m0.x + kyz * m1.x + kzz * m2.x), scale * (kxz * m0.y + kyz * m1.y + kzz * m2.y));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) RDft<P, +1>::run(x[c]);
    if (s) {
#pragma unroll
        for (int z = 1; z < P; z++) {
            const float2 w = wtab<+1>(tw, z, 2 * P);
#pragma unroll
            for (int c = 0; c < 3; c++) x[c][z] = cmul(x[c][z], w);
        }
    }
    // sum of the even and odd halves of the inverse; each lane stores half of the planes
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int z = 0; z < P; z++) {
            float2 v = x[c][z];
            v.x += __shfl_xor_sync(0xffffffffu, v.x, 1);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, 1);
            const bool mine = (P == 1) ? (s == 0) : ((z < P / 2) == (s == 0));
            if (active && mine) base[c * comp_stride + z * zstride] = v;
        }
}

// Four lanes per column (P >= 4): lane s computes the outputs kz = 4k' + s, k' < P/2,
//   X[4k'+s] = DFT_{P/2}( y )[k'],  y[z'] = sum_{j<2} x[z' + jP/2] W_{2P}^((z' + jP/2) s),
// and contributes W_{2P}^(-z s) IDFT_{P/2}(H_s)[z mod P/2] to every output plane z; the
// four contributions are summed by a two-round shuffle reduce-scatter after which lane s
// owns the planes z with z mod 4 == s.
template <int P, bool BATCH>
__global__ void __launch_bounds__(128) zmul_reg4_kernel(float2* __restrict__ S, KernelView K, int L1, int h, int hp,
                                                         long long comp_stride, long long zstride, float scale,
                                                         const float2* __restrict__ tw, const DevCtl* ctl,
                                                         int skip_retry, long long sim_stride,
                                                         const float* __restrict__ sim_scale) {
    pdl_begin();
    if (BATCH) {  // the single-simulation variant keeps the shorter prologue
        if (ctl) ctl += blockIdx.y;
        S += blockIdx.y * sim_stride;
        if (sim_scale) scale = sim_scale[blockIdx.y];
    }
    if (conv_skip(ctl, skip_retry)) return;
    constexpr int H = P / 2;
    const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s = (int)(gt & 3);
    const long long colg = gt >> 2;
    const bool active = colg < (long long)L1 * h;
    const int ky = active ? (int)(colg / h) : 0;
    const int kx = active ? (int)(colg % h) : 0;
    float2* base = S + (long long)ky * hp + kx;
    // W_{2P}^m, m < 2P, in shared memory (the lane-dependent twiddles below)
    __shared__ float2 wz[2 * P];
    for (int m = threadIdx.x; m < 2 * P; m += blockDim.x) wz[m] = wtab<-1>(tw, m, 2 * P);
    __syncthreads();
    float2 g[3][H];
    // forward: fold the P input planes onto P/2 with the lane's twiddles
#pragma unroll
    for (int zp = 0; zp < H; zp++) {
        const float2 w0 = wz[(zp * s) & (2 * P - 1)];
        const float2 w1 = wz[((zp + H) * s) & (2 * P - 1)];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 a = active ? base[c * comp_stride + zp * zstride] : make_float2(0.f, 0.f);
            const float2 b = active ? base[c * comp_stride + (zp + H) * zstride] : make_float2(0.f, 0.f);
            g[c][zp] = cadd(cmul(a, w0), cmul(b, w1));
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) RDft<H, -1>::run(g[c]);
    const int kyy = (ky > (K.L1 >> 1)) ? K.L1 - ky : ky;
    const float sy = (ky > (K.L1 >> 1)) ? -1.f : 1.f;
    const int cs = K.kd0 * K.kd1 * K.kd2;
#pragma unroll
    for (int k = 0; k < H; k++) {
        int kz = 4 * k + s;
        float sz = 1.f;
        if (kz > P) { kz = 2 * P - kz; sz = -1.f; }
        const int idx = (kz * K.kd1 + kyy) * K.kd2 + kx;
        const float kxx = __ldg(K.k + idx);
        const float kyy_ = __ldg(K.k + cs + idx);
        const float kzz = __ldg(K.k + 2 * cs + idx);
        const float kyz = K.nz[3] ? sy * __ldg(K.k + 3 * cs + idx) : 0.f;
        const float kxz = K.nz[4] ? sz * __ldg(K.k + 4 * cs + idx) : 0.f;
        const float kxy = K.nz[5] ? sz * sy * __ldg(K.k + 5 * cs + idx) : 0.f;
        const float2 m0 = g[0][k], m1 = g[1][k], m2 = g[2][k];
        g[0][k] = make_float2(scale * (kxx * m0.x + kxy * m1.x + kxz * m2.x), scale * (kxx * m0.y + kxy * m1.y + kxz * m2.y));
        g[1][k] = make_float2(scale * (kxy * m0.x + kyy_ * m1.x + kyz * m2.x), scale * (kxy * m0.y + kyy_ * m1.y + kyz * m2.y));
        g[2][k] = make_float2(scale * (kxz * m0.x + kyz * m1.x + kzz * m2.x), scale * (kxz * m0.y + kyz * m1.y + kzz * m2.y));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) RDft<H, +1>::run(g[c]);
    // reduce-scatter.  Round A (lane ^ 2): keep the planes with bit 1 of z equal to bit 1
    // of s; round B (lane ^ 1): keep bit 0 of z equal to bit 0 of s.
    const int b1 = (s >> 1) & 1, b0 = s & 1;
    float2 a[3][H];  // a[c][i]: partial sum for plane z = zA(i)
#pragma unroll
    for (int i = 0; i < H; i++) {
        // the i-th plane kept after round A and the one sent: same position with bit 1 toggled
        // (register indices chosen by select, so that g stays in registers)
        const int z0 = ((i >> 1) << 2) | (i & 1);  // bit 1 clear
        const int z1 = z0 | 2;                     // bit 1 set
        const int zk = b1 ? z1 : z0;
        const int zs = b1 ? z0 : z1;
        const float2 wkf = wz[(zk * s) & (2 * P - 1)], wsf = wz[(zs * s) & (2 * P - 1)];
        const float2 wk = make_float2(wkf.x, -wkf.y), ws = make_float2(wsf.x, -wsf.y);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 g0 = g[c][z0 & (H - 1)], g1 = g[c][z1 & (H - 1)];
            const float2 keep = cmul(wk, b1 ? g1 : g0);
            const float2 send = cmul(ws, b1 ? g0 : g1);
            float2 recv;
            recv.x = __shfl_xor_sync(0xffffffffu, send.x, 2);
            recv.y = __shfl_xor_sync(0xffffffffu, send.y, 2);
            a[c][i] = cadd(keep, recv);
        }
    }
    // round B: among the kept planes (index i, bit 0 of i = bit 0 of z), keep bit0(z) == b0
#pragma unroll
    for (int i2 = 0; i2 < H / 2; i2++) {
        const int z = (i2 << 2) | (b1 << 1) | b0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 a0 = a[c][2 * i2], a1 = a[c][2 * i2 + 1];
            const float2 send = b0 ? a0 : a1;
            float2 recv;
            recv.x = __shfl_xor_sync(0xffffffffu, send.x, 1);
            recv.y = __shfl_xor_sync(0xffffffffu, send.y, 1);
            const float2 v = cadd(b0 ? a1 : a0, recv);
            if (active) base[c * comp_stride + z * zstride] = v;
        }
    }
}

template <int P>
static cudaError_t launch_zmul_reg_t(float2* S, const KernelView& K, int L1, int h, int hp, long long comp_stride,
                                     long long zstride, float scale, const float2* tw, const DevCtl* ctl,
                                     int skip_retry, cudaStream_t st, int nsim, long long sim_stride,
                                     const float* sim_scale) {
    const long long threads = 2LL * L1 * h;
    const dim3 grid((unsigned)((threads + 127) / 128), (unsigned)nsim);
    if (nsim > 1)
        return launch_pdl(zmul_reg_kernel<P, true>, grid, dim3(128), 0, st, S, K, L1, h, hp, comp_stride, zstride,
                          scale, tw, ctl, skip_retry, sim_stride, sim_scale);
    return launch_pdl(zmul_reg_kernel<P, false>, grid, dim3(128), 0, st, S, K, L1, h, hp, comp_stride, zstride, scale,
                      tw, ctl, skip_retry, sim_stride, sim_scale);
}

template <int P>
static cudaError_t launch_zmul_reg4_t(float2* S, const KernelView& K, int L1, int h, int hp, long long comp_stride,
                                      long long zstride, float scale, const float2* tw, const DevCtl* ctl,
                                      int skip_retry, cudaStream_t st, int nsim, long long sim_stride,
                                      const float* sim_scale) {
    const long long threads = 4LL * L1 * h;
    const dim3 grid((unsigned)((threads + 127) / 128), (unsigned)nsim);
    if (nsim > 1)
        return launch_pdl(zmul_reg4_kernel<P, true>, grid, dim3(128), 0, st, S, K, L1, h, hp, comp_stride, zstride,
                          scale, tw, ctl, skip_retry, sim_stride, sim_scale);
    return launch_pdl(zmul_reg4_kernel<P, false>, grid, dim3(128), 0, st, S, K, L1, h, hp, comp_stride, zstride, scale,
                      tw, ctl, skip_retry, sim_stride, sim_scale);
}

// P = N0 = L0/2 (zero-padded z); returns cudaErrorNotSupported for other shapes
cudaError_t launch_zmul_reg(int P, float2* S, const KernelView& K, int L1, int h, int hp, long long comp_stride,
                            long long zstride, float scale, const float2* tw, const DevCtl* ctl, int skip_retry,
                            cudaStream_t st, int nsim, long long sim_stride, const float* sim_scale) {
    switch (P) {
#define X(p, f) case p: return f<p>(S, K, L1, h, hp, comp_stride, zstride, scale, tw, ctl, skip_retry, st, nsim, sim_stride, sim_scale);
        // two lanes per column up to P = 8 (measured: P = 4, 128x128x4 ensemble class
        // 1073 -> 1012 us; P = 8, 8x128x128 film 11.8 -> 11.0 us), four at P = 16
        X(1, launch_zmul_reg_t) X(2, launch_zmul_reg_t) X(4, launch_zmul_reg_t) X(8, launch_zmul_reg_t)
        X(16, launch_zmul_reg4_t)
#undef X
        default: return cudaErrorNotSupported;
    }
}

// ---------------------------------------------------------------- four-step kernels (L <= 1024)
// Column tile of the four-step column pass: 256 threads per block, at most 48 KB.
__host__ __device__ constexpr int col4_tile(int L) {
    int tc = 256 / fs_p2(L);
    if (tc > 32) tc = 32;
    while (tc > 1 && tc * (L / fs_p2(L)) * (fs_p2(L) + 1) * 8 > 48 * 1024) tc /= 2;
    return tc;
}

// Per-column stride of the exchange buffers: a half-warp holds HW = min(TC, 16) columns
// and 16/HW consecutive t, so a stride congruent to 16/HW (mod 16) puts every
// (column, t) pair of a half-warp on its own pair of banks.
template <int L>
__host__ __device__ constexpr int col4_stride(int tc) {
    const int hw = tc < 16 ? tc : 16;
    const int want = (16 / hw) & 15;
    int s = FS<L>::LBUF;
    while ((s & 15) != want) s++;
    return s;
}

// Tile variants picked by the plan's autotuner: shift -1, 0, +1 halves, keeps or doubles
// the default columns (column pass) or rows (row pass) per block.  A variant that breaks a
// limit of the kernel (threads per block, shared memory, the lane-pair shuffle of the
// length-512 column transform) falls back to the default.
static int shifted(int base, int shift) { return shift > 0 ? base << shift : (shift < 0 ? base >> (-shift) : base); }

template <int L, int SIGN>
__global__ void __launch_bounds__(512) colfft4_kernel(float2* __restrict__ S, int ncols, long long outer_stride,
                                                      long long line_stride, int n_in, int n_out,
                                                      const float2* __restrict__ tw, const DevCtl* ctl,
                                                      int skip_retry, long long sim_stride, int TC, int cstride) {
    pdl_begin();
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    using F = FS<L>;
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int col = threadIdx.x % TC, t = threadIdx.x / TC;
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    const bool active = (t < F::P2) && (kx0 + col < ncols);
    float2* base = S + (long long)o * outer_stride + kx0 + col;
    float2* twt = sm + TC * cstride;
    F::fill_twiddles(twt, tw);
    float2 v[F::P1];
#pragma unroll
    for (int j = 0; j < F::P1; j++) {
        const int n = F::in_index(t, j);
        v[j] = (active && n < n_in) ? base[n * line_stride] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    F::template run<SIGN>(v, sm + col * cstride, t, active, twt, TC);
#pragma unroll
    for (int r = 0; r < F::P1; r++) {
        const int n = F::out_index(t, r);
        if (active && n < n_out) base[n * line_stride] = v[r];
    }
}

// R2C rows (zero-padded to 2M reals) with the four-step transform of the packed
// sequence z[n] = x[2n] + i x[2n+1], then the real-to-complex post-processing.
template <int M>
__global__ void __launch_bounds__(512) xfwd4_kernel(const float* __restrict__ in_fixed, PP in_pp,
                                                    const float* __restrict__ mask, float2* __restrict__ out,
                                                    int nrows, int Z, int Y, int Yout, int in_pitch, int n_in, int hp,
                                                    const float2* __restrict__ tw, const DevCtl* ctl, int skip_retry,
                                                    long long in_bstride, long long out_bstride,
                                                    long long mask_bstride, int RPB) {
    pdl_begin();
    const int sim = blockIdx.y;
    if (ctl) ctl += sim;
    if (conv_skip(ctl, skip_retry)) return;
    using F = FS<M>;
    const float* in = (in_fixed ? in_fixed : in_pp.get(ctl ? ctl->cur : 0)) + sim * in_bstride;
    out += sim * out_bstride;
    if (mask) mask += sim * mask_bstride;
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int t = threadIdx.x % F::P2, lr = threadIdx.x / F::P2;
    const int row = blockIdx.x * RPB + lr;
    const bool active = (lr < RPB) && (row < nrows);
    float2* buf = sm + (lr < RPB ? lr : 0) * F::LBUF;
    float2* twt = sm + RPB * F::LBUF;
    F::fill_twiddles(twt, tw);
    float2 v[F::P1];
    const float* src = in + (long long)(active ? row : 0) * in_pitch;
    const int zy = (active ? row : 0) % (Z * Y);
    const float* msk = mask ? mask + (long long)zy * in_pitch : nullptr;
    const bool pairs = ((in_pitch & 1) == 0);
#pragma unroll
    for (int j = 0; j < F::P1; j++) {
        const int n = F::in_index(t, j);
        float a = 0.f, b = 0.f;
        if (active) {
            if (pairs && 2 * n + 1 < n_in) {
                float2 ab = __ldg(reinterpret_cast<const float2*>(src) + n);
                if (msk) {
                    const float2 mm = __ldg(reinterpret_cast<const float2*>(msk) + n);
                    ab.x *= mm.x;
                    ab.y *= mm.y;
                }
                a = ab.x;
                b = ab.y;
            } else {
                if (2 * n < n_in) a = src[2 * n] * (msk ? msk[2 * n] : 1.f);
                if (2 * n + 1 < n_in) b = src[2 * n + 1] * (msk ? msk[2 * n + 1] : 1.f);
            }
        }
        v[j] = make_float2(a, b);
    }
    __syncthreads();
    F::template run<-1>(v, buf, t, active, twt, 1);
    if (active) {
#pragma unroll
        for (int r = 0; r < F::P1; r++) buf[F::out_index(t, r)] = v[r];
    }
    __syncthreads();
    if (active) {
        const int c = row / (Z * Y);
        const int z = zy / Y, y = zy % Y;
        float2* dst = out + ((long long)(c * Z + z) * Yout + y) * hp;
        for (int k = t; k <= M / 2; k += F::P2) {
            const float2 zk = buf[k & (M - 1)];
            const float2 zm = buf[(M - k) & (M - 1)];
            const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 od = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));  // (Z[k] - conj Z[M-k]) / 2i
            const float2 w = TwSrc<-1, float2>::get(tw, k, 2 * M);
            dst[k] = cadd(e, cmul(w, od));
            if (k != M - k) dst[M - k] = cadd(cconj(e), cmul(make_float2(-w.x, w.y), cconj(od)));
        }
    }
}

// Column pass of single-layer films (lines along y, kz = 0) with the four-step
// transform: the three components of TC columns are loaded straight into registers
// (3 x TC x P2 threads, rows n >= n_in are the zero padding and are not read), transformed,
// put in natural order in shared memory, multiplied by the symmetric kernel there (all
// three components of a (ky, kx) point meet in one thread), taken back into registers
// and inverse-transformed; only the rows n < n_in are stored.  Replaces the Stockham
// colmul_kernel for 2-D films (seven barrier-separated stages per transform and
// component there, two barriers per transform here).
template <int L, int TC>
__global__ void __launch_bounds__(384) colmul4_kernel(float2* __restrict__ S, KernelView K, int ncols,
                                                      long long comp_stride, long long line_stride, int n_in,
                                                      float scale, const float2* __restrict__ tw, const DevCtl* ctl,
                                                      int skip_retry, long long sim_stride,
                                                      const float* __restrict__ sim_scale, int cstride) {
    pdl_begin();
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    if (sim_scale) scale = sim_scale[blockIdx.y];
    using F = FS<L>;
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int per = TC * F::P2;                    // threads per component
    const int c = threadIdx.x / per, r = threadIdx.x - c * per;
    const int col = r % TC, t = r / TC;
    const int kx0 = blockIdx.x * TC;
    const bool active = c < 3 && kx0 + col < ncols;
    float2* line = sm + ((c < 3 ? c : 0) * TC + col) * cstride;
    float2* twt = sm + 3 * TC * cstride;
    F::fill_twiddles(twt, tw);
    float2* base = S + (long long)(c < 3 ? c : 0) * comp_stride + kx0 + col;
    float2 v[F::P1];
#pragma unroll
    for (int j = 0; j < F::P1; j++) {
        const int n = F::in_index(t, j);
        v[j] = (active && n < n_in) ? base[n * line_stride] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    F::template run<-1>(v, line, t, active, twt, TC);
    if (active) {
#pragma unroll
        for (int q = 0; q < F::P1; q++) line[F::out_index(t, q)] = v[q];
    }
    __syncthreads();
    // symmetric kernel multiply at every (ky, kx) of the tile
    const int nh = min(TC, ncols - kx0);
    for (int e = threadIdx.x; e < L * TC; e += blockDim.x) {
        const int ky = e / TC, c2 = e - ky * TC;
        if (c2 >= nh) continue;
        float kk[6];
        kernel_at(K, 0, ky, kx0 + c2, kk);
        float2* l0 = sm + (0 * TC + c2) * cstride + ky;
        float2* l1 = sm + (1 * TC + c2) * cstride + ky;
        float2* l2 = sm + (2 * TC + c2) * cstride + ky;
        const float2 m0 = *l0, m1 = *l1, m2 = *l2;
        // q: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy
        *l0 = make_float2(scale * (kk[0] * m0.x + kk[5] * m1.x + kk[4] * m2.x),
                          scale * (kk[0] * m0.y + kk[5] * m1.y + kk[4] * m2.y));
        *l1 = make_float2(scale * (kk[5] * m0.x + kk[1] * m1.x + kk[3] * m2.x),
                          scale * (kk[5] * m0.y + kk[1] * m1.y + kk[3] * m2.y));
        *l2 = make_float2(scale * (kk[4] * m0.x + kk[3] * m1.x + kk[2] * m2.x),
                          scale * (kk[4] * m0.y + kk[3] * m1.y + kk[2] * m2.y));
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int j = 0; j < F::P1; j++) v[j] = line[F::in_index(t, j)];
    }
    __syncthreads();
    F::template run<+1>(v, line, t, active, twt, TC);
#pragma unroll
    for (int q = 0; q < F::P1; q++) {
        const int n = F::out_index(t, q);
        if (active && n < n_in) base[n * line_stride] = v[q];
    }
}

// ---------------------------------------------------------------- launch helpers
template <typename KT> static cudaError_t set_smem(KT kern, size_t bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

#define MM_FOR_POW2(X) X(1) X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)

#define XFWD_SIM_ARGS int nsim, long long in_bstride, long long out_bstride, long long mask_bstride
#define XFWD_SIM_PASS nsim, in_bstride, out_bstride, mask_bstride

template <int M, typename V, typename S>
static cudaError_t launch_xfwd_t(const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                                 int in_pitch, int n_in, int hp, const float2* tw, const DevCtl* ctl, int skip_retry,
                                 cudaStream_t st, XFWD_SIM_ARGS) {
    constexpr int TPL = tpl(M);
    constexpr int RPB = TPL >= 256 ? 1 : 256 / TPL;
    const size_t smem = (size_t)RPB * line_len(M) * sizeof(V);
    cudaError_t e = set_smem(xfwd_kernel<M, V, S>, smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((nrows + RPB - 1) / RPB), (unsigned)nsim);
    int threads = RPB * TPL < 32 ? 32 : RPB * TPL;
    xfwd_kernel<M, V, S><<<grid, threads, smem, st>>>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp,
                                                      tw, ctl, skip_retry, in_bstride, out_bstride, mask_bstride);
    return cudaGetLastError();
}

template <int M>
static cudaError_t launch_xfwd4_t(const float* in, PP pp, const float* mask, float2* out, int nrows, int Z, int Y,
                                  int Yout, int in_pitch, int n_in, int hp, const float2* tw, const DevCtl* ctl,
                                  int skip_retry, cudaStream_t st, XFWD_SIM_ARGS, int tile) {
    using F = FS<M>;
    constexpr int RPB0 = (256 / F::P2) > 0 ? 256 / F::P2 : 1;
    auto smem_of = [](int r) { return (size_t)(r * F::LBUF + F::TWT) * sizeof(float2); };
    int RPB = shifted(RPB0, tile);
    if (RPB < 1 || RPB * F::P2 > 512 || RPB * F::P2 < 32 || smem_of(RPB) > 200 * 1024) RPB = RPB0;
    const size_t smem = smem_of(RPB);
    cudaError_t e = set_smem(xfwd4_kernel<M>, smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((nrows + RPB - 1) / RPB), (unsigned)nsim);
    return launch_pdl(xfwd4_kernel<M>, grid, dim3(RPB * F::P2), smem, st, in, pp, mask, out, nrows, Z, Y, Yout, in_pitch,
                      n_in, hp, tw, ctl, skip_retry, in_bstride, out_bstride, mask_bstride, RPB);
}

template <typename V, typename S>
cudaError_t launch_xfwd(int M, const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                        int in_pitch, int n_in, int hp, const float2* tw, const DevCtl* ctl, int skip_retry,
                        cudaStream_t st, XFWD_SIM_ARGS, int tile) {
    if constexpr (sizeof(V) == 8) {
        switch (M) {
#define X(m) case m: return launch_xfwd4_t<m>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, tw, ctl, skip_retry, st, XFWD_SIM_PASS, tile);
            X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
            default: break;
        }
    }
    switch (M) {
#define X(m) case m: return launch_xfwd_t<m, V, S>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, tw, ctl, skip_retry, st, XFWD_SIM_PASS);
        MM_FOR_POW2(X)
#undef X
        default:  // not a power of two: the mixed-radix pass (mixed.cu)
            return launch_mr_xfwd<V, S>(M, in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, ctl, skip_retry,
                                        st, XFWD_SIM_PASS);
    }
}

template <int L, int SIGN, typename V>
static cudaError_t launch_colfft_t(V* S, int ncols, int nouter, long long outer_stride, long long line_stride,
                                   int n_in, int n_out, const float2* tw, const DevCtl* ctl, int skip_retry,
                                   cudaStream_t st, int nsim, long long sim_stride) {
    constexpr int TC = col_tile(L, 1, sizeof(V));
    const size_t smem = (size_t)TC * line_len(L) * sizeof(V);
    cudaError_t e = set_smem(colfft_kernel<L, SIGN, V>, smem);
    if (e != cudaSuccess) return e;
    int ntiles = (ncols + TC - 1) / TC;
    int threads = TC * tpl(L);
    if (threads < 32) threads = 32;
    colfft_kernel<L, SIGN, V><<<dim3((unsigned)(nouter * ntiles), (unsigned)nsim), threads, smem, st>>>(
        S, ncols, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, sim_stride);
    return cudaGetLastError();
}

template <int L, int SIGN>
static cudaError_t launch_colfft4_t(float2* S, int ncols, int nouter, long long outer_stride, long long line_stride,
                                    int n_in, int n_out, const float2* tw, const DevCtl* ctl, int skip_retry,
                                    cudaStream_t st, int nsim, long long sim_stride, int tile) {
    using F = FS<L>;
    int TC = shifted(col4_tile(L), tile);
    auto smem_of = [](int tc) { return (size_t)(tc * col4_stride<L>(tc) + F::TWT) * sizeof(float2); };
    if (TC < 1 || TC > 16 || TC * F::P2 > 512 || smem_of(TC) > 200 * 1024) TC = col4_tile(L);
    const size_t smem = smem_of(TC);
    cudaError_t e = set_smem(colfft4_kernel<L, SIGN>, smem);
    if (e != cudaSuccess) return e;
    const int ntiles = (ncols + TC - 1) / TC;
    int threads = TC * F::P2;
    if (threads < 32) threads = 32;
    return launch_pdl(colfft4_kernel<L, SIGN>, dim3((unsigned)(nouter * ntiles), (unsigned)nsim), dim3(threads), smem, st,
                      S, ncols, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, sim_stride, TC,
                      col4_stride<L>(TC));
}

template <typename V>
cudaError_t launch_colfft(int L, int sign, V* S, int ncols, int nouter, long long outer_stride,
                          long long line_stride, int n_in, int n_out, const float2* tw, const DevCtl* ctl,
                          int skip_retry, cudaStream_t st, int nsim, long long sim_stride, int tile) {
    if constexpr (sizeof(V) == 8) {
        if (sign < 0) {
            switch (L) {
#define X(l) case l: return launch_colfft4_t<l, -1>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, st, nsim, sim_stride, tile);
                X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
                default: break;
            }
        } else {
            switch (L) {
#define X(l) case l: return launch_colfft4_t<l, 1>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, st, nsim, sim_stride, tile);
                X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
                default: break;
            }
        }
    }
    if (sign < 0) {
        switch (L) {
#define X(l) case l: return launch_colfft_t<l, -1, V>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, st, nsim, sim_stride);
            MM_FOR_POW2(X)
#undef X
            default:
                return launch_mr_colfft<V>(L, -1, S, ncols, nouter, outer_stride, line_stride, n_in, n_out, ctl,
                                           skip_retry, st, nsim, sim_stride);
        }
    } else {
        switch (L) {
#define X(l) case l: return launch_colfft_t<l, 1, V>(S, ncols, nouter, outer_stride, line_stride, n_in, n_out, tw, ctl, skip_retry, st, nsim, sim_stride);
            MM_FOR_POW2(X)
#undef X
            default:
                return launch_mr_colfft<V>(L, 1, S, ncols, nouter, outer_stride, line_stride, n_in, n_out, ctl,
                                           skip_retry, st, nsim, sim_stride);
        }
    }
}

template <int L>
static cudaError_t launch_colmul_t(float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                                   long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                                   const float2* tw, const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim,
                                   long long sim_stride, const float* sim_scale) {
    constexpr int TC = col_tile(L, 3, 8);
    const size_t smem = (size_t)3 * TC * line_len(L) * sizeof(float2);
    cudaError_t e = set_smem(colmul_kernel<L>, smem);
    if (e != cudaSuccess) return e;
    int ntiles = (ncols + TC - 1) / TC;
    int threads = TC * tpl(L);
    if (threads < 32) threads = 32;
    colmul_kernel<L><<<dim3((unsigned)(nouter * ntiles), (unsigned)nsim), threads, smem, st>>>(
        S, K, ncols, comp_stride, outer_stride, line_stride, n_in, kaxis, scale, tw, ctl, skip_retry, sim_stride,
        sim_scale);
    return cudaGetLastError();
}

// columns per block: 64 / P2 (192 threads) by default, halved or doubled by the tile
template <int L, int SHIFT>
__host__ __device__ constexpr int colmul4_tc() {
    constexpr int t0 = (64 / FS<L>::P2) > 0 ? 64 / FS<L>::P2 : 1;
    constexpr int t = SHIFT > 0 ? t0 * 2 : (SHIFT < 0 ? t0 / 2 : t0);
    return (t < 1 || t > 32 || 3 * t * FS<L>::P2 > 384) ? (t0 > 32 ? 32 : t0) : t;
}

template <int L, int SHIFT>
static cudaError_t launch_colmul4_s(float2* S, const KernelView& K, int ncols, long long comp_stride,
                                    long long line_stride, int n_in, float scale, const float2* tw,
                                    const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim,
                                    long long sim_stride, const float* sim_scale) {
    using F = FS<L>;
    constexpr int TC = colmul4_tc<L, SHIFT>();
    const int cstride = col4_stride<L>(TC < 16 ? TC : 16) > F::LBUF ? col4_stride<L>(TC < 16 ? TC : 16) : F::LBUF;
    const size_t smem = (size_t)(3 * TC * cstride + F::TWT) * sizeof(float2);
    cudaError_t e = set_smem(colmul4_kernel<L, TC>, smem);
    if (e != cudaSuccess) return e;
    int threads = 3 * TC * F::P2;
    if (threads < 32) threads = 32;
    const int ntiles = (ncols + TC - 1) / TC;
    return launch_pdl(colmul4_kernel<L, TC>, dim3((unsigned)ntiles, (unsigned)nsim), dim3(threads), smem, st, S, K, ncols,
                      comp_stride, line_stride, n_in, scale, tw, ctl, skip_retry, sim_stride, sim_scale, cstride);
}

template <int L>
static cudaError_t launch_colmul4_t(float2* S, const KernelView& K, int ncols, long long comp_stride,
                                    long long line_stride, int n_in, float scale, const float2* tw,
                                    const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim,
                                    long long sim_stride, const float* sim_scale, int tile) {
    if (tile < 0)
        return launch_colmul4_s<L, -1>(S, K, ncols, comp_stride, line_stride, n_in, scale, tw, ctl, skip_retry, st,
                                       nsim, sim_stride, sim_scale);
    if (tile > 0)
        return launch_colmul4_s<L, 1>(S, K, ncols, comp_stride, line_stride, n_in, scale, tw, ctl, skip_retry, st,
                                      nsim, sim_stride, sim_scale);
    return launch_colmul4_s<L, 0>(S, K, ncols, comp_stride, line_stride, n_in, scale, tw, ctl, skip_retry, st, nsim,
                                  sim_stride, sim_scale);
}

cudaError_t launch_colmul(int L, float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                          long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                          const float2* tw, const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim,
                          long long sim_stride, const float* sim_scale, int tile) {
    if (kaxis == 1 && nouter == 1 && L >= 4 && L <= 1024) {
        // single-layer films: the four-step column pass
        switch (L) {
#define X(l) case l: return launch_colmul4_t<l>(S, K, ncols, comp_stride, line_stride, n_in, scale, tw, ctl, skip_retry, st, nsim, sim_stride, sim_scale, tile);
            X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
            default: break;
        }
    }
    switch (L) {
#define X(l) case l: return launch_colmul_t<l>(S, K, ncols, nouter, comp_stride, outer_stride, line_stride, n_in, kaxis, scale, tw, ctl, skip_retry, st, nsim, sim_stride, sim_scale);
        MM_FOR_POW2(X)
#undef X
        default:
            return launch_mr_colmul(L, S, K, ncols, nouter, comp_stride, outer_stride, line_stride, n_in, kaxis, scale,
                                    ctl, skip_retry, st, nsim, sim_stride, sim_scale);
    }
}

template cudaError_t launch_xfwd<float2, float>(int, const float*, PP, const float*, float2*, int, int, int, int, int,
                                                int, int, const float2*, const DevCtl*, int, cudaStream_t, int,
                                                long long, long long, long long, int);
template cudaError_t launch_xfwd<double2, double>(int, const double*, PP, const float*, double2*, int, int, int, int,
                                                  int, int, int, const float2*, const DevCtl*, int, cudaStream_t, int,
                                                  long long, long long, long long, int);
template cudaError_t launch_colfft<float2>(int, int, float2*, int, int, long long, long long, int, int,
                                           const float2*, const DevCtl*, int, cudaStream_t, int, long long, int);
template cudaError_t launch_colfft<double2>(int, int, double2*, int, int, long long, long long, int, int,
                                            const float2*, const DevCtl*, int, cudaStream_t, int, long long, int);

}  // namespace mm
