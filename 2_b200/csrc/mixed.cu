// mixed.cu -- the convolution passes for transform lengths that are not powers of two.
//
// Same passes, spectrum layout and arithmetic as the power-of-two kernels of conv.cu
// (R2C rows by the packed half-length transform, column transforms of the non-zero
// rows only, the symmetric 3x3 kernel multiply between forward and inverse), with the
// transform itself done by the mixed-radix shared-memory routine of mixed.cuh.  Used
// for padded sizes such as 2^n * {3, 5, 7} (engine/gridsize.go:16-33), which the
// reference convolves through cuFFT (fftplanX.go:59-64).  The C2R + epilogue pass of
// these lengths is in rhs.cu (mr_xinv_epi_kernel).
#include <cmath>
#include <mutex>
#include <vector>

#include "kernel_view.cuh"
#include "mixed.cuh"
#include "mm_internal.h"

namespace mm {
using namespace mmfft;

// ---------------------------------------------------------------- host: factors, tables
bool mr_factor(int L, MrLine* f) {
    if (L < 1 || L > MR_MAXL) return false;
    f->L = L;
    f->nst = 0;
    int n = L;
    while (n % 8 == 0 && f->nst < MR_MAXST) { f->r[f->nst++] = 8; n /= 8; }
    if (n % 4 == 0 && f->nst < MR_MAXST) { f->r[f->nst++] = 4; n /= 4; }
    if (n % 2 == 0 && f->nst < MR_MAXST) { f->r[f->nst++] = 2; n /= 2; }
    for (int p = 3; p <= MR_MAXR && n > 1; p += 2) {
        while (n % p == 0 && f->nst < MR_MAXST) { f->r[f->nst++] = p; n /= p; }
    }
    return n == 1;
}

namespace {
struct MrEntry {
    int dev, L;
    float2* f;
    double2* d;
};
std::mutex g_mr_mu;
std::vector<MrEntry> g_mr;  // kept until the process exits (a few KB per length)
}  // namespace

int mr_prepare(int L) {
    MrLine f;
    if (!mr_factor(L, &f)) return MM_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MM_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mr_mu);
    for (const MrEntry& e : g_mr)
        if (e.dev == dev && e.L == L) return MM_OK;
    std::vector<float2> hf(L);
    std::vector<double2> hd(L);
    const double two_pi = 6.283185307179586476925286766559;
    for (int t = 0; t < L; t++) {
        // exp(-2 pi i t / L) in FP64, the angle reduced to [-pi, pi] first
        const int tr = (2 * t > L) ? t - L : t;
        const double a = -two_pi * (double)tr / (double)L;
        hd[t] = make_double2(std::cos(a), std::sin(a));
        hf[t] = make_float2((float)hd[t].x, (float)hd[t].y);
    }
    MrEntry e{dev, L, nullptr, nullptr};
    if (cudaMalloc(&e.f, sizeof(float2) * L) != cudaSuccess) return MM_ERR_CUDA;
    if (cudaMalloc(&e.d, sizeof(double2) * L) != cudaSuccess) {
        cudaFree(e.f);
        return MM_ERR_CUDA;
    }
    if (cudaMemcpy(e.f, hf.data(), sizeof(float2) * L, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(e.d, hd.data(), sizeof(double2) * L, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(e.f);
        cudaFree(e.d);
        return MM_ERR_CUDA;
    }
    g_mr.push_back(e);
    return MM_OK;
}

bool mr_tables(int L, const float2** tf, const double2** td) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lk(g_mr_mu);
    for (const MrEntry& e : g_mr)
        if (e.dev == dev && e.L == L) {
            if (tf) *tf = e.f;
            if (td) *td = e.d;
            return true;
        }
    return false;
}

template <typename V> static const V* pick_table(const float2* f, const double2* d);
template <> const float2* pick_table<float2>(const float2* f, const double2*) { return f; }
template <> const double2* pick_table<double2>(const float2*, const double2* d) { return d; }

template <typename V> static bool table_of(int L, const V** out) {
    const float2* f = nullptr;
    const double2* d = nullptr;
    if (!mr_tables(L, &f, &d)) return false;
    *out = pick_table<V>(f, d);
    return true;
}

template <typename KT> static cudaError_t mr_smem(KT kern, size_t bytes) {
    if (bytes > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

// ---------------------------------------------------------------- R2C row pass
// As xfwd_kernel: rows r = (c*Z + z)*Y + y of n_in reals (times the mask), zero-padded to
// 2M, packed as z[e] = x[2e] + i x[2e+1], transformed (length M) and post-processed into
// the M+1 columns X[k] = E[k] + W_2M^k O[k] of spectrum row (c, z, y).  rpb rows per block,
// blockDim.x / rpb threads per row.
template <typename V, typename S>
__global__ void __launch_bounds__(256) mr_xfwd_kernel(const S* __restrict__ in_fixed, PP in_pp,
                                                      const float* __restrict__ mask, V* __restrict__ out, int nrows,
                                                      int Z, int Y, int Yout, int in_pitch, int n_in, int hp, MrLine f,
                                                      const V* __restrict__ twM, const V* __restrict__ tw2M,
                                                      const DevCtl* ctl, int skip_retry, long long in_bstride,
                                                      long long out_bstride, long long mask_bstride, int rpb) {
    typedef typename Scalar<V>::T T;
    const int sim = blockIdx.y;
    if (ctl) ctl += sim;
    if (conv_skip(ctl, skip_retry)) return;
    const S* in = (in_fixed ? in_fixed : reinterpret_cast<const S*>(in_pp.get(ctl ? ctl->cur : 0))) + sim * in_bstride;
    out += sim * out_bstride;
    if (mask) mask += sim * mask_bstride;
    const int M = f.L;
    const int nt = blockDim.x / rpb;
    const int lr = threadIdx.x / nt, t = threadIdx.x % nt;
    const int row = blockIdx.x * rpb + lr;
    const bool active = (lr < rpb) && (row < nrows);
    extern __shared__ unsigned char smem_raw[];
    V* a = reinterpret_cast<V*>(smem_raw) + (size_t)(lr < rpb ? lr : 0) * 2 * M;
    V* b = a + M;
    if (active) {
        const S* src = in + (long long)row * in_pitch;
        const int zy = row % (Z * Y);
        const float* msk = mask ? mask + (long long)zy * in_pitch : nullptr;
        for (int e = t; e < M; e += nt) {
            S x0 = 0, x1 = 0;
            if (2 * e < n_in) x0 = src[2 * e] * (msk ? (S)msk[2 * e] : (S)1);
            if (2 * e + 1 < n_in) x1 = src[2 * e + 1] * (msk ? (S)msk[2 * e + 1] : (S)1);
            a[e] = mkv((T)x0, (T)x1);
        }
    }
    mr_fft<-1, V>(a, b, f, twM, t, nt, active);
    if (active) {
        const int c = row / (Z * Y);
        const int zy = row % (Z * Y);
        const int z = zy / Y, y = zy % Y;
        V* dst = out + ((long long)(c * Z + z) * Yout + y) * hp;
        for (int k = t; k <= M / 2; k += nt) {
            const V zk = a[k];
            const V zm = a[(M - k) % M];
            const V e = cscale(cadd(zk, cconj(zm)), (T)0.5);
            V o = cscale(csub(zk, cconj(zm)), (T)0.5);
            o = mkv(o.y, -o.x);  // divide by i
            const V w = tw2M[k];  // exp(-2 pi i k / 2M)
            dst[k] = cadd(e, cmul(w, o));
            if (k != M - k) {
                const V wm = mkv(-w.x, w.y);  // W^(M-k) = -conj W^k
                dst[M - k] = cadd(cconj(e), cmul(wm, cconj(o)));
            }
        }
    }
}

static int mr_row_threads(int M) { return M >= 512 ? 256 : (M >= 128 ? 64 : 32); }

template <typename V, typename S>
cudaError_t launch_mr_xfwd(int M, const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                           int in_pitch, int n_in, int hp, const DevCtl* ctl, int skip_retry, cudaStream_t st,
                           int nsim, long long in_bstride, long long out_bstride, long long mask_bstride) {
    MrLine f;
    const V *twM = nullptr, *tw2M = nullptr;
    if (!mr_factor(M, &f) || !table_of<V>(M, &twM) || !table_of<V>(2 * M, &tw2M)) return cudaErrorInvalidValue;
    const int nt = mr_row_threads(M);
    const int rpb = 256 / nt;
    const size_t smem = (size_t)rpb * 2 * M * sizeof(V);
    cudaError_t e = mr_smem(mr_xfwd_kernel<V, S>, smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((nrows + rpb - 1) / rpb), (unsigned)nsim);
    mr_xfwd_kernel<V, S><<<grid, rpb * nt, smem, st>>>(in, pp, mask, out, nrows, Z, Y, Yout, in_pitch, n_in, hp, f,
                                                       twM, tw2M, ctl, skip_retry, in_bstride, out_bstride,
                                                       mask_bstride, rpb);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- column passes
// Columns per block: up to 16, as many as keep `lines` lines of L elements within 64 KB
// (a single column may take up to 128 KB).
static int mr_cols(int L, int lines_per_col, size_t vsize) {
    int tc = 16;
    while (tc > 1 && (size_t)lines_per_col * tc * L * vsize > 64 * 1024) tc /= 2;
    return tc;
}

// One component per line: block b covers outer index o = b / ntiles and kx tile
// (b % ntiles)*TC; element e of column kx is at base + o*outer_stride + e*line_stride + kx.
// Rows e < n_in are read (the rest zero), rows e < n_out written.
template <int SIGN, typename V>
__global__ void __launch_bounds__(256) mr_colfft_kernel(V* __restrict__ S, int ncols, long long outer_stride,
                                                        long long line_stride, int n_in, int n_out, MrLine f,
                                                        const V* __restrict__ tw, const DevCtl* ctl, int skip_retry,
                                                        long long sim_stride, int TC) {
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    const int L = f.L;
    extern __shared__ unsigned char smem_raw[];
    V* sm = reinterpret_cast<V*>(smem_raw);
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    const int nh = min(TC, ncols - kx0);
    V* base = S + (long long)o * outer_stride + kx0;
    const V zero = mkv((typename Scalar<V>::T)0, (typename Scalar<V>::T)0);
    for (int i = threadIdx.x; i < L * TC; i += blockDim.x) {
        const int e = i / TC, col = i % TC;
        sm[col * L + e] = (e < n_in && col < nh) ? base[e * line_stride + col] : zero;
    }
    const int nt = blockDim.x / TC;
    const int col = threadIdx.x / nt, t = threadIdx.x % nt;
    const bool act = col < TC;
    V* a = sm + (act ? col : 0) * L;
    mr_fft<SIGN, V>(a, a + TC * L, f, tw, t, nt, act);
    for (int i = threadIdx.x; i < n_out * TC; i += blockDim.x) {
        const int e = i / TC, c2 = i % TC;
        if (c2 < nh) base[e * line_stride + c2] = sm[c2 * L + e];
    }
}

template <typename V>
cudaError_t launch_mr_colfft(int L, int sign, V* S, int ncols, int nouter, long long outer_stride,
                             long long line_stride, int n_in, int n_out, const DevCtl* ctl, int skip_retry,
                             cudaStream_t st, int nsim, long long sim_stride) {
    MrLine f;
    const V* tw = nullptr;
    if (!mr_factor(L, &f) || !table_of<V>(L, &tw)) return cudaErrorInvalidValue;
    const int TC = mr_cols(L, 2, sizeof(V));
    const size_t smem = (size_t)2 * TC * L * sizeof(V);
    const int ntiles = (ncols + TC - 1) / TC;
    const dim3 grid((unsigned)(nouter * ntiles), (unsigned)nsim);
    cudaError_t e;
    if (sign < 0) {
        if ((e = mr_smem(mr_colfft_kernel<-1, V>, smem)) != cudaSuccess) return e;
        mr_colfft_kernel<-1, V><<<grid, 256, smem, st>>>(S, ncols, outer_stride, line_stride, n_in, n_out, f, tw, ctl,
                                                         skip_retry, sim_stride, TC);
    } else {
        if ((e = mr_smem(mr_colfft_kernel<1, V>, smem)) != cudaSuccess) return e;
        mr_colfft_kernel<1, V><<<grid, 256, smem, st>>>(S, ncols, outer_stride, line_stride, n_in, n_out, f, tw, ctl,
                                                        skip_retry, sim_stride, TC);
    }
    return cudaGetLastError();
}

// Three components per column: forward transforms, H = sum_s K_sd M_s (symmetric, real
// kernel from the stored octant), inverse transforms; kaxis 0: lines along z (ky = outer
// index), kaxis 1: lines along y (kz = 0, single-layer films).  The three components are
// transformed one after the other through one scratch line per column.
__global__ void __launch_bounds__(256) mr_colmul_kernel(float2* __restrict__ S, KernelView K, int ncols,
                                                        long long comp_stride, long long outer_stride,
                                                        long long line_stride, int n_in, int kaxis, float scale,
                                                        MrLine f, const float2* __restrict__ tw, const DevCtl* ctl,
                                                        int skip_retry, long long sim_stride,
                                                        const float* __restrict__ sim_scale, int TC) {
    if (ctl) ctl += blockIdx.y;
    if (conv_skip(ctl, skip_retry)) return;
    S += blockIdx.y * sim_stride;
    if (sim_scale) scale = sim_scale[blockIdx.y];
    const int L = f.L;
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);  // [3][TC][L] lines, then [TC][L] scratch
    const int ntiles = (ncols + TC - 1) / TC;
    const int o = blockIdx.x / ntiles;
    const int kx0 = (blockIdx.x % ntiles) * TC;
    const int nh = min(TC, ncols - kx0);
    float2* base = S + (long long)o * outer_stride + kx0;
    for (int c = 0; c < 3; c++)
        for (int i = threadIdx.x; i < L * TC; i += blockDim.x) {
            const int e = i / TC, col = i % TC;
            sm[(c * TC + col) * L + e] =
                (e < n_in && col < nh) ? base[c * comp_stride + e * line_stride + col] : make_float2(0.f, 0.f);
        }
    const int nt = blockDim.x / TC;
    const int col = threadIdx.x / nt, t = threadIdx.x % nt;
    const bool act = col < TC;
    const int cc = act ? col : 0;
    float2* scratch = sm + (3 * TC + cc) * L;
    for (int c = 0; c < 3; c++) mr_fft<-1, float2>(sm + (c * TC + cc) * L, scratch, f, tw, t, nt, act);
    for (int i = threadIdx.x; i < L * TC; i += blockDim.x) {
        const int e = i / TC, c2 = i % TC;
        if (c2 >= nh) continue;
        const int kx = kx0 + c2;
        float kk[6];
        if (kaxis == 0) kernel_at(K, e, o, kx, kk);
        else kernel_at(K, 0, e, kx, kk);
        const float2 m0 = sm[(0 * TC + c2) * L + e];
        const float2 m1 = sm[(1 * TC + c2) * L + e];
        const float2 m2 = sm[(2 * TC + c2) * L + e];
        // q: 0 xx, 1 yy, 2 zz, 3 yz, 4 xz, 5 xy
        sm[(0 * TC + c2) * L + e] = make_float2(scale * (kk[0] * m0.x + kk[5] * m1.x + kk[4] * m2.x),
                                                scale * (kk[0] * m0.y + kk[5] * m1.y + kk[4] * m2.y));
        sm[(1 * TC + c2) * L + e] = make_float2(scale * (kk[5] * m0.x + kk[1] * m1.x + kk[3] * m2.x),
                                                scale * (kk[5] * m0.y + kk[1] * m1.y + kk[3] * m2.y));
        sm[(2 * TC + c2) * L + e] = make_float2(scale * (kk[4] * m0.x + kk[3] * m1.x + kk[2] * m2.x),
                                                scale * (kk[4] * m0.y + kk[3] * m1.y + kk[2] * m2.y));
    }
    for (int c = 0; c < 3; c++) mr_fft<+1, float2>(sm + (c * TC + cc) * L, scratch, f, tw, t, nt, act);
    for (int c = 0; c < 3; c++)
        for (int i = threadIdx.x; i < n_in * TC; i += blockDim.x) {
            const int e = i / TC, c2 = i % TC;
            if (c2 < nh) base[c * comp_stride + e * line_stride + c2] = sm[(c * TC + c2) * L + e];
        }
}

cudaError_t launch_mr_colmul(int L, float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                             long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                             const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim, long long sim_stride,
                             const float* sim_scale) {
    MrLine f;
    const float2* tw = nullptr;
    if (!mr_factor(L, &f) || !table_of<float2>(L, &tw)) return cudaErrorInvalidValue;
    const int TC = mr_cols(L, 4, sizeof(float2));
    const size_t smem = (size_t)4 * TC * L * sizeof(float2);
    cudaError_t e = mr_smem(mr_colmul_kernel, smem);
    if (e != cudaSuccess) return e;
    const int ntiles = (ncols + TC - 1) / TC;
    mr_colmul_kernel<<<dim3((unsigned)(nouter * ntiles), (unsigned)nsim), 256, smem, st>>>(
        S, K, ncols, comp_stride, outer_stride, line_stride, n_in, kaxis, scale, f, tw, ctl, skip_retry, sim_stride,
        sim_scale, TC);
    return cudaGetLastError();
}

template cudaError_t launch_mr_xfwd<float2, float>(int, const float*, PP, const float*, float2*, int, int, int, int,
                                                   int, int, int, const DevCtl*, int, cudaStream_t, int, long long,
                                                   long long, long long);
template cudaError_t launch_mr_xfwd<double2, double>(int, const double*, PP, const float*, double2*, int, int, int,
                                                     int, int, int, int, const DevCtl*, int, cudaStream_t, int,
                                                     long long, long long, long long);
template cudaError_t launch_mr_colfft<float2>(int, int, float2*, int, int, long long, long long, int, int,
                                              const DevCtl*, int, cudaStream_t, int, long long);
template cudaError_t launch_mr_colfft<double2>(int, int, double2*, int, int, long long, long long, int, int,
                                               const DevCtl*, int, cudaStream_t, int, long long);

}  // namespace mm
