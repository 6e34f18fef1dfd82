// fft.cuh -- shared-memory Stockham FFT building blocks for the demag convolution.
//
// Every line of length L (a power of two, 2..4096) is transformed by TPL = max(1, L/8)
// threads that each keep 8 complex values in registers per stage (radix-8 stages, a
// final radix-4 or radix-2 stage when log2(L) is not a multiple of 3).  Stages exchange
// data through shared memory; the Stockham autosort formulation (Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors", SC'08) leaves
// the output in natural order, so no bit reversal pass is needed.
//
// Shared memory lines are padded with one element every 8 (PADX) so that the stride-R
// stores of the early stages spread over the banks.
//
// V is float2 (hot path) or double2 (one-off demag tensor transform at plan time).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace mmfft {

__host__ __device__ constexpr int padx(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int line_len(int L) { return L + (L >> 3) + 1; }
__host__ __device__ constexpr int tpl(int L) { return L >= 8 ? L / 8 : 1; }

template <typename V> struct Scalar;
template <> struct Scalar<float2> { typedef float T; };
template <> struct Scalar<double2> { typedef double T; };

__device__ __forceinline__ float2 mkv(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mkv(double a, double b) { return make_double2(a, b); }

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mkv(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mkv(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    return mkv(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cconj(V a) { return mkv(a.x, -a.y); }
template <typename V, typename S> __device__ __forceinline__ V cscale(V a, S s) { return mkv(a.x * s, a.y * s); }
// multiply by SIGN*i
template <int SIGN, typename V> __device__ __forceinline__ V mul_si(V a) {
    return SIGN > 0 ? mkv(-a.y, a.x) : mkv(a.y, -a.x);
}

// exp(SIGN * 2 pi i * num / den)
template <int SIGN> __device__ __forceinline__ float2 twiddle_f(int num, int den) {
    float s, c;
    sincospif(2.0f * (float)num / (float)den, &s, &c);
    return make_float2(c, SIGN > 0 ? s : -s);
}
template <int SIGN> __device__ __forceinline__ double2 twiddle_d(int num, int den) {
    double s, c;
    sincospi(2.0 * (double)num / (double)den, &s, &c);
    return make_double2(c, SIGN > 0 ? s : -s);
}
template <int SIGN, typename V> struct Tw;
template <int SIGN> struct Tw<SIGN, float2> {
    static __device__ __forceinline__ float2 get(int n, int d) { return twiddle_f<SIGN>(n, d); }
};
template <int SIGN> struct Tw<SIGN, double2> {
    static __device__ __forceinline__ double2 get(int n, int d) { return twiddle_d<SIGN>(n, d); }
};

// ---- small DFTs in registers: X[k] = sum_n a[n] exp(SIGN 2 pi i n k / R)
template <int R, int SIGN, typename V> struct Dft;

template <int SIGN, typename V> struct Dft<1, SIGN, V> {
    static __device__ __forceinline__ void run(V*) {}
};
template <int SIGN, typename V> struct Dft<2, SIGN, V> {
    static __device__ __forceinline__ void run(V* a) {
        V t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    }
};
template <int SIGN, typename V> struct Dft<4, SIGN, V> {
    static __device__ __forceinline__ void run(V* a) {
        V t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        V t2 = cadd(a[1], a[3]), t3 = mul_si<SIGN>(csub(a[1], a[3]));
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        a[1] = cadd(t1, t3);
        a[3] = csub(t1, t3);
    }
};
template <int SIGN, typename V> struct Dft<8, SIGN, V> {
    static __device__ __forceinline__ void run(V* a) {
        typedef typename Scalar<V>::T S;
        const S c = (S)0.70710678118654752440;
        V e[4] = {a[0], a[2], a[4], a[6]};
        V o[4] = {a[1], a[3], a[5], a[7]};
        Dft<4, SIGN, V>::run(e);
        Dft<4, SIGN, V>::run(o);
        // W^k, W = exp(SIGN i pi / 4)
        V w1 = mkv(c, SIGN > 0 ? c : -c);
        V w3 = mkv(-c, SIGN > 0 ? c : -c);
        V o1 = cmul(o[1], w1);
        V o2 = mul_si<SIGN>(o[2]);
        V o3 = cmul(o[3], w3);
        a[0] = cadd(e[0], o[0]);
        a[4] = csub(e[0], o[0]);
        a[1] = cadd(e[1], o1);
        a[5] = csub(e[1], o1);
        a[2] = cadd(e[2], o2);
        a[6] = csub(e[2], o2);
        a[3] = cadd(e[3], o3);
        a[7] = csub(e[3], o3);
    }
};

// ---- twiddles.  FP32: read from a table of exp(-2 pi i k / TWN), k < TWN, rounded
// once from FP64 on the host (one load instead of a sincos per factor).  FP64 (plan
// set-up only): computed.
constexpr int TWN = 4096;
template <int SIGN, typename V> struct TwSrc;
template <int SIGN> struct TwSrc<SIGN, float2> {
    // exp(SIGN 2 pi i num / den), den a power of two <= TWN
    static __device__ __forceinline__ float2 get(const float2* tw, int num, int den) {
        float2 w = __ldg(tw + ((num * (TWN / den)) & (TWN - 1)));
        return SIGN > 0 ? make_float2(w.x, -w.y) : w;
    }
};
template <int SIGN> struct TwSrc<SIGN, double2> {
    static __device__ __forceinline__ double2 get(const float2*, int num, int den) { return twiddle_d<SIGN>(num, den); }
};

// ---- one Stockham stage on a padded shared-memory line, then the remaining stages.
// All threads of the block must call this (it synchronises); `active` masks the work.
template <int L, int Ns, int SIGN, typename V>
__device__ __forceinline__ void stockham(V* x, int t, bool active, const float2* tw) {
    constexpr int R = (L / Ns >= 8) ? 8 : (L / Ns);
    constexpr int TPL = tpl(L);
    constexpr int NB = (L / R) / TPL;
    V v[NB][R];
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int j = t + b * TPL;
#pragma unroll
            for (int r = 0; r < R; r++) v[b][r] = x[padx(j + r * (L / R))];
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int j = t + b * TPL;
            const int k = j & (Ns - 1);
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[b][r] = cmul(v[b][r], TwSrc<SIGN, V>::get(tw, r * k, Ns * R));
            }
            Dft<R, SIGN, V>::run(v[b]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) x[padx(base + r * Ns)] = v[b][r];
        }
    }
    __syncthreads();
    if constexpr (Ns * R < L) stockham<L, Ns * R, SIGN, V>(x, t, active, tw);
}

// Full in-place FFT of one padded line (unnormalised).  SIGN = -1 forward, +1 inverse.
template <int L, int SIGN, typename V>
__device__ __forceinline__ void fft_line(V* x, int t, bool active, const float2* tw) {
    if constexpr (L > 1) stockham<L, 1, SIGN, V>(x, t, active, tw);
}

// Host: the FP32 twiddle table exp(-2 pi i k / TWN), rounded from FP64.
inline void make_twiddle_table(float2* host) {
    for (int k = 0; k < TWN; k++) {
        double a = -2.0 * 3.14159265358979323846264338327950288 * (double)k / TWN;
        host[k] = make_float2((float)cos(a), (float)sin(a));
    }
}

}  // namespace mmfft
