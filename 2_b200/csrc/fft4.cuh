// fft4.cuh -- register four-step FFT of one line of length L = P1 * P2 (L <= 1024).
//
// A line is transformed by P2 threads.  Thread t holds the P1 elements x[t + P2*j] in
// registers, does a length-P1 DFT over j, multiplies by the twiddles W_L^(t*k1), writes
// the P1 results to a padded shared-memory buffer (row k1, column t), and after one
// barrier reads back rows k1 = t + q*P2 (q < P1/P2) and does length-P2 DFTs over t.  The
// result X[k1 + P1*k2] ends up in registers, so loads come straight from global memory
// and stores go straight back: one shared-memory round trip per line instead of one per
// radix stage.  (Bailey's four-step factorisation X[k1 + P1 k2] =
// sum_t W_P2^(t k2) W_L^(t k1) sum_j W_P1^(j k1) x[t + P2 j].)
//
// Buffer rows have an odd pitch (P2 + 1), so both the column writes and the row reads
// of a warp fall on distinct banks.
#pragma once
#include "fft.cuh"

namespace mmfft {

// exp(SIGN 2 pi i m / 32); m is a compile-time constant after unrolling
template <int SIGN>
__device__ __forceinline__ float2 w32(int m) {
    constexpr float C[9] = {1.000000000e+00f, 9.807852804e-01f, 9.238795325e-01f, 8.314696123e-01f,
                            7.071067812e-01f, 5.555702330e-01f, 3.826834324e-01f, 1.950903220e-01f, 0.0f};
    m &= 31;
    const int q = m >> 3, r = m & 7;
    const float cr = C[r], sr = C[8 - r];
    float2 v = (q == 0) ? make_float2(cr, sr) : (q == 1) ? make_float2(-sr, cr) : (q == 2) ? make_float2(-cr, -sr)
                                                                                         : make_float2(sr, -cr);
    return SIGN > 0 ? v : make_float2(v.x, -v.y);
}

// in-register DFT of length P in {1,2,4,8,16,32}: a[k] = sum_n a[n] exp(SIGN 2 pi i n k / P)
template <int P, int SIGN> struct RDft {
    static __device__ __forceinline__ void run(float2* a) { Dft<P, SIGN, float2>::run(a); }
};
template <int SIGN> struct RDft<16, SIGN> {
    static __device__ __forceinline__ void run(float2* a) {
        float2 t[4][4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
#pragma unroll
            for (int n = 0; n < 4; n++) t[r][n] = a[4 * n + r];
            Dft<4, SIGN, float2>::run(t[r]);
        }
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            float2 u[4];
#pragma unroll
            for (int r = 0; r < 4; r++) u[r] = (r * k1 == 0) ? t[r][k1] : cmul(t[r][k1], w32<SIGN>(2 * r * k1));
            Dft<4, SIGN, float2>::run(u);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) a[k1 + 4 * k2] = u[k2];
        }
    }
};
template <int SIGN> struct RDft<32, SIGN> {
    static __device__ __forceinline__ void run(float2* a) {
        float2 e[16], o[16];
#pragma unroll
        for (int n = 0; n < 16; n++) {
            e[n] = a[2 * n];
            o[n] = a[2 * n + 1];
        }
        RDft<16, SIGN>::run(e);
        RDft<16, SIGN>::run(o);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            float2 wo = (k == 0) ? o[k] : cmul(o[k], w32<SIGN>(k));
            a[k] = cadd(e[k], wo);
            a[k + 16] = csub(e[k], wo);
        }
    }
};

__host__ __device__ constexpr int fs_p2(int L) {
    int lg = 0;
    while ((1 << lg) < L) lg++;
    return 1 << (lg / 2);
}

template <int L>
struct FS {
    static constexpr int P2 = fs_p2(L);   // threads per line
    static constexpr int P1 = L / P2;     // elements per thread (P2 or 2*P2)
    static constexpr int Q = P1 / P2;
    static constexpr int PITCH = P2 + 1;
    static constexpr int LBUF = P1 * PITCH;  // float2 per line buffer

    // input element index of register j for thread t
    static __device__ __forceinline__ int in_index(int t, int j) { return t + P2 * j; }
    // output element index of register r (= q*P2 + k2) for thread t
    static __device__ __forceinline__ int out_index(int t, int r) { return t + (r / P2) * P2 + P1 * (r % P2); }

    // Transforms the line held by the P2 threads (t = 0..P2-1) of this line.  All threads of
    // the block must call it (it synchronises twice); `active` masks the buffer traffic.
    // Shared-memory table of the step-1 twiddles, twt[k1 * P2 + t] = W_L^(t k1) (forward
    // sign), filled cooperatively by the block; L entries.
    static constexpr int TWT = P1 * P2;
    static __device__ __forceinline__ void fill_twiddles(float2* twt, const float2* __restrict__ tw) {
        for (int e = threadIdx.x; e < TWT; e += blockDim.x) {
            const int k1 = e / P2, t = e % P2;
            twt[e] = TwSrc<-1, float2>::get(tw, (t * k1) & (L - 1), L);
        }
    }

    template <int SIGN>
    static __device__ __forceinline__ void run(float2 (&v)[P1], float2* buf, int t, bool active,
                                               const float2* twt, int pair_mask = 1) {
        if (active) {
            RDft<P1, SIGN>::run(v);
#pragma unroll
            for (int k1 = 1; k1 < P1; k1++) {
                const float2 w = twt[k1 * P2 + t];
                v[k1] = cmul(v[k1], SIGN > 0 ? make_float2(w.x, -w.y) : w);
            }
#pragma unroll
            for (int k1 = 0; k1 < P1; k1++) buf[k1 * PITCH + t] = v[k1];
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int q = 0; q < Q; q++) {
                float2 u[P2];
                const int k1 = t + q * P2;
#pragma unroll
                for (int tt = 0; tt < P2; tt++) u[tt] = buf[k1 * PITCH + tt];
                RDft<P2, SIGN>::run(u);
#pragma unroll
                for (int k2 = 0; k2 < P2; k2++) v[q * P2 + k2] = u[k2];
            }
        }
        __syncthreads();
    }
};

// L = 512 = 16 x 32: 32 threads per line, 16 elements each (half the registers of a
// 32 x 16 split).  The length-32 second stage of column k1 is shared by the thread pair
// (2 k1, 2 k1 + 1): each does a length-16 DFT of the even or odd t, and the halves are
// combined with one shuffle, X[k1 + 16 k2] = D0[k2 mod 16] +- W_32^(k2 mod 16) D1[k2 mod 16].
// `pair_mask` is the lane distance between threads t and t^1.
template <>
struct FS<512> {
    static constexpr int P2 = 32;
    static constexpr int P1 = 16;
    static constexpr int PITCH = 34;  // = 2 (mod 16): the pair-strided reads hit distinct banks
    static constexpr int LBUF = P1 * PITCH;

    static __device__ __forceinline__ int in_index(int t, int j) { return t + 32 * j; }
    static __device__ __forceinline__ int out_index(int t, int r) { return (t >> 1) + 16 * (r + 16 * (t & 1)); }

    static constexpr int TWT = P1 * P2;
    static __device__ __forceinline__ void fill_twiddles(float2* twt, const float2* __restrict__ tw) {
        for (int e = threadIdx.x; e < TWT; e += blockDim.x) {
            const int k1 = e / P2, t = e % P2;
            twt[e] = TwSrc<-1, float2>::get(tw, t * k1, 512);
        }
    }

    template <int SIGN>
    static __device__ __forceinline__ void run(float2 (&v)[16], float2* buf, int t, bool active,
                                               const float2* twt, int pair_mask) {
        if (active) {
            RDft<16, SIGN>::run(v);
#pragma unroll
            for (int k1 = 1; k1 < 16; k1++) {
                const float2 w = twt[k1 * P2 + t];
                v[k1] = cmul(v[k1], SIGN > 0 ? make_float2(w.x, -w.y) : w);
            }
#pragma unroll
            for (int k1 = 0; k1 < 16; k1++) buf[k1 * PITCH + t] = v[k1];
        }
        __syncthreads();
        const int h = t & 1;
        if (active) {
            const int k1 = t >> 1;
#pragma unroll
            for (int u = 0; u < 16; u++) v[u] = buf[k1 * PITCH + 2 * u + h];
            RDft<16, SIGN>::run(v);
        }
#pragma unroll
        for (int k = 0; k < 16; k++) {
            float2 o;
            o.x = __shfl_xor_sync(0xffffffffu, v[k].x, pair_mask);
            o.y = __shfl_xor_sync(0xffffffffu, v[k].y, pair_mask);
            const float2 w = w32<SIGN>(k);
            v[k] = h == 0 ? cadd(v[k], cmul(w, o)) : csub(o, cmul(w, v[k]));
        }
        __syncthreads();
    }
};

}  // namespace mmfft
