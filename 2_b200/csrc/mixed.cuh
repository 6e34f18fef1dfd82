// mixed.cuh -- mixed-radix FFT of one shared-memory line, for transform lengths that are
// not powers of two.
//
// The reference accepts any padded size (cuFFT, fftplanX.go:59-64) and recommends
// 2^n * {1, 3, 5, 7} (engine/gridsize.go:16-33).  The power-of-two passes (fft.cuh,
// fft4.cuh) serve the common case; every other length L <= 4096 whose prime factors are
// at most MR_MAXR goes through these routines: a self-sorting Stockham transform
// (Govindaraju et al., SC'08; natural-order output, no bit reversal) with one stage per
// factor, radices 8, 4, 2 in registers and every other prime factor as a direct DFT.
// Twiddles come from per-length tables of exp(-2 pi i t / L), computed in FP64 on the
// host and kept per device (mr_prepare at plan creation, mr_tables at launch).
//
// A line lives in shared memory with a scratch line of the same length; the stages
// ping-pong between them and the result ends in the line itself.  nt threads transform
// one line; all threads of the block call mr_fft the same number of times (it
// synchronises the block), `active` masks the work.
#pragma once
#include "fft.cuh"

namespace mm {

constexpr int MR_MAXST = 16;   // stages: 4096 = 8^4, and at most 12 prime factors beyond
constexpr int MR_MAXR = 31;    // largest prime factor of a supported length
constexpr int MR_MAXL = 4096;  // largest supported length

struct MrLine {
    int L;
    int nst;
    int r[MR_MAXST];  // radix of each stage
};

// Host: factorisation of L into stages (8s, then 4, 2, then odd primes); false if L has
// a prime factor above MR_MAXR or is out of range.
bool mr_factor(int L, MrLine* f);
// Host: builds (once per device and length) the FP32 and FP64 twiddle tables of length L
// on the current device; call outside stream capture.  MM_OK or an error code.
int mr_prepare(int L);
// Host: the tables of length L on the current device (prepared earlier), or false.
bool mr_tables(int L, const float2** tf, const double2** td);
// Whether the power-of-two passes serve length L (else the mixed-radix ones do).
inline bool mr_pow2(int L) { return L > 0 && (L & (L - 1)) == 0 && L <= MR_MAXL; }

template <typename V> struct MrTab;
template <> struct MrTab<float2> { typedef const float2* type; };
template <> struct MrTab<double2> { typedef const double2* type; };

// exp(SIGN 2 pi i t / L) from the table (t < L)
template <int SIGN, typename V>
__device__ __forceinline__ V mr_w(const V* __restrict__ tw, int t) {
    const V w = tw[t];
    return SIGN > 0 ? mmfft::mkv(w.x, -w.y) : w;
}

// direct DFT of prime length R (odd): X[k] = sum_n v[n] W^(n k), W = exp(SIGN 2 pi i / R)
template <int R, int SIGN, typename V>
__device__ __forceinline__ void mr_dft_direct(V* v, const V* __restrict__ tw, int L) {
    using namespace mmfft;
    const int step = L / R;
    V out[R];
#pragma unroll
    for (int k = 0; k < R; k++) {
        V acc = v[0];
#pragma unroll
        for (int n = 1; n < R; n++) acc = cadd(acc, cmul(v[n], mr_w<SIGN>(tw, ((n * k) % R) * step)));
        out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = out[k];
}

template <int R, int SIGN, typename V>
__device__ __forceinline__ void mr_small_dft(V* v, const V* __restrict__ tw, int L) {
    if constexpr (R == 2 || R == 4 || R == 8) mmfft::Dft<R, SIGN, V>::run(v);
    else mr_dft_direct<R, SIGN, V>(v, tw, L);
}

// One Stockham stage of radix R: in -> out, Ns = product of the radices before it.
template <int R, int SIGN, typename V>
__device__ __forceinline__ void mr_stage_t(const V* in, V* out, int L, int Ns, const V* __restrict__ tw, int t,
                                           int nt) {
    using namespace mmfft;
    const int Lr = L / R;
    const int ts = L / (Ns * R);
    for (int j = t; j < Lr; j += nt) {
        const int k = j % Ns;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = in[j + r * Lr];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) v[r] = cmul(v[r], mr_w<SIGN>(tw, k * r * ts));
        }
        mr_small_dft<R, SIGN, V>(v, tw, L);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) out[base + r * Ns] = v[r];
    }
}

// a prime radix that has no compiled stage: the same stage with a local array
template <int SIGN, typename V>
__device__ void mr_stage_any(const V* in, V* out, int L, int R, int Ns, const V* __restrict__ tw, int t, int nt) {
    using namespace mmfft;
    const int Lr = L / R;
    const int ts = L / (Ns * R);
    const int step = L / R;
    for (int j = t; j < Lr; j += nt) {
        const int k = j % Ns;
        V v[MR_MAXR];
        for (int r = 0; r < R; r++) {
            v[r] = in[j + r * Lr];
            if (r > 0 && Ns > 1) v[r] = cmul(v[r], mr_w<SIGN>(tw, k * r * ts));
        }
        const int base = (j - k) * R + k;
        for (int q = 0; q < R; q++) {
            V acc = v[0];
            for (int n = 1; n < R; n++) acc = cadd(acc, cmul(v[n], mr_w<SIGN>(tw, ((n * q) % R) * step)));
            out[base + q * Ns] = acc;
        }
    }
}

// In-place transform of line a (scratch b, both L elements), unnormalised; SIGN -1
// forward, +1 inverse.  Synchronises the block before, between and after the stages.
template <int SIGN, typename V>
__device__ void mr_fft(V* a, V* b, const MrLine& f, const V* __restrict__ tw, int t, int nt, bool active) {
    V* src = a;
    V* dst = b;
    int Ns = 1;
    for (int s = 0; s < f.nst; s++) {
        __syncthreads();
        const int R = f.r[s];
        if (active) {
            switch (R) {
                case 2: mr_stage_t<2, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                case 3: mr_stage_t<3, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                case 4: mr_stage_t<4, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                case 5: mr_stage_t<5, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                case 7: mr_stage_t<7, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                case 8: mr_stage_t<8, SIGN, V>(src, dst, f.L, Ns, tw, t, nt); break;
                default: mr_stage_any<SIGN, V>(src, dst, f.L, R, Ns, tw, t, nt); break;
            }
        }
        Ns *= R;
        V* tmp = src;
        src = dst;
        dst = tmp;
    }
    __syncthreads();
    if (src != a) {
        if (active)
            for (int e = t; e < f.L; e += nt) a[e] = src[e];
        __syncthreads();
    }
}

}  // namespace mm
