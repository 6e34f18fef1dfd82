// rhs.cu -- fused right-hand side epilogue.
//
// One pass over the cells computes, per cell,
//   H_eff = H_demag (inverse row transform of the convolved spectrum, in shared memory)
//         + H_ex (exchange6.cu:12-142)  + B_ext/mu0 (mod_zeeman.go, add.cu:82-95)
//         + H_anis (uniaxialanisotropy.cu:12-86) + H_therm (temperature.cu:14-66 with
//           in-register Philox normals instead of a cuRAND noise buffer)
//   k     = (m x H - alpha m x (m x H))/(1+alpha^2)            (torque.cu:13-57)
//         + (zzt + stt)/gamma                                  (update_addterm.go:37-40,
//           zhang-li_torque.cu:123-300, slonczewski_torque.cu:14-116)
// and then whatever the time stepper needs from k at that cell (StageOp): the store
// of k, the next Runge-Kutta stage state (normalised, normalize.cu:14-42), the error
// estimate and the max-torque reduction.  The reference runs these as separate
// kernels with a host sync after each (libmumax2.go), plus a D2H copy per reduction
// (reductor.go:69-186).
#include <cstdio>

#include "fft.cuh"
#include "fft4.cuh"
#include "mixed.cuh"
#include "mm_internal.h"
#include "kernel_view.cuh"
#include "pdl.cuh"

namespace mm {
using namespace mmfft;

__device__ __forceinline__ bool skip_eval(const DevCtl* ctl, int skip_retry) {
    return ctl && (ctl->done || (skip_retry == 1 && ctl->tries > 0) || (skip_retry == 2 && ctl->am_skip));
}

// ---------------------------------------------------------------- Philox4x32-10
// Salmon, Moraes, Dror, Shaw, SC'11 (published constants of the Philox4x32 family).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        unsigned int hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        unsigned int hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Three standard normals for (cell, step): Box-Muller on 24-bit uniforms in (0,1).
__device__ __forceinline__ void thermal_normals(unsigned long long seed, long long cell, long long step, float eta[3]) {
    uint4 c = make_uint4((unsigned)cell, (unsigned)((unsigned long long)step & 0xffffffffu),
                         (unsigned)((unsigned long long)step >> 32), 0x7e57u);
    uint4 r = philox4x32_10(c, make_uint2((unsigned)(seed & 0xffffffffu), (unsigned)(seed >> 32)));
    const float s = 5.9604644775390625e-08f;  // 2^-24
    float u0 = ((float)(r.x >> 8) + 0.5f) * s, u1 = ((float)(r.y >> 8) + 0.5f) * s;
    float u2 = ((float)(r.z >> 8) + 0.5f) * s, u3 = ((float)(r.w >> 8) + 0.5f) * s;
    float r0 = sqrtf(-2.0f * logf(u0)), r1 = sqrtf(-2.0f * logf(u2));
    float s1, c1, s3, c3;
    sincospif(2.0f * u1, &s1, &c1);
    sincospif(2.0f * u3, &s3, &c3);
    eta[0] = r0 * c1;
    eta[1] = r0 * s1;
    eta[2] = r1 * c3;
}

__device__ __forceinline__ float mval(const float* m, long long i) { return m ? __ldg(m + i) : 1.0f; }
// The masked exchange weights (Aex/Msat ratios of a cell and its neighbour, and their
// harmonic mean, common_func.h:298-317) with the fast single-precision quotient
// __fdividef (at most 2 ulp for the mask ratios of order one met here): nine quotients
// per cell took a quarter of the masked epilogue with IEEE division (batched 64x64 relax
// plan: C2R + epilogue 78.5 -> 59.5 us per evaluation, RK23 step 459 -> 433 us).  Unit
// weights stay exact (1/1 and 2/2 are 1), so an all-ones mask still reproduces the unmasked
// result bit for bit.
__device__ __forceinline__ float fdiv_zero(float a, float b) { return (b == 0.0f) ? 0.0f : __fdividef(a, b); }
__device__ __forceinline__ float avg_geom_zero(float a, float b) {
    float ab = a + b;
    return (ab == 0.0f) ? 0.0f : __fdividef(2.0f * a * b, ab);
}
// crossf of common_func.h:222-225: -(a x b)
__device__ __forceinline__ float3 crossf(float3 a, float3 b) {
    return make_float3(-a.y * b.z + a.z * b.y, -a.z * b.x + a.x * b.z, -a.x * b.y + a.y * b.x);
}

// neighbour index for the 6-point stencil: clamp, or wrap when periodic
__device__ __forceinline__ int nb6(int i, int d, int n, int wrap) {
    int j = i + d;
    if (d < 0) { if (j < 0 && wrap) j += n; j = max(j, 0); }
    else { if (j == n && wrap) j -= n; j = min(j, n - 1); }
    return j;
}
// neighbour index for the 5-point Zhang-Li stencil: out of range -> the cell itself,
// unless periodic (zhang-li_torque.cu:187-225)
__device__ __forceinline__ int nb5(int i, int d, int n, int wrap) {
    int j = i + d;
    if (!wrap && (j < 0 || j >= n)) return i;
    if (j < 0) j += n;
    if (j >= n) j -= n;
    return j;
}

struct CellTerms {
    float hd[3], hex[3], han[3], hz[3], hth[3];
};

// Effective field and torque at one cell.  Returns k (tau/gamma + STT/gamma).
// m points at this simulation's state, i is the cell within the simulation, mo the
// offset of the simulation's masks (0 when masks are shared), S its scalars.
// SPEC: what the evaluation is known, at compile time, not to have (the launcher checks):
// SPEC_NOMASK no per-cell mask of any kind (every mask reads as absent, unit exchange
// weights, 32-bit neighbour offsets), SPEC_NOTHERMAL no thermal term, SPEC_NOSTT no
// Zhang-Li or Slonczewski term.  The absent parts are compiled out, which leaves the same
// arithmetic with fewer registers and instructions per cell.  SPEC_LEAN has all three.
constexpr int SPEC_NOMASK = 1, SPEC_NOTHERMAL = 2, SPEC_NOSTT = 4, SPEC_LEAN = 7;
template <int SPEC>
__device__ __forceinline__ const float* lean_mask(const float* q) { return (SPEC & SPEC_NOMASK) ? nullptr : q; }

template <bool WANT_TERMS, int SPEC = 0>
__device__ __forceinline__ float3 cell_rhs(const FieldParams& P, const SimScalars& S, const float* __restrict__ m,
                                           long long i, long long mo, int z, int y, int x, float3 hd,
                                           long long noise_step, float dt_th, float3& m0, CellTerms* terms) {
    const long long N = P.N;
    const long long im = i + mo;
    m0 = make_float3(__ldg(m + i), __ldg(m + N + i), __ldg(m + 2 * N + i));
    float3 H = hd;
    if (WANT_TERMS) { terms->hd[0] = hd.x; terms->hd[1] = hd.y; terms->hd[2] = hd.z; }
    if (P.exchange) {
        const int n1 = P.n[1], n2 = P.n[2];
        const bool masked = !(SPEC & SPEC_NOMASK) && (P.msat_mask || P.aex_mask);
        const float lex0 = masked ? fdiv_zero(mval(P.aex_mask, im), mval(P.msat_mask, im)) : 1.0f;
        float3 hex = make_float3(0.f, 0.f, 0.f);
        const int c[3] = {z, y, x};
        const long long str[3] = {(long long)n1 * n2, n2, 1};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (P.n[d] == 1) continue;  // both neighbours clamp onto the cell itself: no contribution
            int lo = nb6(c[d], -1, P.n[d], P.pbc[d]);
            int hi = nb6(c[d], +1, P.n[d], P.pbc[d]);
            if constexpr ((SPEC & SPEC_NOMASK) != 0) {
                // unit weights (no masks); neighbour offsets in 32 bits from the cell's
                // component pointers (a simulation holds fewer than 2^31 cells)
                const int st = d == 0 ? n1 * n2 : (d == 1 ? n2 : 1);
                const int dl = (lo - c[d]) * st, dh = (hi - c[d]) * st;
                const float* mc = m + i;
                const float f = S.ex_pre * P.cinv2[d];
                float3 a = make_float3(__ldg(mc + dl), __ldg(mc + N + dl), __ldg(mc + 2 * N + dl));
                float3 b = make_float3(__ldg(mc + dh), __ldg(mc + N + dh), __ldg(mc + 2 * N + dh));
                hex.x += f * ((a.x - m0.x) + (b.x - m0.x));
                hex.y += f * ((a.y - m0.y) + (b.y - m0.y));
                hex.z += f * ((a.z - m0.z) + (b.z - m0.z));
                continue;
            }
            long long il = i + (long long)(lo - c[d]) * str[d];
            long long ih = i + (long long)(hi - c[d]) * str[d];
            float l1 = 1.f, l2 = 1.f;
            if (masked) {
                l1 = avg_geom_zero(lex0, fdiv_zero(mval(P.aex_mask, il + mo), mval(P.msat_mask, il + mo)));
                l2 = avg_geom_zero(lex0, fdiv_zero(mval(P.aex_mask, ih + mo), mval(P.msat_mask, ih + mo)));
            }
            const float f = S.ex_pre * P.cinv2[d];
            float3 a = make_float3(__ldg(m + il), __ldg(m + N + il), __ldg(m + 2 * N + il));
            float3 b = make_float3(__ldg(m + ih), __ldg(m + N + ih), __ldg(m + 2 * N + ih));
            hex.x += f * (l1 * (a.x - m0.x) + l2 * (b.x - m0.x));
            hex.y += f * (l1 * (a.y - m0.y) + l2 * (b.y - m0.y));
            hex.z += f * (l1 * (a.z - m0.z) + l2 * (b.z - m0.z));
        }
        H.x += hex.x; H.y += hex.y; H.z += hex.z;
        if (WANT_TERMS) { terms->hex[0] = hex.x; terms->hex[1] = hex.y; terms->hex[2] = hex.z; }
    }
    if (P.zeeman) {
        float3 hz = make_float3(S.hz[0] * mval(lean_mask<SPEC>(P.bext_mask[0]), im),
                                S.hz[1] * mval(lean_mask<SPEC>(P.bext_mask[1]), im),
                                S.hz[2] * mval(lean_mask<SPEC>(P.bext_mask[2]), im));
        H.x += hz.x; H.y += hz.y; H.z += hz.z;
        if (WANT_TERMS) { terms->hz[0] = hz.x; terms->hz[1] = hz.y; terms->hz[2] = hz.z; }
    }
    if (P.anis) {
        float msm = mval(lean_mask<SPEC>(P.msat_mask), im);
        if (msm == 0.0f) msm = 1.0f;
        float k2 = (S.kmul / msm) * mval(lean_mask<SPEC>(P.ku_mask), im);
        float ux = S.anisu[0] * mval(lean_mask<SPEC>(P.anisu_mask[0]), im);
        float uy = S.anisu[1] * mval(lean_mask<SPEC>(P.anisu_mask[1]), im);
        float uz = S.anisu[2] * mval(lean_mask<SPEC>(P.anisu_mask[2]), im);
        float mu = m0.x * ux + m0.y * uy + m0.z * uz;
        float3 ha = make_float3(k2 * mu * ux, k2 * mu * uy, k2 * mu * uz);
        H.x += ha.x; H.y += ha.y; H.z += ha.z;
        if (WANT_TERMS) { terms->han[0] = ha.x; terms->han[1] = ha.y; terms->han[2] = ha.z; }
    }
    if (!(SPEC & SPEC_NOTHERMAL) && P.thermal) {
        float ms = mval(lean_mask<SPEC>(P.msat_mask), im);
        float3 ht = make_float3(0.f, 0.f, 0.f);
        if (ms != 0.0f) {
            float eta[3];
            thermal_normals(S.seed, i, noise_step, eta);
            float a = mval(lean_mask<SPEC>(P.alpha_mask), im), tm = mval(lean_mask<SPEC>(P.temp_mask), im);
            float den = (float)(S.therm_den * (double)dt_th);
            float sc = sqrtf((a * tm * S.therm_num) / (den * ms));
            ht = make_float3(eta[0] * sc, eta[1] * sc, eta[2] * sc);
        }
        H.x += ht.x; H.y += ht.y; H.z += ht.z;
        if (WANT_TERMS) { terms->hth[0] = ht.x; terms->hth[1] = ht.y; terms->hth[2] = ht.z; }
    }
    // LLG torque
    const float al = S.alpha * mval(lean_mask<SPEC>(P.alpha_mask), im);
    float cx = m0.y * H.z - H.y * m0.z, cy = -m0.x * H.z + H.x * m0.z, cz = m0.x * H.y - H.x * m0.y;
    float dx = -m0.y * cz + cy * m0.z, dy = m0.x * cz - cx * m0.z, dz = -m0.x * cy + cx * m0.y;
    float g = 1.0f / (1.0f + al * al);
    float3 k = make_float3(g * (cx + dx * al), g * (cy + dy * al), g * (cz + dz * al));
    if (!(SPEC & SPEC_NOSTT) && P.zhangli) {
        float msat = P.msat_mask ? __ldg(P.msat_mask + im) : 1.0f;
        float3 j0 = make_float3(P.j_mask[0] ? __ldg(P.j_mask[0] + im) * S.jmul[0] : S.jmul[0],
                                P.j_mask[1] ? __ldg(P.j_mask[1] + im) * S.jmul[1] : S.jmul[1],
                                P.j_mask[2] ? __ldg(P.j_mask[2] + im) * S.jmul[2] : S.jmul[2]);
        float njn = sqrtf(j0.x * j0.x + j0.y * j0.y + j0.z * j0.z);
        if (msat != 0.0f && njn != 0.0f) {
            msat = 1.0f / msat;
            float PP = P.zl_pol_mask ? __ldg(P.zl_pol_mask + im) : 1.0f;
            float pred = njn * PP * S.zl_pre;
            float ee = P.xi_mask ? __ldg(P.xi_mask + im) * P.xi : P.xi;
            pred = pred / ((1.0f + ee * ee) * (1.0f + al * al));
            float pret = pred * (ee - al);
            pred = pred * (1.0f + ee * al);
            const float inv = 1.0f / njn;
            const float nj[3] = {j0.x * inv, j0.y * inv, j0.z * inv};
            const int c[3] = {z, y, x};
            const long long str[3] = {(long long)P.n[1] * P.n[2], P.n[2], 1};
            float3 dmdj = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int d = 0; d < 3; d++) {
                if (nj[d] == 0.0f) continue;
                long long ib2 = i + (long long)(nb5(c[d], -2, P.n[d], P.pbc[d]) - c[d]) * str[d];
                long long ib1 = i + (long long)(nb5(c[d], -1, P.n[d], P.pbc[d]) - c[d]) * str[d];
                long long if1 = i + (long long)(nb5(c[d], +1, P.n[d], P.pbc[d]) - c[d]) * str[d];
                long long if2 = i + (long long)(nb5(c[d], +2, P.n[d], P.pbc[d]) - c[d]) * str[d];
                const float s = P.c12inv[d] * nj[d];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const float* a = m + q * N;
                    float dv = __ldg(a + ib2) - 8.0f * __ldg(a + ib1) + 8.0f * __ldg(a + if1) - __ldg(a + if2);
                    if (q == 0) dmdj.x += s * dv;
                    else if (q == 1) dmdj.y += s * dv;
                    else dmdj.z += s * dv;
                }
            }
            float3 dmdjxm = crossf(dmdj, m0);
            float3 mxdmxm = crossf(m0, dmdjxm);
            k.x += P.inv_gamma * msat * (pred * mxdmxm.x + pret * dmdjxm.x);
            k.y += P.inv_gamma * msat * (pred * mxdmxm.y + pret * dmdjxm.y);
            k.z += P.inv_gamma * msat * (pred * mxdmxm.z + pret * dmdjxm.z);
        }
    }
    if (!(SPEC & SPEC_NOSTT) && P.slonczewski) {
        float Ms = P.msat_mask ? __ldg(P.msat_mask + im) : 1.0f;
        float3 J = make_float3(P.j_mask[0] ? __ldg(P.j_mask[0] + im) * S.jmul[0] : S.jmul[0],
                               P.j_mask[1] ? __ldg(P.j_mask[1] + im) * S.jmul[1] : S.jmul[1],
                               P.j_mask[2] ? __ldg(P.j_mask[2] + im) * S.jmul[2] : S.jmul[2]);
        float nJn = sqrtf(J.x * J.x + J.y * J.y + J.z * J.z);
        float tfl = P.t_fl_mask ? __ldg(P.t_fl_mask + im) * P.t_fl : P.t_fl;
        if (nJn != 0.0f && Ms != 0.0f && tfl != 0.0f) {
            tfl = 1.0f / tfl;
            Ms = 1.0f / Ms;
            float prex = S.sl_beta_prime * Ms, prey = S.sl_pre_fld * Ms;
            float3 p = make_float3(P.p_mask[0] ? P.p[0] * __ldg(P.p_mask[0] + im) : P.p[0],
                                   P.p_mask[1] ? P.p[1] * __ldg(P.p_mask[1] + im) : P.p[1],
                                   P.p_mask[2] ? P.p[2] * __ldg(P.p_mask[2] + im) : P.p[2]);
            float pl = sqrtf(p.x * p.x + p.y * p.y + p.z * p.z);
            float pinv = (pl != 0.0f) ? 1.0f / pl : 0.0f;
            p.x *= pinv; p.y *= pinv; p.z *= pinv;
            float3 pxm = crossf(p, m0);
            float3 mxpxm = crossf(m0, pxm);
            float pdotm = p.x * m0.x + p.y * m0.y + p.z * m0.z;
            float jinv = 1.0f / nJn;
            float Jdir = J.x * jinv + J.y * jinv + J.z * jinv;
            float Jsign = Jdir / fabsf(Jdir);
            float nj = nJn * Jsign;
            prex *= nj; prey *= nj;
            prex *= tfl; prey *= tfl;
            float lam = P.lambda_mask ? P.lambda * __ldg(P.lambda_mask + im) : P.lambda;
            float l2 = lam * lam;
            float eps = l2 / ((l2 + 1.0f) + (l2 - 1.0f) * pdotm);
            prex *= eps;
            float af = 1.0f / (1.0f + al * al);
            prex *= P.sl_pol_mask ? __ldg(P.sl_pol_mask + im) : 1.0f;
            prey *= P.eps_prime_mask ? __ldg(P.eps_prime_mask + im) : 1.0f;
            float f1 = (prex - al * prey) * af;
            float f2 = (prey - al * prex) * af;
            k.x += P.inv_gamma * (f1 * mxpxm.x + f2 * pxm.x);
            k.y += P.inv_gamma * (f1 * mxpxm.y + f2 * pxm.y);
            k.z += P.inv_gamma * (f1 * mxpxm.z + f2 * pxm.z);
        }
    }
    return k;
}

// Kahan-style compensated accumulation of FP32 values (Neumaier's variant).
struct KSum {
    float s, c;
    __device__ __forceinline__ void add(float v) {
        float t = s + v;
        if (fabsf(s) >= fabsf(v)) c += (s - t) + v;
        else c += (v - t) + s;
        s = t;
    }
};
__device__ __forceinline__ KSum ksum_merge(KSum a, KSum b) {
    KSum r = a;
    r.add(b.s);
    r.c += b.c;
    return r;
}

// Everything after k is known at one cell (StageOp).  Resolved pointers in `rp`.
struct ResolvedOp {
    float* k_out;
    const float* base;
    float* next;
    const float* kp[MM_MAXK];
    float ak[MM_MAXK];
    const float* ep[MM_MAXK];
    float ek[MM_MAXK];
};

// off: this simulation's offset into the per-cell arrays
__device__ __forceinline__ float* at_off(float* q, long long off) { return q ? q + off : nullptr; }
__device__ __forceinline__ void resolve_op(const StageOp& op, int cur, float h, ResolvedOp& r, long long off) {
    r.k_out = at_off(op.k_out.get(cur), off);
    r.base = at_off(op.base.get(cur), off);
    r.next = at_off(op.next.get(cur), off);
#pragma unroll
    for (int j = 0; j < MM_MAXK; j++) {
        r.kp[j] = (j < op.nk) ? at_off(op.kp[j].get(cur), off) : nullptr;
        r.ak[j] = (j < op.nk) ? (float)(op.ak[j] * (double)h) : 0.f;
        r.ep[j] = (j < op.ne) ? at_off(op.ep[j].get(cur), off) : nullptr;
        r.ek[j] = (j < op.ne) ? (float)op.ek[j] : 0.f;
    }
}

struct ThreadRed {
    float tq;
    float err;
    int bad;
    KSum e[4];
};

// stg (optional): receives the next state as the R2C row pass would read it, i.e. the
// stored value times the Msat mask when fwd_mask (the convolution input Ms_mask * m).
template <int SPEC = 0>
__device__ __forceinline__ void cell_post(const FieldParams& P, const StageOp& op, const ResolvedOp& r, long long i,
                                          long long mo, float3 m0, float3 k, ThreadRed& tr, float3* stg = nullptr,
                                          int fwd_mask = 0) {
    const long long N = P.N;
    if (!(isfinite(k.x) && isfinite(k.y) && isfinite(k.z))) tr.bad = 1;
    if (r.k_out) {
        r.k_out[i] = k.x;
        r.k_out[N + i] = k.y;
        r.k_out[2 * N + i] = k.z;
    }
    if (op.want_tq) tr.tq = fmaxf(tr.tq, k.x * k.x + k.y * k.y + k.z * k.z);
    if (op.do_combine) {
        float3 v = op.base_is_cur ? m0 : make_float3(r.base[i], r.base[N + i], r.base[2 * N + i]);
#pragma unroll
        for (int j = 0; j < MM_MAXK; j++) {
            if (j >= op.nk) break;
            float3 kj = (j == op.kcur) ? k : make_float3(r.kp[j][i], r.kp[j][N + i], r.kp[j][2 * N + i]);
            v.x += r.ak[j] * kj.x;
            v.y += r.ak[j] * kj.y;
            v.z += r.ak[j] * kj.z;
        }
        // normalize.cu:14-42 with the Msat mask as norm map
        float norm = mval(lean_mask<SPEC>(P.msat_mask), i + mo);
        float mn = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        const float3 nx = make_float3(v.x * sc, v.y * sc, v.z * sc);
        r.next[i] = nx.x;
        r.next[N + i] = nx.y;
        r.next[2 * N + i] = nx.z;
        if (stg) {
            const float fm = fwd_mask ? norm : 1.0f;
            *stg = make_float3(nx.x * fm, nx.y * fm, nx.z * fm);
        }
    }
    if (op.ne > 0) {
        float3 e = make_float3(0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < MM_MAXK; j++) {
            if (j >= op.ne) break;
            float3 kj = (j == op.ecur) ? k : make_float3(r.ep[j][i], r.ep[j][N + i], r.ep[j][2 * N + i]);
            e.x += r.ek[j] * kj.x;
            e.y += r.ek[j] * kj.y;
            e.z += r.ek[j] * kj.z;
        }
        tr.err = fmaxf(tr.err, fmaxf(fabsf(e.x), fmaxf(fabsf(e.y), fabsf(e.z))));
    }
}

__device__ __forceinline__ void energy_acc(const FieldParams& P, long long i, float3 m0, const CellTerms& t,
                                           ThreadRed& tr) {
    // m . B_ext (T): B_ext = mu0 * hz
    const float mu0 = 1.2566370614359172e-06f;
    tr.e[0].add(mu0 * (m0.x * t.hz[0] + m0.y * t.hz[1] + m0.z * t.hz[2]));
    tr.e[1].add(m0.x * t.hex[0] + m0.y * t.hex[1] + m0.z * t.hex[2]);
    tr.e[2].add(m0.x * t.hd[0] + m0.y * t.hd[1] + m0.z * t.hd[2]);
    tr.e[3].add(m0.x * t.han[0] + m0.y * t.han[1] + m0.z * t.han[2]);
}

// Block-level reduction of ThreadRed; thread 0 publishes.
__device__ void block_reduce_publish(ThreadRed tr, const StageOp& op, DevCtl* ctl, unsigned int* tq_out, float* red) {
    __shared__ float s_tq[32], s_err[32];
    __shared__ int s_bad[32];
    __shared__ float s_e[32][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tr.tq = fmaxf(tr.tq, __shfl_xor_sync(0xffffffffu, tr.tq, o));
        tr.err = fmaxf(tr.err, __shfl_xor_sync(0xffffffffu, tr.err, o));
        tr.bad |= __shfl_xor_sync(0xffffffffu, tr.bad, o);
    }
    if (op.want_energy) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                KSum b;
                b.s = __shfl_xor_sync(0xffffffffu, tr.e[q].s, o);
                b.c = __shfl_xor_sync(0xffffffffu, tr.e[q].c, o);
                tr.e[q] = ksum_merge(tr.e[q], b);
            }
        }
    }
    if (lane == 0) {
        s_tq[wid] = tr.tq;
        s_err[wid] = tr.err;
        s_bad[wid] = tr.bad;
        for (int q = 0; q < 4; q++) { s_e[wid][2 * q] = tr.e[q].s; s_e[wid][2 * q + 1] = tr.e[q].c; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float tq = 0.f, err = 0.f;
        int bad = 0;
        KSum e[4] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
        for (int w = 0; w < nw; w++) {
            tq = fmaxf(tq, s_tq[w]);
            err = fmaxf(err, s_err[w]);
            bad |= s_bad[w];
            for (int q = 0; q < 4; q++) {
                KSum b = {s_e[w][2 * q], s_e[w][2 * q + 1]};
                e[q] = ksum_merge(e[q], b);
            }
        }
        // ctl is this simulation's control block; tq_out and red are indexed by simulation
        if (ctl) {
            if (op.want_tq) atomicMax(&ctl->tq_bits, __float_as_uint(tq));
            if (op.ne > 0) atomicMax(&ctl->err_bits, __float_as_uint(err));
            if (bad) atomicExch(&ctl->status, (int)MM_ERR_NAN);
        } else if (tq_out && op.want_tq) {
            atomicMax(tq_out + blockIdx.y, __float_as_uint(tq));
        }
        if (op.want_energy && red) {
            const long long slot = (long long)blockIdx.y * gridDim.x + blockIdx.x;
            for (int q = 0; q < 4; q++) {
                red[slot * 8 + 2 * q] = e[q].s;
                red[slot * 8 + 2 * q + 1] = e[q].c;
            }
        }
    }
}

__device__ __forceinline__ void write_terms(float* const* dbg, long long N, long long i, const CellTerms& t) {
    const float* src[5] = {t.hd, t.hex, t.han, t.hz, t.hth};
    for (int q = 0; q < 5; q++)
        if (dbg[q])
            for (int c = 0; c < 3; c++) dbg[q][c * N + i] = src[q][c];
    if (dbg[5])
        for (int c = 0; c < 3; c++)
            dbg[5][c * N + i] = t.hd[c] + t.hex[c] + t.han[c] + t.hz[c] + t.hth[c];
}

// i: cell within the simulation; m, r and the dbg outputs already point at the simulation
template <bool TERMS, int SPEC = 0>
__device__ __forceinline__ void process_cell(const EpiArgs& A, const SimScalars& S, const float* m,
                                             const ResolvedOp& r, float* const* dbg, long long i, long long mo,
                                             int z, int y, int x, float3 hd, long long ns, float dtth,
                                             ThreadRed& tr, float3* stg = nullptr) {
    float3 m0;
    if (TERMS) {
        CellTerms t = {};
        float3 k = cell_rhs<true>(A.P, S, m, i, mo, z, y, x, hd, ns, dtth, m0, &t);
        if (A.op.want_energy) energy_acc(A.P, i, m0, t, tr);
        write_terms(dbg, A.P.N, i, t);
        cell_post(A.P, A.op, r, i, mo, m0, k, tr, stg, A.fwd_mask);
    } else {
        float3 k = cell_rhs<false, SPEC>(A.P, S, m, i, mo, z, y, x, hd, ns, dtth, m0, nullptr);
        cell_post<SPEC>(A.P, A.op, r, i, mo, m0, k, tr, stg, A.fwd_mask);
    }
}

// Per-block context of one simulation for the epilogue kernels.  BATCH = false is the
// single-simulation plan: simulation 0, scalars straight from the kernel parameters, no
// offsets.  BATCH = true takes the simulation from blockIdx.y and its scalars from
// S (staged in shared memory by the kernel).
template <bool TERMS, bool BATCH>
__device__ __forceinline__ void epilogue_cells_begin(const EpiArgs& A, const DevCtl*& ctl, ResolvedOp& r,
                                                     const float*& m, float** dbg, long long& mo, long long& ns,
                                                     float& dtth) {
    const int sim = BATCH ? (int)blockIdx.y : 0;
    const long long off = BATCH ? (long long)sim * A.P.bstride : 0;
    mo = BATCH ? (long long)sim * A.P.mask_bstride : 0;
    ctl = A.ctl ? A.ctl + sim : nullptr;
    const int cur = ctl ? ctl->cur : 0;
    const float h = ctl ? (float)ctl->h : 0.f;
    ns = ctl ? ctl->noise_step : A.noise_step;
    dtth = ctl ? (float)(ctl->dt_thermal > 0 ? ctl->dt_thermal : ctl->dt) : (float)A.dt_thermal;
    resolve_op(A.op, cur, h, r, off);
    m = A.op.m_in.get(cur) + off;
    if (TERMS)
        for (int q = 0; q < 6; q++) dbg[q] = at_off(A.dbg[q], off);
}

// PointwiseUpdater.Update (update_pointwise.go:30-88): first row with time >= t, linear
// interpolation from the row before; 0 at or before the first row; false past the last.
__device__ bool table_value(const FieldParams::TimeTable& T, double t, double out[3]) {
    int i = 0;
    while (i < T.n && T.rows[4 * i] < t) i++;
    if (i >= T.n) return false;
    if (i == 0) {
        out[0] = out[1] = out[2] = 0.0;
        return true;
    }
    const double* a = T.rows + 4 * (i - 1);
    const double* b = T.rows + 4 * i;
    const double f = (t - a[0]) / (b[0] - a[0]);
    for (int c = 0; c < 3; c++) out[c] = a[1 + c] + f * (b[1 + c] - a[1 + c]);
    return true;
}

// The block's simulation scalars for the staged (shared-memory) variants: the
// simulation's entry, with B_ext and j from their time tables at this evaluation's time.
// Called by one thread.
__device__ void stage_scalars(const EpiArgs& A, const DevCtl* ctl, SimScalars& s) {
    s = A.P.sims ? A.P.sims[blockIdx.y] : A.P.s;
    if (A.P.tab[0].n || A.P.tab[1].n) {
        const double t = ctl ? ctl->t + A.op.c_time * ctl->dt : A.t_eval;
        double v[3];
        bool ok = true;
        if (A.P.tab[0].n) {
            ok = table_value(A.P.tab[0], t, v) && ok;
            for (int c = 0; c < 3; c++) s.hz[c] = (float)(v[c] / 1.2566370614359172e-06);
        }
        if (A.P.tab[1].n) {
            ok = table_value(A.P.tab[1], t, v) && ok;
            for (int c = 0; c < 3; c++) s.jmul[c] = (float)v[c];
        }
        if (!ok && ctl) atomicExch(&const_cast<DevCtl*>(ctl)->status, (int)MM_ERR_RANGE);
    }
}

template <bool BATCH>
__device__ __forceinline__ const SimScalars& pick_scalars(const SimScalars& staged, const SimScalars& single) {
    if constexpr (BATCH) return staged;
    else return single;
}

// ---------------------------------------------------------------- C2R row pass + epilogue
// Cells of the block's rows; H_demag of (row, c) at cell x is element x>>1 (real part for
// even x, imaginary part for odd x) of shared-memory line (lrow*3 + c), stride LS.
// FWD: float x of line (lrow, c) then takes the cell's next state (times the Msat mask
// when A.fwd_mask) for the R2C rows of the next evaluation (four-step lines only).
template <bool TERMS, bool PADDED, bool BATCH, bool FWD = false, int SPEC = 0>
__device__ __forceinline__ void epilogue_rows(const EpiArgs& A, const SimScalars& S, const float2* sm, int LS,
                                              int row0, int nrow_here) {
    static_assert(!(FWD && (PADDED || TERMS)), "row output: four-step lines, no per-term outputs");
    const int n1 = A.P.n[1], n2 = A.P.n[2];
    const DevCtl* ctl;
    ResolvedOp r;
    const float* m;
    float* dbg[6];
    long long mo, ns;
    float dtth;
    epilogue_cells_begin<TERMS, BATCH>(A, ctl, r, m, dbg, mo, ns, dtth);
    ThreadRed tr = {0.f, 0.f, 0, {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}}};
    // (lrow, x) of element e = threadIdx.x + k*blockDim.x, advanced without divisions
    const int total = nrow_here * n2;
    int lrow = threadIdx.x / n2, x = threadIdx.x - lrow * n2;
    const int dr = blockDim.x / n2, dx = blockDim.x - dr * n2;
    int grow = row0 + lrow;
    int z = grow / n1, y = grow - z * n1;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const long long i = (long long)grow * n2 + x;
        const int pi = PADDED ? padx(x >> 1) : (x >> 1);
        const float2 v0 = sm[(lrow * 3 + 0) * LS + pi];
        const float2 v1 = sm[(lrow * 3 + 1) * LS + pi];
        const float2 v2 = sm[(lrow * 3 + 2) * LS + pi];
        const float3 hd = (x & 1) ? make_float3(v0.y, v1.y, v2.y) : make_float3(v0.x, v1.x, v2.x);
        if constexpr (FWD) {
            // float x of line (lrow, c) held H_demag of this cell only
            float3 nx = make_float3(0.f, 0.f, 0.f);
            process_cell<TERMS, SPEC>(A, S, m, r, dbg, i, mo, z, y, x, hd, ns, dtth, tr, &nx);
            float* fl = reinterpret_cast<float*>(const_cast<float2*>(sm)) + 2 * (long long)(lrow * 3) * LS + x;
            fl[0] = nx.x;
            fl[2 * LS] = nx.y;
            fl[4 * LS] = nx.z;
        } else {
            process_cell<TERMS, SPEC>(A, S, m, r, dbg, i, mo, z, y, x, hd, ns, dtth, tr);
        }
        // advance by blockDim.x cells
        x += dx;
        int adv = dr;
        if (x >= n2) { x -= n2; adv++; }
        lrow += adv;
        grow += adv;
        y += adv;
        while (y >= n1) { y -= n1; z++; }
    }
    block_reduce_publish(tr, A.op, const_cast<DevCtl*>(ctl), A.tq_out, A.red);
}

// Stockham variant (any power-of-two M up to 2048; single-simulation plans)
template <int M, bool TERMS>
__global__ void __launch_bounds__(512) xinv_epi_kernel(const float2* __restrict__ S, int hp, int L1,
                                                       const float2* __restrict__ tw, EpiArgs A) {
    const DevCtl* ctl = A.ctl ? A.ctl + blockIdx.y : nullptr;
    if (skip_eval(ctl, A.skip_retry)) return;
    S += blockIdx.y * A.spec_bstride;
    constexpr int TPL = tpl(M);
    constexpr int LL = line_len(M);
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int n0 = A.P.n[0], n1 = A.P.n[1];
    const int nrows = n0 * n1;
    const int rpb = blockDim.x / (3 * TPL);
    const int lr = threadIdx.x / (3 * TPL);
    const int c = (threadIdx.x / TPL) % 3;
    const int t = threadIdx.x % TPL;
    const int row = blockIdx.x * rpb + lr;
    const bool active = (lr < rpb) && (row < nrows);
    float2* xl = sm + (lr < rpb ? lr * 3 + c : 0) * LL;
    if (active) {
        const int z = row / n1, y = row % n1;
        const float2* src = S + ((long long)(c * n0 + z) * L1 + y) * hp;
        // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k]),  W = exp(-2 pi i / 2M)
        for (int k = t; k < M; k += TPL) {
            float2 a = src[k], b = src[M - k];
            float2 s = make_float2(a.x + b.x, a.y - b.y);
            float2 d = make_float2(a.x - b.x, a.y + b.y);
            float2 w = TwSrc<+1, float2>::get(tw, k, 2 * M);
            float2 wd = cmul(w, d);
            xl[padx(k)] = make_float2(s.x - wd.y, s.y + wd.x);
        }
    }
    __syncthreads();
    fft_line<M, +1, float2>(xl, t, active, tw);
    const int row0 = blockIdx.x * rpb;
    epilogue_rows<TERMS, true, false>(A, A.P.s, sm, LL, row0, min(rpb, nrows - row0));
}

// Four-step variant (4 <= M <= 1024): the pre-processed spectrum goes straight from
// global memory into registers, one shared-memory transpose, the result is written to
// shared memory in natural order for the epilogue.
template <int M>
__host__ __device__ constexpr int xinv4_rpb() {
    return (384 / (3 * FS<M>::P2)) > 0 ? 384 / (3 * FS<M>::P2) : 1;
}

// Rows per block of the four-step epilogue: the default, or half of it (the autotuner's
// other variant; at least 32 threads).  A compile-time constant, so that the row loops
// of the epilogue unroll and its register budget stays that of a fixed tile.
template <int M, bool HALF>
__host__ __device__ constexpr int xinv4_rows_c() {
    return (HALF && xinv4_rpb<M>() >= 2 && (xinv4_rpb<M>() / 2) * 3 * FS<M>::P2 >= 32) ? xinv4_rpb<M>() / 2
                                                                                          : xinv4_rpb<M>();
}

// R2C rows from the block's shared-memory lines: float x of the line of (row, c) holds the
// input at cell x (n_in reals; the rest of the length-2M row is zero).  The packing,
// four-step transform and real-to-complex post-processing of xfwd4_kernel, value for
// value, so dst (the line's spectrum row, hp >= M+1 complex; ignored when !active) gets
// what the separate row pass would write from the same values.  The post-processing
// twiddles W_2M^-k, k <= M/2, go to shared memory after the step-1 table (the launchers
// size the shared memory for them).  All threads of the block call this.
template <int M>
__device__ __forceinline__ void r2c_staged_lines(float2 (&v)[FS<M>::P1], float2* buf, float2* twt,
                                                 const float2* __restrict__ tw, int t, bool active, int n_in,
                                                 float2* dst) {
    using F = FS<M>;
    float2* pw = twt + F::TWT;
    for (int k = threadIdx.x; k <= M / 2; k += blockDim.x) pw[k] = TwSrc<-1, float2>::get(tw, k, 2 * M);
    __syncthreads();
    const float* fl = reinterpret_cast<const float*>(buf);
#pragma unroll
    for (int j = 0; j < F::P1; j++) {
        const int n = F::in_index(t, j);
        float2 val = make_float2(0.f, 0.f);
        if (active && 2 * n + 1 < n_in) val = buf[n];          // the packed pair (x[2n], x[2n+1])
        else if (active && 2 * n < n_in) val.x = fl[2 * n];
        v[j] = val;
    }
    __syncthreads();
    F::template run<-1>(v, buf, t, active, twt, 1);
    if (active) {
#pragma unroll
        for (int r = 0; r < F::P1; r++) buf[F::out_index(t, r)] = v[r];
    }
    __syncthreads();
    if (active) {
        for (int k = t; k <= M / 2; k += F::P2) {
            const float2 zk = buf[k & (M - 1)];
            const float2 zm = buf[(M - k) & (M - 1)];
            const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 od = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
            const float2 w = pw[k];
            dst[k] = cadd(e, cmul(w, od));
            if (k != M - k) dst[M - k] = cadd(cconj(e), cmul(make_float2(-w.x, w.y), cconj(od)));
        }
    }
}

// The spectrum argument of the C2R + epilogue pass: read-only, except in the FWD variant,
// which writes the R2C rows of the next stage state back into the rows it has read.
template <bool FWD> struct SpecIn { using type = const float2* __restrict__; };
template <> struct SpecIn<true> { using type = const float2*; };

// L2 prefetch of the stage inputs (base, kp, ep) that the epilogue of rows
// [row0, row0 + nrow) will read.  Issued at the start of the block, so the lines arrive
// while its spectrum is loaded and transformed; the epilogue reads them only after it has
// stored k (the pointers may alias), one dependent round trip per cell that now hits L2.
// Measured on the 256x256x16 film: RK23 step 505 -> 497-498 us.  Prefetching m and its
// exchange neighbours as well made the standalone evaluation slower (45.8 -> 47.5 us).
// Hints only: every address is a cell of the named rows.
__device__ __forceinline__ void prefetch_l2_range(const float* p, long long n) {
    if (!p || n <= 0) return;
    const long long lines = (n * 4 + 127) / 128;
    for (long long l = threadIdx.x; l < lines; l += blockDim.x) {
        const long long e = l * 32 < n - 1 ? l * 32 : n - 1;
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p + e));
    }
}

template <bool BATCH>
__device__ __forceinline__ void prefetch_epilogue_rows(const EpiArgs& A, int row0, int nrow) {
    // only plans of 2^18 cells and more: on the small single-simulation films the prefetch
    // lengthens each latency-bound launch (RK45 Neel wall 512x128x1: 4784 -> 4594 steps/s)
    if (nrow <= 0 || A.P.N * (long long)gridDim.y < (1LL << 18)) return;
    const int sim = BATCH ? (int)blockIdx.y : 0;
    const long long off = BATCH ? (long long)sim * A.P.bstride : 0;
    const DevCtl* ctl = A.ctl ? A.ctl + sim : nullptr;
    const int cur = ctl ? ctl->cur : 0;
    const long long N = A.P.N, n2 = A.P.n[2];
    const StageOp& op = A.op;
    const long long c0 = (long long)row0 * n2, nc = (long long)nrow * n2;
    auto streams3 = [&](const float* q) {
        if (!q) return;
        for (int c = 0; c < 3; c++) prefetch_l2_range(q + off + c * N + c0, nc);
    };
    if (op.do_combine && !op.base_is_cur) streams3(op.base.get(cur));
    for (int j = 0; j < op.nk && j < MM_MAXK; j++)
        if (j != op.kcur) streams3(op.kp[j].get(cur));
    for (int j = 0; j < op.ne && j < MM_MAXK; j++)
        if (j != op.ecur) streams3(op.ep[j].get(cur));
}

template <int M, bool TERMS, bool BATCH, bool HALF, bool FWD, int SPEC>
__device__ __forceinline__ void xinv4_epi_body(typename SpecIn<FWD>::type S, int hp, int L1,
                                               const float2* __restrict__ tw, const EpiArgs& A) {
    pdl_begin();
    constexpr int RPB = xinv4_rows_c<M, HALF>();
    const DevCtl* ctl = A.ctl ? A.ctl + blockIdx.y : nullptr;
    if (skip_eval(ctl, A.skip_retry)) return;
    S += blockIdx.y * A.spec_bstride;
    {
        const int nr = A.P.n[0] * A.P.n[1] - (int)blockIdx.x * RPB;
        prefetch_epilogue_rows<BATCH>(A, (int)blockIdx.x * RPB, nr < RPB ? nr : RPB);
    }
    __shared__ SimScalars s_sim;  // this simulation's scalars (BATCH); covered by the barriers below
    if (BATCH && threadIdx.x == 0) stage_scalars(A, ctl, s_sim);
    using F = FS<M>;
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int n0 = A.P.n[0], n1 = A.P.n[1];
    const int nrows = n0 * n1;
    const int t = threadIdx.x % F::P2;
    const int c = (threadIdx.x / F::P2) % 3;
    const int lr = threadIdx.x / (3 * F::P2);
    const int row = blockIdx.x * RPB + lr;
    const bool active = (lr < RPB) && (row < nrows);
    float2* buf = sm + (lr < RPB ? lr * 3 + c : 0) * F::LBUF;
    float2* twt = sm + RPB * 3 * F::LBUF;
    F::fill_twiddles(twt, tw);
    float2 v[F::P1];
    {
        const int rr = active ? row : 0;
        const int z = rr / n1, y = rr % n1;
        const float2* src = S + ((long long)(c * n0 + z) * L1 + y) * hp;
#pragma unroll
        for (int j = 0; j < F::P1; j++) {
            const int k = F::in_index(t, j);
            float2 val = make_float2(0.f, 0.f);
            if (active) {
                const float2 a = src[k], b = src[M - k];
                const float2 s = make_float2(a.x + b.x, a.y - b.y);
                const float2 d = make_float2(a.x - b.x, a.y + b.y);
                const float2 wd = cmul(TwSrc<+1, float2>::get(tw, k, 2 * M), d);
                val = make_float2(s.x - wd.y, s.y + wd.x);
            }
            v[j] = val;
        }
    }
    __syncthreads();
    F::template run<+1>(v, buf, t, active, twt, 1);
    if (active) {
#pragma unroll
        for (int r = 0; r < F::P1; r++) buf[F::out_index(t, r)] = v[r];
    }
    __syncthreads();
    const int row0 = blockIdx.x * RPB;
    epilogue_rows<TERMS, false, BATCH, FWD, SPEC>(A, pick_scalars<BATCH>(s_sim, A.P.s), sm, F::LBUF, row0,
                                            min(RPB, nrows - row0));
    if constexpr (FWD) {
        // R2C rows of the next stage state (float x of line (lr, c) = its value at cell x,
        // staged by epilogue_rows) into the rows of the spectrum this block has read
        float2* dst = nullptr;
        if (active) {
            const int z = row / n1, y = row % n1;
            dst = A.fwd + blockIdx.y * A.spec_bstride + ((long long)(c * n0 + z) * L1 + y) * hp;
        }
        r2c_staged_lines<M>(v, buf, twt, tw, t, active, A.P.n[2], dst);
    }
}

// Single plans: launch bounds alone, so ptxas sizes the registers for the 384-thread tile
// (78-80 registers; the SPEC_LEAN epilogue 56-69); batched plans: two blocks per SM requested
// explicitly (their staged-scalar variant would otherwise take 136-150 registers and one
// block).
template <int M, bool TERMS, bool HALF, bool FWD, int SPEC>
__global__ void __launch_bounds__(384) xinv4_epi_kernel(typename SpecIn<FWD>::type S, int hp, int L1,
                                                        const float2* __restrict__ tw, EpiArgs A) {
    xinv4_epi_body<M, TERMS, false, HALF, FWD, SPEC>(S, hp, L1, tw, A);
}

// The SPEC_LEAN epilogue without the next stage's rows fits 56 registers: three blocks per SM
// requested (RK23 film step 478 -> 476 us; the variant that writes the rows spills at 56
// and keeps the kernel above, two blocks per SM).
template <int M, bool HALF>
__global__ void __launch_bounds__(384, 3) xinv4_epi_lean3_kernel(const float2* __restrict__ S, int hp, int L1,
                                                                 const float2* __restrict__ tw, EpiArgs A) {
    xinv4_epi_body<M, false, false, HALF, false, SPEC_LEAN>(S, hp, L1, tw, A);
}

template <int M, bool TERMS, bool HALF, bool FWD, int SPEC>
__global__ void __launch_bounds__(384, M <= 512 ? 2 : 1) xinv4_epi_batch_kernel(typename SpecIn<FWD>::type S,
                                                                                int hp, int L1,
                                                                                const float2* __restrict__ tw,
                                                                                EpiArgs A) {
    xinv4_epi_body<M, TERMS, true, HALF, FWD, SPEC>(S, hp, L1, tw, A);
}

// ---------------------------------------------------------------- stage combine + R2C rows
// The first stage state of an attempt, formed as combine_kernel forms it (same operations
// in the same order), written to A.next and, times the Msat mask when fwd_mask, turned
// into its R2C rows in the spectrum: the attempt's first evaluation then starts at its
// column pass.  Blocks and threads as the four-step C2R + epilogue pass: RPB rows (z, y)
// per block, P2 threads per (row, component) line.
template <int M>
__global__ void __launch_bounds__(384) combine_rows_kernel(CombineArgs A, int n0, int n1, int n2, float2* S, int hp,
                                                           int L1, long long spec_bstride,
                                                           const float2* __restrict__ tw, int fwd_mask) {
    pdl_begin();
    constexpr int RPB = xinv4_rows_c<M, false>();
    using F = FS<M>;
    const DevCtl* ctl = A.ctl + blockIdx.y;
    if (ctl->done) return;
    const int cur = ctl->cur;
    const long long off = blockIdx.y * A.bstride;
    const float* base = A.base.get(cur) + off;
    float* next = A.next.get(cur) + off;
    const float* msk = A.msat_mask ? A.msat_mask + blockIdx.y * A.mask_bstride : nullptr;
    const float* kp[MM_MAXK];
    float ak[MM_MAXK];
#pragma unroll
    for (int j = 0; j < MM_MAXK; j++) {
        kp[j] = j < A.nk ? A.kp[j].get(cur) + off : nullptr;
        ak[j] = j < A.nk ? (float)(A.ak[j] * ctl->h) : 0.f;
    }
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    float* slots = reinterpret_cast<float*>(sm);
    float2* twt = sm + RPB * 3 * F::LBUF;
    F::fill_twiddles(twt, tw);
    const long long N = A.N;
    const int nrows = n0 * n1;
    const int row0 = blockIdx.x * RPB;
    const int here = min(RPB, nrows - row0);
    for (int e = threadIdx.x; e < here * n2; e += blockDim.x) {
        const int lrow = e / n2, x = e - lrow * n2;
        const long long i = (long long)(row0 + lrow) * n2 + x;
        float xv = base[i], yv = base[N + i], zv = base[2 * N + i];
#pragma unroll
        for (int j = 0; j < MM_MAXK; j++) {
            if (j >= A.nk) break;
            xv += ak[j] * kp[j][i];
            yv += ak[j] * kp[j][N + i];
            zv += ak[j] * kp[j][2 * N + i];
        }
        const float norm = msk ? msk[i] : 1.0f;
        const float mn = sqrtf(xv * xv + yv * yv + zv * zv);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        const float3 nx = make_float3(xv * sc, yv * sc, zv * sc);
        next[i] = nx.x;
        next[N + i] = nx.y;
        next[2 * N + i] = nx.z;
        const float fm = fwd_mask ? norm : 1.0f;
        float* fl = slots + 2 * (long long)(lrow * 3) * F::LBUF + x;
        fl[0] = nx.x * fm;
        fl[2 * F::LBUF] = nx.y * fm;
        fl[4 * F::LBUF] = nx.z * fm;
    }
    __syncthreads();
    const int t = threadIdx.x % F::P2;
    const int c = (threadIdx.x / F::P2) % 3;
    const int lr = threadIdx.x / (3 * F::P2);
    const int row = row0 + lr;
    const bool active = (lr < RPB) && (row < nrows);
    float2* buf = sm + (lr < RPB ? lr * 3 + c : 0) * F::LBUF;
    float2* dst = nullptr;
    if (active) {
        const int z = row / n1, y = row % n1;
        dst = S + blockIdx.y * spec_bstride + ((long long)(c * n0 + z) * L1 + y) * hp;
    }
    float2 v[F::P1];
    r2c_staged_lines<M>(v, buf, twt, tw, t, active, n2, dst);
}

template <int M>
static cudaError_t launch_combine_rows_t(const CombineArgs& A, const int n[3], float2* S, int hp, int L1,
                                         long long spec_bstride, const float2* tw, int fwd_mask, int nsim,
                                         cudaStream_t st) {
    constexpr int RPB = xinv4_rows_c<M, false>();
    const size_t smem = (size_t)(RPB * 3 * FS<M>::LBUF + FS<M>::TWT + M / 2 + 1) * sizeof(float2);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(combine_rows_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (n[0] * n[1] + RPB - 1) / RPB;
    int threads = RPB * 3 * FS<M>::P2;
    if (threads < 32) threads = 32;
    return launch_pdl(combine_rows_kernel<M>, dim3((unsigned)blocks, (unsigned)nsim), dim3(threads), smem, st, A, n[0],
                      n[1], n[2], S, hp, L1, spec_bstride, tw, fwd_mask);
}

cudaError_t launch_combine_rows(int M, const CombineArgs& A, const int n[3], float2* S, int hp, int L1,
                                long long spec_bstride, const float2* tw, int fwd_mask, int nsim, cudaStream_t st) {
    if (A.no_norm || A.nk > MM_MAXK) return cudaErrorInvalidValue;
    switch (M) {
#define X(m) case m: return launch_combine_rows_t<m>(A, n, S, hp, L1, spec_bstride, tw, fwd_mask, nsim, st);
        X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

static bool staged_scalars(const EpiArgs& A, int nsim);

// ---------------------------------------------------------------- fused single-layer evaluation
// One block per simulation of a single-layer film (n0 = 1) whose half spectrum
// [3][N1][M+1] fits in shared memory: the R2C rows, the y transform with the kernel
// multiply and its inverse, the C2R rows and the epilogue all run in one launch, and the
// spectrum never leaves the SM.  Each phase uses the same four-step transforms and the
// same arithmetic as the separate passes (xfwd4, colmul4, xinv4), so the results are
// identical to theirs.  L1 = 2 N1 (padded column length), M = N2 (complex row length).
template <int L1, int M>
struct Fused2D {
    using FR = FS<M>;
    using FC = FS<L1>;
    static constexpr int N1 = L1 / 2;
    static constexpr int HP = M + 1;                             // spectrum row pitch (odd)
    static constexpr int SPEC = 3 * N1 * HP;                     // float2
    static constexpr int LPP = 512 / FR::P2;                     // row lines per pass
    static constexpr int CC = (512 / (3 * FC::P2)) < 32 ? 512 / (3 * FC::P2) : 32;  // columns per batch
    static constexpr int CSTR = FC::LBUF + ((FC::LBUF & 1) ? 0 : 1);                 // column line stride
    static constexpr int RR = 512 / (3 * FR::P2);                // epilogue rows per chunk
    static constexpr int W1 = LPP * FR::LBUF, W2 = 3 * CC * CSTR, W3 = 3 * RR * FR::LBUF;
    static constexpr int WORK = W1 > W2 ? (W1 > W3 ? W1 : W3) : (W2 > W3 ? W2 : W3);
    static constexpr int TOTAL = SPEC + WORK + FR::TWT + FC::TWT;  // float2
    static constexpr size_t BYTES = (size_t)TOTAL * sizeof(float2);
};

template <int L1, int M, bool BATCH>
__global__ void __launch_bounds__(512, 1) fused2d_kernel(const float* __restrict__ in_mask, long long mask_bstride,
                                                         KernelView K, float scale, const float* __restrict__ sim_scale,
                                                         const float2* __restrict__ tw, EpiArgs A) {
    using G = Fused2D<L1, M>;
    using FR = typename G::FR;
    using FC = typename G::FC;
    constexpr int N1 = G::N1, HP = G::HP;
    const int sim = blockIdx.y;
    const DevCtl* ctl = A.ctl ? A.ctl + sim : nullptr;
    if (skip_eval(ctl, A.skip_retry)) return;
    __shared__ SimScalars s_sim;
    if (BATCH && threadIdx.x == 0) stage_scalars(A, ctl, s_sim);
    if (sim_scale) scale = sim_scale[sim];
    extern __shared__ unsigned char smem_raw[];
    float2* sp = reinterpret_cast<float2*>(smem_raw);        // [3][N1][HP]
    float2* work = sp + G::SPEC;
    float2* twr = work + G::WORK;
    float2* twc = twr + FR::TWT;
    FR::fill_twiddles(twr, tw);
    FC::fill_twiddles(twc, tw);
    const int N2 = A.P.n[2];
    const long long N = (long long)N1 * N2;
    const float* m = A.op.m_in.get(ctl ? ctl->cur : 0) + (long long)sim * 3 * N;
    const float* msk = in_mask ? in_mask + (long long)sim * mask_bstride : nullptr;
    const int tid = threadIdx.x;

    // ---- 1. R2C rows: (c, y) lines of 2M reals (N2 of them non-zero), packed complex
    {
        const int t = tid % FR::P2, ll = tid / FR::P2;
        float2* buf = work + ll * FR::LBUF;
        for (int l0 = 0; l0 < 3 * N1; l0 += G::LPP) {
            const int l = l0 + ll;
            const bool active = l < 3 * N1;
            const int c = active ? l / N1 : 0, y = active ? l - c * N1 : 0;
            const float* src = m + c * N + (long long)y * N2;
            const float* mr = msk ? msk + (long long)y * N2 : nullptr;
            float2 v[FR::P1];
#pragma unroll
            for (int j = 0; j < FR::P1; j++) {
                const int n = FR::in_index(t, j);
                float a = 0.f, b = 0.f;
                if (active) {
                    if (2 * n < N2) a = src[2 * n] * (mr ? mr[2 * n] : 1.f);
                    if (2 * n + 1 < N2) b = src[2 * n + 1] * (mr ? mr[2 * n + 1] : 1.f);
                }
                v[j] = make_float2(a, b);
            }
            __syncthreads();
            FR::template run<-1>(v, buf, t, active, twr, 1);
            if (active) {
#pragma unroll
                for (int r = 0; r < FR::P1; r++) buf[FR::out_index(t, r)] = v[r];
            }
            __syncthreads();
            if (active) {
                float2* dst = sp + (c * N1 + y) * HP;
                for (int k = t; k <= M / 2; k += FR::P2) {
                    const float2 zk = buf[k & (M - 1)];
                    const float2 zm = buf[(M - k) & (M - 1)];
                    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
                    const float2 od = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
                    const float2 w = TwSrc<-1, float2>::get(tw, k, 2 * M);
                    dst[k] = cadd(e, cmul(w, od));
                    if (k != M - k) dst[M - k] = cadd(cconj(e), cmul(make_float2(-w.x, w.y), cconj(od)));
                }
            }
        }
    }
    __syncthreads();

    // ---- 2. columns: forward y transform, symmetric kernel multiply, inverse
    {
        constexpr int CC = G::CC, CSTR = G::CSTR;
        const int per = CC * FC::P2;
        const int c = tid / per, r = tid - c * per;
        const int col = r % CC, t = r / CC;
        float2* line = work + ((c < 3 ? c : 0) * CC + col) * CSTR;
        for (int kx0 = 0; kx0 < HP; kx0 += CC) {
            const bool active = c < 3 && kx0 + col < HP;
            const float2* colp = sp + (c < 3 ? c : 0) * N1 * HP + kx0 + col;
            float2 v[FC::P1];
#pragma unroll
            for (int j = 0; j < FC::P1; j++) {
                const int n = FC::in_index(t, j);
                v[j] = (active && n < N1) ? colp[n * HP] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            FC::template run<-1>(v, line, t, active, twc, CC);
            if (active) {
#pragma unroll
                for (int q = 0; q < FC::P1; q++) line[FC::out_index(t, q)] = v[q];
            }
            __syncthreads();
            const int nh = min(CC, HP - kx0);
            for (int e = tid; e < L1 * CC; e += blockDim.x) {
                const int ky = e / CC, c2 = e - ky * CC;
                if (c2 >= nh) continue;
                float kk[6];
                kernel_at(K, 0, ky, kx0 + c2, kk);
                float2* l0 = work + (0 * CC + c2) * CSTR + ky;
                float2* l1 = work + (1 * CC + c2) * CSTR + ky;
                float2* l2 = work + (2 * CC + c2) * CSTR + ky;
                const float2 m0 = *l0, m1 = *l1, m2 = *l2;
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
                for (int j = 0; j < FC::P1; j++) v[j] = line[FC::in_index(t, j)];
            }
            __syncthreads();
            FC::template run<+1>(v, line, t, active, twc, CC);
            if (active) {
                float2* cold = sp + c * N1 * HP + kx0 + col;
#pragma unroll
                for (int q = 0; q < FC::P1; q++) {
                    const int n = FC::out_index(t, q);
                    if (n < N1) cold[n * HP] = v[q];
                }
            }
            __syncthreads();
        }
    }

    // ---- 3. C2R rows in chunks of RR, each followed by the epilogue of its rows
    {
        constexpr int RR = G::RR;
        const int t = tid % FR::P2;
        const int c = (tid / FR::P2) % 3;
        const int lr = tid / (3 * FR::P2);
        float2* buf = work + (lr < RR ? lr * 3 + c : 0) * FR::LBUF;
        const SimScalars& S = pick_scalars<BATCH>(s_sim, A.P.s);
        for (int row0 = 0; row0 < N1; row0 += RR) {
            const int row = row0 + lr;
            const bool active = lr < RR && row < N1;
            const float2* src = sp + (c * N1 + (active ? row : 0)) * HP;
            float2 v[FR::P1];
#pragma unroll
            for (int j = 0; j < FR::P1; j++) {
                const int k = FR::in_index(t, j);
                float2 val = make_float2(0.f, 0.f);
                if (active) {
                    const float2 a = src[k], b = src[M - k];
                    const float2 s = make_float2(a.x + b.x, a.y - b.y);
                    const float2 d = make_float2(a.x - b.x, a.y + b.y);
                    const float2 wd = cmul(TwSrc<+1, float2>::get(tw, k, 2 * M), d);
                    val = make_float2(s.x - wd.y, s.y + wd.x);
                }
                v[j] = val;
            }
            __syncthreads();
            FR::template run<+1>(v, buf, t, active, twr, 1);
            if (active) {
#pragma unroll
                for (int r = 0; r < FR::P1; r++) buf[FR::out_index(t, r)] = v[r];
            }
            __syncthreads();
            epilogue_rows<false, false, BATCH>(A, S, work, FR::LBUF, row0, min(RR, N1 - row0));
            __syncthreads();
        }
    }
}

// Whether the fused evaluation serves a single-layer geometry (n0 = 1, power-of-two N1,
// N2 in 32..128 with N1 <= 64) within 227 KB of shared memory.
bool fused2d_ok(const int n[3]) {
    if (n[0] != 1) return false;
    const int L1 = 2 * n[1], M = n[2];
    size_t bytes = 0;
#define F2(l, mm) if (L1 == l && M == mm) bytes = Fused2D<l, mm>::BYTES;
    F2(32, 32) F2(32, 64) F2(32, 128) F2(64, 32) F2(64, 64) F2(64, 128) F2(128, 32) F2(128, 64) F2(128, 128)
#undef F2
    return bytes > 0 && bytes <= 227 * 1024;
}

template <int L1, int M>
static cudaError_t launch_fused2d_t(const float* in_mask, long long mask_bstride, const KernelView& K, float scale,
                                    const float* sim_scale, const float2* tw, const EpiArgs& A, bool batch,
                                    cudaStream_t st, int nsim) {
    using G = Fused2D<L1, M>;
    auto kern = batch ? fused2d_kernel<L1, M, true> : fused2d_kernel<L1, M, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::BYTES);
    if (e != cudaSuccess) return e;
    kern<<<dim3(1u, (unsigned)nsim), 512, G::BYTES, st>>>(in_mask, mask_bstride, K, scale, sim_scale, tw, A);
    return cudaGetLastError();
}

cudaError_t launch_fused2d(const float* in_mask, long long mask_bstride, const KernelView& K, float scale,
                           const float* sim_scale, const float2* tw, const EpiArgs& A, cudaStream_t st, int* nblocks,
                           int nsim) {
    const int L1 = 2 * A.P.n[1], M = A.P.n[2];
    const bool batch = staged_scalars(A, nsim);
    *nblocks = 1;
#define F2(l, mm)                                                                                          \
    if (L1 == l && M == mm)                                                                                \
        return launch_fused2d_t<l, mm>(in_mask, mask_bstride, K, scale, sim_scale, tw, A, batch, st, nsim);
    F2(32, 32) F2(32, 64) F2(32, 128) F2(64, 32) F2(64, 64) F2(64, 128) F2(128, 32) F2(128, 64) F2(128, 128)
#undef F2
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------- epilogue without demag
template <bool TERMS, bool BATCH>
__global__ void __launch_bounds__(256) local_epi_kernel(EpiArgs A) {
    if (skip_eval(A.ctl ? A.ctl + blockIdx.y : nullptr, A.skip_retry)) return;
    const int n1 = A.P.n[1], n2 = A.P.n[2];
    __shared__ SimScalars s_sim;
    if (BATCH) {
        if (threadIdx.x == 0) stage_scalars(A, A.ctl ? A.ctl + blockIdx.y : nullptr, s_sim);
        __syncthreads();
    }
    const SimScalars& S = pick_scalars<BATCH>(s_sim, A.P.s);
    const DevCtl* ctl;
    ResolvedOp r;
    const float* m;
    float* dbg[6];
    long long mo, ns;
    float dtth;
    epilogue_cells_begin<TERMS, BATCH>(A, ctl, r, m, dbg, mo, ns, dtth);
    ThreadRed tr = {0.f, 0.f, 0, {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A.P.N;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % n2);
        const long long zy = i / n2;
        const int y = (int)(zy % n1), z = (int)(zy / n1);
        process_cell<TERMS>(A, S, m, r, dbg, i, mo, z, y, x, make_float3(0.f, 0.f, 0.f), ns, dtth, tr);
    }
    block_reduce_publish(tr, A.op, const_cast<DevCtl*>(ctl), A.tq_out, A.red);
}

// ---------------------------------------------------------------- launchers
template <int M, bool TERMS>
static cudaError_t launch_xinv_t(const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A, cudaStream_t st,
                                 int* nblocks, int nsim) {
    constexpr int TPL = tpl(M);
    int rpb = (3 * TPL >= 384) ? 1 : 384 / (3 * TPL);
    size_t smem = (size_t)rpb * 3 * line_len(M) * sizeof(float2);
    while (smem > 100 * 1024 && rpb > 1) { rpb /= 2; smem = (size_t)rpb * 3 * line_len(M) * sizeof(float2); }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(xinv_epi_kernel<M, TERMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int nrows = A.P.n[0] * A.P.n[1];
    int blocks = (nrows + rpb - 1) / rpb;
    int threads = rpb * 3 * TPL;
    if (threads < 32) threads = 32;
    *nblocks = blocks;
    xinv_epi_kernel<M, TERMS><<<dim3((unsigned)blocks, (unsigned)nsim), threads, smem, st>>>(S, hp, L1, tw, A);
    return cudaGetLastError();
}

// What the evaluation lacks, as SPEC_* bits: no per-cell mask of any kind, no thermal
// term, no Zhang-Li or Slonczewski term.
static int epilogue_spec(const FieldParams& P) {
    int spec = SPEC_NOMASK;
    if (!P.thermal) spec |= SPEC_NOTHERMAL;
    if (!P.zhangli && !P.slonczewski) spec |= SPEC_NOSTT;
    const float* masks[] = {P.msat_mask,      P.aex_mask,      P.alpha_mask,     P.ku_mask,        P.anisu_mask[0],
                            P.anisu_mask[1],  P.anisu_mask[2], P.bext_mask[0],   P.bext_mask[1],   P.bext_mask[2],
                            P.j_mask[0],      P.j_mask[1],     P.j_mask[2],      P.temp_mask,      P.xi_mask,
                            P.zl_pol_mask,    P.p_mask[0],     P.p_mask[1],      P.p_mask[2],      P.sl_pol_mask,
                            P.lambda_mask,    P.eps_prime_mask, P.t_fl_mask};
    for (const float* q : masks)
        if (q) spec &= ~SPEC_NOMASK;
    return spec;
}

// ---------------------------------------------------------------- mixed-radix C2R + epilogue
// Row lengths M that are not powers of two: the pre-processing of xinv_epi_kernel, the
// mixed-radix inverse transform of mixed.cuh, then the same epilogue.  rpb rows of three
// component lines per block (line (row, c) at sm + (row*3 + c)*M, natural order; the
// scratch lines follow), blockDim.x / (3 rpb) threads per line.  BATCH: the simulation's
// scalars are staged in shared memory (batched plans, time tables).
template <bool TERMS, bool BATCH, int SPEC>
__global__ void __launch_bounds__(384) mr_xinv_epi_kernel(const float2* __restrict__ S, int hp, int L1, MrLine f,
                                                          const float2* __restrict__ twM,
                                                          const float2* __restrict__ tw2M, EpiArgs A, int rpb) {
    const DevCtl* ctl = A.ctl ? A.ctl + blockIdx.y : nullptr;
    if (skip_eval(ctl, A.skip_retry)) return;
    S += blockIdx.y * A.spec_bstride;
    {
        const int nr = A.P.n[0] * A.P.n[1] - (int)blockIdx.x * rpb;
        prefetch_epilogue_rows<BATCH>(A, (int)blockIdx.x * rpb, nr < rpb ? nr : rpb);
    }
    __shared__ SimScalars s_sim;  // covered by the barriers of the transform
    if (BATCH && threadIdx.x == 0) stage_scalars(A, ctl, s_sim);
    const int M = f.L;
    const int nlines = 3 * rpb;
    const int nt = blockDim.x / nlines;
    const int li = threadIdx.x / nt, t = threadIdx.x % nt;
    const int lr = li / 3, c = li % 3;
    const int n0 = A.P.n[0], n1 = A.P.n[1];
    const int nrows = n0 * n1;
    const int row = blockIdx.x * rpb + lr;
    const bool active = (li < nlines) && (row < nrows);
    extern __shared__ unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int lc = li < nlines ? li : 0;
    float2* xl = sm + (size_t)lc * M;
    float2* scratch = sm + (size_t)(nlines + lc) * M;
    if (active) {
        const int z = row / n1, y = row % n1;
        const float2* src = S + ((long long)(c * n0 + z) * L1 + y) * hp;
        // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k]),  W = exp(-2 pi i / 2M)
        for (int k = t; k < M; k += nt) {
            const float2 a = src[k], b = src[M - k];
            const float2 s = make_float2(a.x + b.x, a.y - b.y);
            const float2 d = make_float2(a.x - b.x, a.y + b.y);
            const float2 w0 = tw2M[k];
            const float2 wd = cmul(make_float2(w0.x, -w0.y), d);
            xl[k] = make_float2(s.x - wd.y, s.y + wd.x);
        }
    }
    mr_fft<+1, float2>(xl, scratch, f, twM, t, nt, active);
    const int row0 = blockIdx.x * rpb;
    epilogue_rows<TERMS, false, BATCH, false, SPEC>(A, pick_scalars<BATCH>(s_sim, A.P.s), sm, M, row0,
                                                    min(rpb, nrows - row0));
}

// rows per block and threads per line of the mixed-radix epilogue
static void mr_xinv_shape(int M, int* rpb, int* nt) {
    *nt = M >= 256 ? 128 : (M >= 64 ? 64 : 32);
    *rpb = 384 / (3 * *nt) > 0 ? 384 / (3 * *nt) : 1;
    while (*rpb > 1 && (size_t)*rpb * 6 * M * sizeof(float2) > 96 * 1024) *rpb /= 2;
}

template <bool TERMS, bool BATCH>
static cudaError_t launch_mr_xinv_t(int M, const float2* S, int hp, int L1, const EpiArgs& A, cudaStream_t st,
                                    int* nblocks, int nsim) {
    MrLine f;
    const float2 *twM = nullptr, *tw2M = nullptr;
    if (!mr_factor(M, &f) || !mr_tables(M, &twM, nullptr) || !mr_tables(2 * M, &tw2M, nullptr))
        return cudaErrorInvalidValue;
    int rpb, nt;
    mr_xinv_shape(M, &rpb, &nt);
    const size_t smem = (size_t)rpb * 6 * M * sizeof(float2);
    // the epilogue without what the evaluation lacks (as the four-step pass chooses it)
    auto kern = mr_xinv_epi_kernel<TERMS, BATCH, 0>;
    if constexpr (!TERMS) {
        const int spec = epilogue_spec(A.P);
        constexpr int NOTS = SPEC_NOTHERMAL | SPEC_NOSTT, NOMS = SPEC_NOMASK | SPEC_NOSTT,
                      NOMT = SPEC_NOMASK | SPEC_NOTHERMAL;
        if (spec == SPEC_LEAN) kern = mr_xinv_epi_kernel<false, BATCH, SPEC_LEAN>;
        else if ((spec & NOTS) == NOTS) kern = mr_xinv_epi_kernel<false, BATCH, NOTS>;
        else if ((spec & NOMS) == NOMS) kern = mr_xinv_epi_kernel<false, BATCH, NOMS>;
        else if ((spec & NOMT) == NOMT) kern = mr_xinv_epi_kernel<false, BATCH, NOMT>;
    }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int nrows = A.P.n[0] * A.P.n[1];
    const int blocks = (nrows + rpb - 1) / rpb;
    *nblocks = blocks;
    kern<<<dim3((unsigned)blocks, (unsigned)nsim), 3 * rpb * nt, smem, st>>>(S, hp, L1, f, twM, tw2M, A, rpb);
    return cudaGetLastError();
}

template <int M>
static int xinv4_rows(int tile) {
    return tile < 0 ? xinv4_rows_c<M, true>() : xinv4_rows_c<M, false>();
}

template <int M, bool TERMS, bool BATCH, bool HALF, bool FWD>
static cudaError_t launch_xinv4_h(const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A,
                                  cudaStream_t st, int* nblocks, int nsim) {
    constexpr int RPB = xinv4_rows_c<M, HALF>();
    const size_t smem = (size_t)(RPB * 3 * FS<M>::LBUF + FS<M>::TWT + (FWD ? M / 2 + 1 : 0)) * sizeof(float2);
    // Single plans: the SPEC_LEAN kernels when nothing of the three is present, else the
    // kernel without what is absent of masks and thermal (see below), else the general one.  Batched plans: without thermal and spin-transfer terms (relaxation
    // pools, masks kept) or without masks and spin-transfer terms (thermal ensembles).
    const int spec = TERMS ? 0 : epilogue_spec(A.P);
    auto kern = xinv4_epi_kernel<M, TERMS, HALF, FWD, 0>;
    if (BATCH) {
        constexpr int NOTS = SPEC_NOTHERMAL | SPEC_NOSTT, NOMS = SPEC_NOMASK | SPEC_NOSTT;
        kern = xinv4_epi_batch_kernel<M, TERMS, HALF, FWD, 0>;
        if constexpr (!TERMS) {
            if ((spec & NOTS) == NOTS) kern = xinv4_epi_batch_kernel<M, false, HALF, FWD, NOTS>;
            else if ((spec & NOMS) == NOMS) kern = xinv4_epi_batch_kernel<M, false, HALF, FWD, NOMS>;
        }
    } else if (spec == SPEC_LEAN) {
        if constexpr (FWD) kern = xinv4_epi_kernel<M, false, HALF, true, SPEC_LEAN>;
        else kern = xinv4_epi_lean3_kernel<M, HALF>;
    } else if constexpr (!TERMS) {
        // masked films without thermal and spin-transfer terms; unmasked ones with a
        // spin-transfer term and no thermal one (the Neel wall under current)
        constexpr int NOTS = SPEC_NOTHERMAL | SPEC_NOSTT, NOMT = SPEC_NOMASK | SPEC_NOTHERMAL;
        if ((spec & NOTS) == NOTS) kern = xinv4_epi_kernel<M, false, HALF, FWD, NOTS>;
        else if ((spec & NOMT) == NOMT) kern = xinv4_epi_kernel<M, false, HALF, FWD, NOMT>;
    }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    // batched plans: two blocks per SM (the launch bounds) need the shared-memory carveout
    // as well; single plans keep the default split, whose larger L1 serves the stencil's
    // neighbour loads
    if (BATCH) {
        cudaError_t ec = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                              (int)cudaSharedmemCarveoutMaxShared);
        if (ec != cudaSuccess) return ec;
    }
    const int nrows = A.P.n[0] * A.P.n[1];
    const int blocks = (nrows + RPB - 1) / RPB;
    int threads = RPB * 3 * FS<M>::P2;
    if (threads < 32) threads = 32;
    *nblocks = blocks;
    return launch_pdl(kern, dim3((unsigned)blocks, (unsigned)nsim), dim3(threads), smem, st, S, hp, L1, tw, A);
}

template <int M, bool TERMS, bool BATCH, bool FWD>
static cudaError_t launch_xinv4_f(const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A,
                                  cudaStream_t st, int* nblocks, int nsim, int tile) {
    if (tile < 0 && xinv4_rows_c<M, true>() != xinv4_rows_c<M, false>())
        return launch_xinv4_h<M, TERMS, BATCH, true, FWD>(S, hp, L1, tw, A, st, nblocks, nsim);
    return launch_xinv4_h<M, TERMS, BATCH, false, FWD>(S, hp, L1, tw, A, st, nblocks, nsim);
}

// A.fwd selects the variant that also writes the R2C rows of the next stage state (no
// per-term outputs there; the host never asks for both).
template <int M, bool TERMS, bool BATCH>
static cudaError_t launch_xinv4_t(const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A,
                                  cudaStream_t st, int* nblocks, int nsim, int tile) {
    if constexpr (!TERMS) {
        if (A.fwd) return launch_xinv4_f<M, false, BATCH, true>(S, hp, L1, tw, A, st, nblocks, nsim, tile);
    } else {
        if (A.fwd) return cudaErrorInvalidValue;
    }
    return launch_xinv4_f<M, TERMS, BATCH, false>(S, hp, L1, tw, A, st, nblocks, nsim, tile);
}

static bool use_xinv4(int M) { return M >= 4 && M <= 1024 && mr_pow2(M); }

// The four-step epilogue (and the four-step row pass whose output it reproduces) serve
// these row lengths.
bool epi_r2c_supported(int M) { return use_xinv4(M); }

int xinv_blocks(int M, int n0n1) {
    if (!mr_pow2(M)) {
        int rpb, nt;
        mr_xinv_shape(M, &rpb, &nt);
        return (n0n1 + rpb - 1) / rpb;
    }
    if (use_xinv4(M)) {
        int rpb = 1;
        switch (M) {
#define X(m) case m: rpb = xinv4_rows<m>(-1); break;
            X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
        }
        return (n0n1 + rpb - 1) / rpb;
    }
    int TPL = mmfft::tpl(M);
    int rpb = (3 * TPL >= 384) ? 1 : 384 / (3 * TPL);
    size_t smem = (size_t)rpb * 3 * mmfft::line_len(M) * sizeof(float2);
    while (smem > 100 * 1024 && rpb > 1) { rpb /= 2; smem = (size_t)rpb * 3 * mmfft::line_len(M) * sizeof(float2); }
    return (n0n1 + rpb - 1) / rpb;
}

// Staged variants (scalars in shared memory) serve batched plans and time tables.
static bool staged_scalars(const EpiArgs& A, int nsim) { return nsim > 1 || A.P.tab[0].n || A.P.tab[1].n; }

cudaError_t launch_xinv_epi(int M, const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A, bool terms,
                            cudaStream_t st, int* nblocks, int nsim, int tile) {
    const bool staged = staged_scalars(A, nsim);
    if (use_xinv4(M)) {
        switch (M) {
#define X(m)                                                                      \
    case m:                                                                       \
        if (staged)                                                                     \
            return terms ? launch_xinv4_t<m, true, true>(S, hp, L1, tw, A, st, nblocks, nsim, tile)  \
                         : launch_xinv4_t<m, false, true>(S, hp, L1, tw, A, st, nblocks, nsim, tile); \
        return terms ? launch_xinv4_t<m, true, false>(S, hp, L1, tw, A, st, nblocks, 1, tile)     \
                     : launch_xinv4_t<m, false, false>(S, hp, L1, tw, A, st, nblocks, 1, tile);
            X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024)
#undef X
        }
    }
    if (!mr_pow2(M)) {  // not a power of two: the mixed-radix pass
        if (staged)
            return terms ? launch_mr_xinv_t<true, true>(M, S, hp, L1, A, st, nblocks, nsim)
                         : launch_mr_xinv_t<false, true>(M, S, hp, L1, A, st, nblocks, nsim);
        return terms ? launch_mr_xinv_t<true, false>(M, S, hp, L1, A, st, nblocks, 1)
                     : launch_mr_xinv_t<false, false>(M, S, hp, L1, A, st, nblocks, 1);
    }
    if (staged) return cudaErrorNotSupported;  // batched plans and time tables use the four-step pass
    switch (M) {
#define X(m)                                                                      \
    case m:                                                                       \
        return terms ? launch_xinv_t<m, true>(S, hp, L1, tw, A, st, nblocks, nsim)      \
                     : launch_xinv_t<m, false>(S, hp, L1, tw, A, st, nblocks, nsim);
        X(1) X(2) X(4) X(8) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048)
#undef X
        default: return cudaErrorInvalidValue;
    }
}

// blocks per simulation of the grid-stride cell kernels (about 16 per SM in total)
int local_blocks(long long N, int nsim) {
    long long b = (N + 255) / 256;
    long long cap = (148 * 16 + nsim - 1) / nsim;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_local_epi(const EpiArgs& A, bool terms, cudaStream_t st, int* nblocks, int nsim) {
    int b = local_blocks(A.P.N, nsim);
    *nblocks = b;
    const dim3 grid((unsigned)b, (unsigned)nsim);
    if (staged_scalars(A, nsim)) {
        if (terms) local_epi_kernel<true, true><<<grid, 256, 0, st>>>(A);
        else local_epi_kernel<false, true><<<grid, 256, 0, st>>>(A);
    } else {
        if (terms) local_epi_kernel<true, false><<<grid, 256, 0, st>>>(A);
        else local_epi_kernel<false, false><<<grid, 256, 0, st>>>(A);
    }
    return cudaGetLastError();
}

}  // namespace mm
