// compat.cu -- libmumax2-compatible entry points (include/libmumax2_compat.h).
//
// The reference's Go engine calls one exported C function per elementary operation
// (src/mumax/gpu/libmumax2.go); this file provides the same symbols, computing the
// same values, as grid-stride sm_100a kernels sized to the SM count.  The fused
// plan API (plan.cu) is the fast path; these keep the reference's own callers
// working unchanged.
#include <cstdio>
#include <cstdlib>

#include "../../include/libmumax2_compat.h"
#include "mm_internal.h"

namespace {

int g_ngpu = 0;
int g_ids[64];
int g_status = 0;

inline void note(cudaError_t e) {
    if (e != cudaSuccess && g_status == 0) g_status = (int)e;
}

inline int ndev() { return g_ngpu > 0 ? g_ngpu : 1; }
inline void setdev(int dev) {
    if (g_ngpu > 0) note(cudaSetDevice(g_ids[dev]));
}
inline cudaStream_t sget(CUstream* s, int dev) { return s ? (cudaStream_t)s[dev] : (cudaStream_t)0; }

inline int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 8) b = 148LL * 8;
    return (int)(b < 1 ? 1 : b);
}

#define GS_LOOP(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ float mk1(const float* m, long long i) { return m ? m[i] : 1.0f; }

// ---------------------------------------------------------------- torque.cu:13-57
__global__ void k_torque(float* tx, float* ty, float* tz, const float* mx, const float* my, const float* mz,
                         const float* hx, const float* hy, const float* hz, const float* amap, float amul, int N) {
    GS_LOOP(i, N) {
        float a = amap ? amul * amap[i] : amul;
        float Mx = mx[i], My = my[i], Mz = mz[i], Hx = hx[i], Hy = hy[i], Hz = hz[i];
        float cx = My * Hz - Hy * Mz, cy = -Mx * Hz + Hx * Mz, cz = Mx * Hy - Hx * My;
        float dx = -My * cz + cy * Mz, dy = Mx * cz - cx * Mz, dz = -Mx * cy + cx * My;
        float g = 1.0f / (1.0f + a * a);
        tx[i] = g * (cx + dx * a);
        ty[i] = g * (cy + dy * a);
        tz[i] = g * (cz + dz * a);
    }
}

// ---------------------------------------------------------------- exchange6.cu:12-142
__device__ __forceinline__ float fdz(float a, float b) { return (b == 0.0f) ? 0.0f : a / b; }
__device__ __forceinline__ float agz(float a, float b) {
    float s = a + b;
    return (s == 0.0f) ? 0.0f : 2.0f * a * b / s;
}
__global__ void k_exchange6(float* hx, float* hy, float* hz, const float* mx, const float* my, const float* mz,
                            const float* msat, const float* aex, float pre, int N0, int N1, int N2, int w0, int w1,
                            int w2, float c0, float c1, float c2) {
    const long long N = (long long)N0 * N1 * N2;
    GS_LOOP(I, N) {
        int k = (int)(I % N2);
        long long r = I / N2;
        int j = (int)(r % N1), i = (int)(r / N1);
        float lex0 = fdz(mk1(aex, I), mk1(msat, I));
        float m0[3] = {mx[I], my[I], mz[I]};
        float H[3] = {0.f, 0.f, 0.f};
        const int cc[3] = {i, j, k};
        const int nn[3] = {N0, N1, N2};
        const int ww[3] = {w0, w1, w2};
        const long long st[3] = {(long long)N1 * N2, N2, 1};
        const float cf[3] = {c0, c1, c2};
        // reference order: dimension 0, then 2, then 1
        const int order[3] = {0, 2, 1};
        for (int q = 0; q < 3; q++) {
            int d = order[q];
            int lo = cc[d] - 1;
            lo = (lo < 0 && ww[d]) ? nn[d] + lo : lo;
            lo = max(lo, 0);
            int hi = cc[d] + 1;
            hi = (hi == nn[d] && ww[d]) ? hi - nn[d] : hi;
            hi = min(hi, nn[d] - 1);
            long long il = I + (long long)(lo - cc[d]) * st[d];
            long long ih = I + (long long)(hi - cc[d]) * st[d];
            float l1 = agz(lex0, fdz(mk1(aex, il), mk1(msat, il)));
            float l2 = agz(lex0, fdz(mk1(aex, ih), mk1(msat, ih)));
            float a[3] = {mx[il], my[il], mz[il]}, b[3] = {mx[ih], my[ih], mz[ih]};
            for (int c = 0; c < 3; c++) H[c] += pre * cf[d] * (l1 * (a[c] - m0[c]) + l2 * (b[c] - m0[c]));
        }
        hx[I] = H[0];
        hy[I] = H[1];
        hz[I] = H[2];
    }
}

// ---------------------------------------------------------------- uniaxialanisotropy.cu:12-86
__global__ void k_uniaxial(float* hx, float* hy, float* hz, const float* mx, const float* my, const float* mz,
                           const float* ku, const float* msat, float kmul, const float* ux_, float uxm,
                           const float* uy_, float uym, const float* uz_, float uzm, int N) {
    GS_LOOP(i, N) {
        float ms = msat ? msat[i] : 1.0f;
        if (ms == 0.0f) ms = 1.0f;
        float k2 = ku ? (kmul / ms) * ku[i] : kmul / ms;
        float ux = ux_ ? uxm * ux_[i] : uxm, uy = uy_ ? uym * uy_[i] : uym, uz = uz_ ? uzm * uz_[i] : uzm;
        float mu = mx[i] * ux + my[i] * uy + mz[i] * uz;
        hx[i] = k2 * mu * ux;
        hy[i] = k2 * mu * uy;
        hz[i] = k2 * mu * uz;
    }
}

// ---------------------------------------------------------------- normalize.cu:14-42
__global__ void k_normalize(float* mx, float* my, float* mz, const float* norm_map, int N) {
    GS_LOOP(i, N) {
        float norm = norm_map ? norm_map[i] : 1.0f;
        float X = mx[i], Y = my[i], Z = mz[i];
        float mn = sqrtf(X * X + Y * Y + Z * Z);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        mx[i] = X * sc;
        my[i] = Y * sc;
        mz[i] = Z * sc;
    }
}

// ---------------------------------------------------------------- add.cu
__global__ void k_add(float* d, const float* a, const float* b, int N) { GS_LOOP(i, N) d[i] = a[i] + b[i]; }
__global__ void k_addmadd(float* d, const float* a, const float* b, const float* c, float mul, int N) {
    GS_LOOP(i, N) d[i] = a[i] + mul * (b[i] + c[i]);
}
__global__ void k_madd(float* d, const float* a, const float* b, float mulB, int N) {
    GS_LOOP(i, N) d[i] = a[i] + (b ? mulB * b[i] : mulB);
}
__global__ void k_vecmadd(float* dx, float* dy, float* dz, const float* ax, const float* ay, const float* az,
                          const float* bx, const float* by, const float* bz, float mx, float my, float mz, int N) {
    GS_LOOP(i, N) {
        if (bx) {
            dx[i] = ax[i] + mx * bx[i];
            dy[i] = ay[i] + my * by[i];
            dz[i] = az[i] + mz * bz[i];
        } else {
            dx[i] = ax[i] + mx;
            dy[i] = ay[i] + my;
            dz[i] = az[i] + mz;
        }
    }
}
__global__ void k_madd1(float* a, const float* b, float mulB, int N) { GS_LOOP(i, N) a[i] += mulB * (b ? b[i] : 1.0f); }
__global__ void k_madd2(float* a, const float* b, float mulB, const float* c, float mulC, int N) {
    GS_LOOP(i, N) a[i] += mulB * (b ? b[i] : 1.0f) + mulC * (c ? c[i] : 1.0f);
}
__global__ void k_cmadd(float* dst, float a, float b, const float* kern, const float* src, int NC) {
    GS_LOOP(i, NC) {
        float Sa = src[2 * i], Sb = src[2 * i + 1], k = kern[i];
        dst[2 * i] += k * (a * Sa - b * Sb);
        dst[2 * i + 1] += k * (b * Sa + a * Sb);
    }
}
__global__ void k_lin2(float* d, const float* a, float ma, const float* b, float mb, int N) {
    GS_LOOP(i, N) d[i] = ma * a[i] + mb * b[i];
}
__global__ void k_lin3(float* d, const float* a, float ma, const float* b, float mb, const float* c, float mc, int N) {
    GS_LOOP(i, N) d[i] = ma * a[i] + mb * b[i] + mc * c[i];
}
__global__ void k_mul(float* d, const float* a, const float* b, int N) { GS_LOOP(i, N) d[i] = a[i] * b[i]; }

// ---------------------------------------------------------------- kernelmul_micromag.cu:25-70
__global__ void k_kernelmul(float* Mx, float* My, float* Mz, const float* Kxx, const float* Kyy, const float* Kzz,
                            const float* Kyz, const float* Kxz, const float* Kxy, int NC) {
    GS_LOOP(i, NC) {
        float2 mx = reinterpret_cast<float2*>(Mx)[i], my = reinterpret_cast<float2*>(My)[i],
               mz = reinterpret_cast<float2*>(Mz)[i];
        float xx = Kxx[i], yy = Kyy[i], zz = Kzz[i], yz = Kyz[i], xz = Kxz[i], xy = Kxy[i];
        reinterpret_cast<float2*>(Mx)[i] =
            make_float2(mx.x * xx + my.x * xy + mz.x * xz, mx.y * xx + my.y * xy + mz.y * xz);
        reinterpret_cast<float2*>(My)[i] =
            make_float2(mx.x * xy + my.x * yy + mz.x * yz, mx.y * xy + my.y * yy + mz.y * yz);
        reinterpret_cast<float2*>(Mz)[i] =
            make_float2(mx.x * xz + my.x * yz + mz.x * zz, mx.y * xz + my.y * yz + mz.y * zz);
    }
}

// ---------------------------------------------------------------- copypad.cu
__global__ void k_zero(float* A, int N) { GS_LOOP(i, N) A[i] = 0.0f; }
// copy the overlapping box (B0,B1,B2) from src (S dims) to dst (D dims)
__global__ void k_copybox(float* dst, int D1, int D2, const float* src, int S1, int S2, int B0, int B1, int B2) {
    const long long n = (long long)B0 * B1 * B2;
    GS_LOOP(e, n) {
        int k = (int)(e % B2);
        long long r = e / B2;
        int j = (int)(r % B1), i = (int)(r / B1);
        dst[((long long)i * D1 + j) * D2 + k] = src[((long long)i * S1 + j) * S2 + k];
    }
}

// ---------------------------------------------------------------- reductions
enum { R_SUM, R_SDOT, R_MAX, R_MIN, R_MAXABS, R_MAXDIFF, R_MAXSUM, R_MAXN3, R_MAXN3D };

template <int OP>
__global__ void k_partial(const float* a, const float* b, const float* c, const float* d, const float* e,
                          const float* f, float* out, int N) {
    float acc, comp = 0.f;
    if (OP == R_SUM || OP == R_SDOT) acc = 0.f;
    else if (OP == R_MAX) acc = -INFINITY;
    else if (OP == R_MIN) acc = INFINITY;
    else acc = 0.f;
    GS_LOOP(i, N) {
        float v;
        switch (OP) {
            case R_SUM: v = a[i]; break;
            case R_SDOT: v = a[i] * b[i]; break;
            case R_MAX:
            case R_MIN: v = a[i]; break;
            case R_MAXABS: v = fabsf(a[i]); break;
            case R_MAXDIFF: v = fabsf(a[i] - b[i]); break;
            case R_MAXSUM: v = fabsf(a[i] + b[i]); break;
            case R_MAXN3: v = a[i] * a[i] + b[i] * b[i] + c[i] * c[i]; break;
            default: {
                float dx = a[i] - d[i], dy = b[i] - e[i], dz = c[i] - f[i];
                v = dx * dx + dy * dy + dz * dz;
            }
        }
        if (OP == R_SUM || OP == R_SDOT) {  // Neumaier compensated
            float t = acc + v;
            if (fabsf(acc) >= fabsf(v)) comp += (acc - t) + v;
            else comp += (v - t) + acc;
            acc = t;
        } else if (OP == R_MIN) acc = fminf(acc, v);
        else acc = fmaxf(acc, v);
    }
    if (OP == R_SUM || OP == R_SDOT) acc += comp;
    __shared__ float sh[32];
    for (int o = 16; o > 0; o >>= 1) {
        float w = __shfl_xor_sync(0xffffffffu, acc, o);
        if (OP == R_SUM || OP == R_SDOT) acc += w;
        else if (OP == R_MIN) acc = fminf(acc, w);
        else acc = fmaxf(acc, w);
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            if (OP == R_SUM || OP == R_SDOT) r += sh[w];
            else if (OP == R_MIN) r = fminf(r, sh[w]);
            else r = fmaxf(r, sh[w]);
        }
        out[blockIdx.x] = r;
    }
}

template <int OP>
void partial1(const float* a, const float* b, const float* c, const float* d, const float* e, const float* f,
              float* out, int blocks, int N, cudaStream_t st) {
    if (blocks < 1) return;
    k_partial<OP><<<blocks, 256, 0, st>>>(a, b, c, d, e, f, out, N);
    note(cudaGetLastError());
}

// ---------------------------------------------------------------- temperature.cu:14-66
__global__ void k_scale_noise(float* noise, const float* alpha, const float* temp, float aKT, const float* msat,
                              float den, int N) {
    GS_LOOP(i, N) {
        float a = alpha ? alpha[i] : 1.0f, m = msat ? msat[i] : 1.0f, t = temp ? temp[i] : 1.0f;
        noise[i] = (m != 0.f) ? noise[i] * sqrtf((a * t * aKT) / (den * m)) : 0.f;
    }
}

// ---------------------------------------------------------------- zhang-li_torque.cu:123-300
__device__ __forceinline__ float3 crossf3(float3 a, float3 b) {
    return make_float3(-a.y * b.z + a.z * b.y, -a.z * b.x + a.x * b.z, -a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ int nb5c(int i, int d, int n, int wrap) {
    int j = i + d;
    if (!wrap && (j < 0 || j >= n)) return i;
    if (j < 0) j += n;
    if (j >= n) j -= n;
    return j;
}
__global__ void k_zhangli(float* sx_, float* sy_, float* sz_, const float* mx, const float* my, const float* mz,
                          const float* jx, const float* jy, const float* jz, const float* msat, const float* pol,
                          const float* ee, const float* alpha, float3 jMul, float pre, float eeMul, float alphaMul,
                          int sx, int sy, int sz, float3 mstep, int w0, int w1, int w2) {
    const long long N = (long long)sx * sy * sz;
    GS_LOOP(x0, N) {
        int k = (int)(x0 % sz);
        long long r = x0 / sz;
        int j = (int)(r % sy), i = (int)(r / sy);
        float m_sat = msat ? msat[x0] : 1.0f;
        float3 j0 = make_float3(jx ? jx[x0] * jMul.x : jMul.x, jy ? jy[x0] * jMul.y : jMul.y,
                                jz ? jz[x0] * jMul.z : jMul.z);
        float njn = sqrtf(j0.x * j0.x + j0.y * j0.y + j0.z * j0.z);
        if (m_sat == 0.0f || njn == 0.0f) {
            sx_[x0] = 0.f;
            sy_[x0] = 0.f;
            sz_[x0] = 0.f;
            continue;
        }
        m_sat = 1.0f / m_sat;
        float PP = pol ? pol[x0] : 1.0f;
        float pred = njn * PP * pre;
        float e = ee ? ee[x0] * eeMul : eeMul;
        float a = alpha ? alpha[x0] * alphaMul : alphaMul;
        pred = pred / ((1.0f + e * e) * (1.0f + a * a));
        float pret = pred * (e - a);
        pred = pred * (1.0f + e * a);
        const int cc[3] = {i, j, k}, nn[3] = {sx, sy, sz}, ww[3] = {w0, w1, w2};
        const long long st[3] = {(long long)sy * sz, sz, 1};
        const float ms[3] = {mstep.x, mstep.y, mstep.z};
        float inv = 1.0f / njn;
        float nj[3] = {j0.x * inv, j0.y * inv, j0.z * inv};
        const float* comp[3] = {mx, my, mz};
        float dmdj[3] = {0.f, 0.f, 0.f};
        for (int d = 0; d < 3; d++) {
            long long b2 = x0 + (long long)(nb5c(cc[d], -2, nn[d], ww[d]) - cc[d]) * st[d];
            long long b1 = x0 + (long long)(nb5c(cc[d], -1, nn[d], ww[d]) - cc[d]) * st[d];
            long long f1 = x0 + (long long)(nb5c(cc[d], +1, nn[d], ww[d]) - cc[d]) * st[d];
            long long f2 = x0 + (long long)(nb5c(cc[d], +2, nn[d], ww[d]) - cc[d]) * st[d];
            for (int q = 0; q < 3; q++) {
                const float* A = comp[q];
                dmdj[q] += ms[d] * (A[b2] - 8.0f * A[b1] + 8.0f * A[f1] - A[f2]) * nj[d];
            }
        }
        float3 m = make_float3(mx[x0], my[x0], mz[x0]);
        float3 dm = make_float3(dmdj[0], dmdj[1], dmdj[2]);
        float3 dmxm = crossf3(dm, m);
        float3 mxdmxm = crossf3(m, dmxm);
        sx_[x0] = m_sat * (pred * mxdmxm.x + pret * dmxm.x);
        sy_[x0] = m_sat * (pred * mxdmxm.y + pret * dmxm.y);
        sz_[x0] = m_sat * (pred * mxdmxm.z + pret * dmxm.z);
    }
}

// ---------------------------------------------------------------- slonczewski_torque.cu:14-116
__global__ void k_slon(float* sx, float* sy, float* sz, const float* mx, const float* my, const float* mz,
                       const float* msat, const float* px, const float* py, const float* pz, const float* jx,
                       const float* jy, const float* jz, const float* alpha, const float* tfl, const float* pol,
                       const float* lambda, const float* epsp, float3 pMul, float3 jMul, float beta_prime,
                       float pre_fld, float alphaMul, float tflMul, float lambdaMul, int N) {
    GS_LOOP(I, N) {
        float Ms = msat ? msat[I] : 1.0f;
        float3 J = make_float3(jx ? jx[I] * jMul.x : jMul.x, jy ? jy[I] * jMul.y : jMul.y,
                               jz ? jz[I] * jMul.z : jMul.z);
        float nJn = sqrtf(J.x * J.x + J.y * J.y + J.z * J.z);
        float t = tfl ? tfl[I] * tflMul : tflMul;
        if (nJn == 0.0f || Ms == 0.0f || t == 0.0f) {
            sx[I] = 0.f;
            sy[I] = 0.f;
            sz[I] = 0.f;
            continue;
        }
        t = 1.0f / t;
        Ms = 1.0f / Ms;
        float prex = beta_prime * Ms, prey = pre_fld * Ms;
        float3 m = make_float3(mx[I], my[I], mz[I]);
        float3 p = make_float3(px ? pMul.x * px[I] : pMul.x, py ? pMul.y * py[I] : pMul.y, pz ? pMul.z * pz[I] : pMul.z);
        float pl = sqrtf(p.x * p.x + p.y * p.y + p.z * p.z);
        float pi = (pl != 0.0f) ? 1.0f / pl : 0.0f;
        p.x *= pi; p.y *= pi; p.z *= pi;
        float3 pxm = crossf3(p, m);
        float3 mxpxm = crossf3(m, pxm);
        float pdotm = p.x * m.x + p.y * m.y + p.z * m.z;
        float ji = 1.0f / nJn;
        float Jdir = J.x * ji + J.y * ji + J.z * ji;
        float nj = nJn * (Jdir / fabsf(Jdir));
        prex *= nj * t;
        prey *= nj * t;
        float lam = lambda ? lambdaMul * lambda[I] : lambdaMul;
        float l2 = lam * lam;
        prex *= l2 / ((l2 + 1.0f) + (l2 - 1.0f) * pdotm);
        float a = alpha ? alpha[I] * alphaMul : alphaMul;
        float af = 1.0f / (1.0f + a * a);
        prex *= pol ? pol[I] : 1.0f;
        prey *= epsp ? epsp[I] : 1.0f;
        float f1 = (prex - a * prey) * af, f2 = (prey - a * prex) * af;
        sx[I] = f1 * mxpxm.x + f2 * pxm.x;
        sy[I] = f1 * mxpxm.y + f2 * pxm.y;
        sz[I] = f1 * mxpxm.z + f2 * pxm.z;
    }
}

inline float* P(float** a, int dev) { return a ? a[dev] : nullptr; }

}  // namespace

#define FOR_DEV for (int dev = 0; dev < ndev(); dev++)
#define LAUNCH(kern, n, st, ...)                                    \
    do {                                                            \
        kern<<<grid_for(n), 256, 0, st>>>(__VA_ARGS__);             \
        note(cudaGetLastError());                                   \
    } while (0)

extern "C" {

MM_API void setUsedGPUs(int* gpuIds, int Ngpu) {
    g_ngpu = (Ngpu > 64) ? 64 : Ngpu;
    for (int i = 0; i < g_ngpu; i++) g_ids[i] = gpuIds[i];
}
MM_API int nDevice(void) { return ndev(); }
MM_API int deviceId(int i) {
    if (g_ngpu == 0) {
        int d = 0;
        cudaGetDevice(&d);
        return d;
    }
    return (i >= 0 && i < g_ngpu) ? g_ids[i] : -1;
}
MM_API int mm_compat_last_status(void) { return g_status; }

MM_API void torqueAsync(float** tx, float** ty, float** tz, float** mx, float** my, float** mz, float** hx, float** hy,
                        float** hz, float** alpha_map, float alpha_mul, CUstream* stream, int Npart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_torque, Npart, sget(stream, dev), tx[dev], ty[dev], tz[dev], mx[dev], my[dev], mz[dev], hx[dev],
               hy[dev], hz[dev], P(alpha_map, dev), alpha_mul, Npart);
    }
}

MM_API void exchange6Async(float** hx, float** hy, float** hz, float** mx, float** my, float** mz, float** msat,
                           float** aex, float pre, int N0, int N1Part, int N2, int periodic0, int periodic1,
                           int periodic2, float cellSizeX, float cellSizeY, float cellSizeZ, CUstream* streams) {
    float c0 = (float)(1.0 / ((double)cellSizeX * (double)cellSizeX));
    float c1 = (float)(1.0 / ((double)cellSizeY * (double)cellSizeY));
    float c2 = (float)(1.0 / ((double)cellSizeZ * (double)cellSizeZ));
    long long n = (long long)N0 * N1Part * N2;
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_exchange6, n, sget(streams, dev), hx[dev], hy[dev], hz[dev], mx[dev], my[dev], mz[dev],
               P(msat, dev), P(aex, dev), pre, N0, N1Part, N2, periodic0, periodic1, periodic2, c0, c1, c2);
    }
}

MM_API void uniaxialAnisotropyAsync(float** hx, float** hy, float** hz, float** mx, float** my, float** mz,
                                    float** Ku1_map, float** MSat_map, float Ku2_Mu0Msat_mul, float** anisU_mapx,
                                    float anisU_mulx, float** anisU_mapy, float anisU_muly, float** anisU_mapz,
                                    float anisU_mulz, CUstream* stream, int Npart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_uniaxial, Npart, sget(stream, dev), hx[dev], hy[dev], hz[dev], mx[dev], my[dev], mz[dev],
               P(Ku1_map, dev), P(MSat_map, dev), Ku2_Mu0Msat_mul, P(anisU_mapx, dev), anisU_mulx, P(anisU_mapy, dev),
               anisU_muly, P(anisU_mapz, dev), anisU_mulz, Npart);
    }
}

MM_API void normalizeAsync(float** mx, float** my, float** mz, float** norm_map, CUstream* stream, int Npart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_normalize, Npart, sget(stream, dev), mx[dev], my[dev], mz[dev], P(norm_map, dev), Npart);
    }
}

MM_API void addAsync(float** dst, float** a, float** b, CUstream* stream, int Npart) {
    FOR_DEV { setdev(dev); LAUNCH(k_add, Npart, sget(stream, dev), dst[dev], a[dev], b[dev], Npart); }
}
MM_API void addMaddAsync(float** dst, float** a, float** b, float** c, float mul, CUstream* stream, int NPart) {
    FOR_DEV { setdev(dev); LAUNCH(k_addmadd, NPart, sget(stream, dev), dst[dev], a[dev], b[dev], c[dev], mul, NPart); }
}
MM_API void maddAsync(float** dst, float** a, float** b, float mulB, CUstream* stream, int Npart) {
    FOR_DEV { setdev(dev); LAUNCH(k_madd, Npart, sget(stream, dev), dst[dev], a[dev], P(b, dev), mulB, Npart); }
}
MM_API void vecMaddAsync(float** dstx, float** dsty, float** dstz, float** ax, float** ay, float** az, float** bx,
                         float** by, float** bz, float mulBx, float mulBy, float mulBz, CUstream* stream, int Npart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_vecmadd, Npart, sget(stream, dev), dstx[dev], dsty[dev], dstz[dev], ax[dev], ay[dev], az[dev],
               P(bx, dev), P(by, dev), P(bz, dev), mulBx, mulBy, mulBz, Npart);
    }
}
MM_API void madd1Async(float** a, float** b, float mulB, CUstream* stream, int Npart) {
    FOR_DEV { setdev(dev); LAUNCH(k_madd1, Npart, sget(stream, dev), a[dev], P(b, dev), mulB, Npart); }
}
MM_API void madd2Async(float** a, float** b, float mulB, float** c, float mulC, CUstream* stream, int Npart) {
    FOR_DEV { setdev(dev); LAUNCH(k_madd2, Npart, sget(stream, dev), a[dev], P(b, dev), mulB, P(c, dev), mulC, Npart); }
}
MM_API void cmaddAsync(float** dst, float a, float b, float** kern, float** src, CUstream* stream, int NComplexPart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_cmadd, NComplexPart, sget(stream, dev), dst[dev], a, b, kern[dev], src[dev], NComplexPart);
    }
}
MM_API void linearCombination2Async(float** dst, float** a, float mulA, float** b, float mulB, CUstream* stream,
                                    int NPart) {
    FOR_DEV { setdev(dev); LAUNCH(k_lin2, NPart, sget(stream, dev), dst[dev], a[dev], mulA, b[dev], mulB, NPart); }
}
MM_API void linearCombination3Async(float** dst, float** a, float mulA, float** b, float mulB, float** c, float mulC,
                                    CUstream* stream, int NPart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_lin3, NPart, sget(stream, dev), dst[dev], a[dev], mulA, b[dev], mulB, c[dev], mulC, NPart);
    }
}
MM_API void mulAsync(float** dst, float** a, float** b, CUstream* stream, int Npart) {
    FOR_DEV { setdev(dev); LAUNCH(k_mul, Npart, sget(stream, dev), dst[dev], a[dev], b[dev], Npart); }
}
MM_API void kernelMulMicromag3DAsync(float** fftMx, float** fftMy, float** fftMz, float** fftKxx, float** fftKyy,
                                     float** fftKzz, float** fftKyz, float** fftKxz, float** fftKxy, CUstream* stream,
                                     int partLen3D) {
    const int nc = partLen3D / 2;
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_kernelmul, nc, sget(stream, dev), fftMx[dev], fftMy[dev], fftMz[dev], fftKxx[dev], fftKyy[dev],
               fftKzz[dev], fftKyz[dev], fftKxz[dev], fftKxy[dev], nc);
    }
}
MM_API void zeroArrayAsync(float** A, int length, CUstream* streams) {
    FOR_DEV { setdev(dev); LAUNCH(k_zero, length, sget(streams, dev), A[dev], length); }
}
MM_API void copyPad3DAsync(float** dst, int D0, int D1, int D2, float** src, int S0, int S1, int S2, int Ncomp,
                           CUstream* streams) {
    const long long n = (long long)S0 * S1 * S2;
    FOR_DEV {
        setdev(dev);
        for (int c = 0; c < Ncomp; c++)
            LAUNCH(k_copybox, n, sget(streams, dev), dst[dev] + (long long)c * D0 * D1 * D2, D1, D2,
                   src[dev] + (long long)c * S0 * S1 * S2, S1, S2, S0, S1, S2);
    }
}
MM_API void copyUnPad3DAsync(float** dst, int D0, int D1, int D2, float** src, int S0, int S1, int S2, int Ncomp,
                             CUstream* streams) {
    const long long n = (long long)D0 * D1 * D2;
    FOR_DEV {
        setdev(dev);
        for (int c = 0; c < Ncomp; c++)
            LAUNCH(k_copybox, n, sget(streams, dev), dst[dev] + (long long)c * D0 * D1 * D2, D1, D2,
                   src[dev] + (long long)c * S0 * S1 * S2, S1, S2, D0, D1, D2);
    }
}

#define PARTIAL_MULTI(name, OP, ...)                                                               \
    FOR_DEV {                                                                                      \
        setdev(dev);                                                                               \
        partial1<OP>(__VA_ARGS__, output[dev], blocks, N, sget(stream, dev));                      \
    }

MM_API void partialSumAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream) {
    PARTIAL_MULTI(sum, R_SUM, input[dev], nullptr, nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialSDotAsync(float** input1, float** input2, float** output, int blocks, int threadsPerBlock, int N,
                             CUstream* stream) {
    PARTIAL_MULTI(sdot, R_SDOT, input1[dev], input2[dev], nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMaxAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream) {
    PARTIAL_MULTI(max, R_MAX, input[dev], nullptr, nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMinAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream) {
    PARTIAL_MULTI(min, R_MIN, input[dev], nullptr, nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMaxAbsAsync(float** input, float** output, int blocks, int threadsPerBlock, int N,
                               CUstream* stream) {
    PARTIAL_MULTI(maxabs, R_MAXABS, input[dev], nullptr, nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMaxDiffAsync(float** a, float** b, float** output, int blocks, int threadsPerBlock, int N,
                                CUstream* stream) {
    PARTIAL_MULTI(maxdiff, R_MAXDIFF, a[dev], b[dev], nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMaxSumAsync(float** a, float** b, float** output, int blocks, int threadsPerBlock, int N,
                               CUstream* stream) {
    PARTIAL_MULTI(maxsum, R_MAXSUM, a[dev], b[dev], nullptr, nullptr, nullptr, nullptr)
}
MM_API void partialMaxNorm3SqAsync(float** x, float** y, float** z, float** output, int blocks, int threadsPerBlock,
                                   int N, CUstream* stream) {
    PARTIAL_MULTI(maxn3, R_MAXN3, x[dev], y[dev], z[dev], nullptr, nullptr, nullptr)
}
MM_API void partialMaxNorm3SqDiffAsync(float** x1, float** y1, float** z1, float** x2, float** y2, float** z2,
                                       float** output, int blocks, int threadsPerBlock, int N, CUstream* stream) {
    PARTIAL_MULTI(maxn3d, R_MAXN3D, x1[dev], y1[dev], z1[dev], x2[dev], y2[dev], z2[dev])
}
MM_API void partialSumAsync1(float* in, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_SUM>(in, nullptr, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxAsync1(float* in, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_MAX>(in, nullptr, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMinAsync1(float* in, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_MIN>(in, nullptr, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxAbsAsync1(float* in, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_MAXABS>(in, nullptr, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxDiffAsync1(float* a, float* b, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_MAXDIFF>(a, b, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxSumAsync1(float* a, float* b, float* out, int blocks, int threads, int size, CUstream st) {
    partial1<R_MAXSUM>(a, b, nullptr, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxNorm3SqAsync1(float* x, float* y, float* z, float* out, int blocks, int threads, int size,
                                    CUstream st) {
    partial1<R_MAXN3>(x, y, z, nullptr, nullptr, nullptr, out, blocks, size, (cudaStream_t)st);
}
MM_API void partialMaxNorm3SqDiffAsync1(float* x1, float* y1, float* z1, float* x2, float* y2, float* z2, float* out,
                                        int blocks, int threads, int size, CUstream st) {
    partial1<R_MAXN3D>(x1, y1, z1, x2, y2, z2, out, blocks, size, (cudaStream_t)st);
}

MM_API void temperature_scaleNoise(float** noise, float** alpha, float** temp, float alphaKB2tempMul, float** mSat,
                                   float mu0VgammaDtMSatMul, CUstream* stream, int Npart) {
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_scale_noise, Npart, sget(stream, dev), noise[dev], P(alpha, dev), P(temp, dev), alphaKB2tempMul,
               P(mSat, dev), mu0VgammaDtMSatMul, Npart);
    }
}

MM_API void zhangli_async(float** sttx, float** stty, float** sttz, float** mx, float** my, float** mz, float** jx,
                          float** jy, float** jz, float** msat, float** pol, float** ee, float** alpha,
                          const float jMul_x, const float jMul_y, const float jMul_z, const float pred,
                          const float eeMul, const float alphaMul, const int sx, const int sy, const int sz,
                          const float csx, const float csy, const float csz, const int pbc_x, const int pbc_y,
                          const int pbc_z, CUstream* stream) {
    // one launch over all cells instead of one per x-slab (zhang-li_torque.cu:389)
    float3 mstep = make_float3(1.0f / (12.0f * csx), 1.0f / (12.0f * csy), 1.0f / (12.0f * csz));
    float3 jm = make_float3(jMul_x, jMul_y, jMul_z);
    const long long n = (long long)sx * sy * sz;
    // dimension 1 wraps through the neighbour-device pointers, which with one device
    // are the array itself when pbc_y is set (zhang-li_torque.cu:354-382)
    const int wrap1 = (ndev() == 1) ? pbc_y : 0;
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_zhangli, n, sget(stream, dev), sttx[dev], stty[dev], sttz[dev], mx[dev], my[dev], mz[dev],
               P(jx, dev), P(jy, dev), P(jz, dev), P(msat, dev), P(pol, dev), P(ee, dev), P(alpha, dev), jm, pred,
               eeMul, alphaMul, sx, sy, sz, mstep, pbc_x, wrap1, pbc_z);
    }
}

MM_API void slonczewski_async(float** sttx, float** stty, float** sttz, float** mx, float** my, float** mz,
                              float** msat, float** px, float** py, float** pz, float** jx, float** jy, float** jz,
                              float** alphamsk, float** t_flmsk, float** polMsk, float** lambdaMsk,
                              float** epsilon_primeMsk, float pxMul, float pyMul, float pzMul, float jxMul,
                              float jyMul, float jzMul, float beta_prime, float pre_field, float meshSizeX,
                              float meshSizeY, float meshSizeZ, float alphaMul, float t_flMul, float lambdaMul,
                              int NPart, CUstream* stream) {
    (void)meshSizeX; (void)meshSizeY; (void)meshSizeZ;  // unused by the reference kernel too
    FOR_DEV {
        setdev(dev);
        LAUNCH(k_slon, NPart, sget(stream, dev), sttx[dev], stty[dev], sttz[dev], mx[dev], my[dev], mz[dev],
               P(msat, dev), P(px, dev), P(py, dev), P(pz, dev), P(jx, dev), P(jy, dev), P(jz, dev),
               P(alphamsk, dev), P(t_flmsk, dev), P(polMsk, dev), P(lambdaMsk, dev), P(epsilon_primeMsk, dev),
               make_float3(pxMul, pyMul, pzMul), make_float3(jxMul, jyMul, jzMul), beta_prime, pre_field, alphaMul,
               t_flMul, lambdaMul, NPart);
    }
}

}  // extern "C"
