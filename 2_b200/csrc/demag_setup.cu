// demag_setup.cu -- the demag tensor in FP64 on the GPU and its transform.
//
// Kernel_Arne (src/mumax/modules/kernel_magnetostatic.go:30-181) integrates the field
// of the face charges of a source cell over the volume of each destination cell with
// a distance-adaptive number of points.  The reference runs it on the CPU in FP64 and
// stores float32 (:170-173); here one GPU thread computes one (source, x, y, z) entry
// in FP64 and the result stays FP64 through the transform (maxwell_convolution.go:
// 313-410: FFT, keep the real part, scale by 1/prod(L)).  Only one octant of the
// (even or odd) transformed tensor is kept, as FP32.
#include <cmath>
#include <cstdio>
#include <vector>

#include "mm_internal.h"

namespace mm {

__host__ __device__ __forceinline__ int wrap_i(int number, int max) {
    number %= max;
    return number < 0 ? number + max : number;
}
__device__ __forceinline__ double delta_d(int d) {
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}

struct ArneArgs {
    int size[3];
    double cs[3];
    int x1, y1, z1;
    int nx_, ny_, nz_;     // loop extents
    double accuracy;
    double Lmin;
    double* K;             // [6][L0][L1][L2]: xx yy zz yz xz xy
    int accumulate;        // periodic images map several points to one index
};

// component index of (s, d) with s <= d in the order xx yy zz yz xz xy; -1 if s > d
__device__ __forceinline__ int sym_q(int s, int d) {
    if (s > d) return -1;
    if (s == d) return s;
    if (s == 1 && d == 2) return 3;
    if (s == 0 && d == 2) return 4;
    return 5;
}

__global__ void kernel_arne_kernel(ArneArgs A) {
    const long long total = 3LL * A.nx_ * A.ny_ * A.nz_;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
         g += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(g / ((long long)A.nx_ * A.ny_ * A.nz_));
        long long r = g % ((long long)A.nx_ * A.ny_ * A.nz_);
        const int x = A.x1 + (int)(r / ((long long)A.ny_ * A.nz_));
        r %= ((long long)A.ny_ * A.nz_);
        const int y = A.y1 + (int)(r / A.nz_);
        const int z = A.z1 + (int)(r % A.nz_);
        const double* cs = A.cs;
        const int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
        double R[3] = {(double)x * cs[0], (double)y * cs[1], (double)z * cs[2]};
        double dx = delta_d(x) * cs[0], dy = delta_d(y) * cs[1], dz = delta_d(z) * cs[2];
        double d = sqrt(dx * dx + dy * dy + dz * dz);
        if (d == 0) d = A.Lmin;
        double maxSize = d / A.accuracy;
        int nv = (int)(fmax(cs[v] / maxSize, 1.) + 0.5);
        int nw = (int)(fmax(cs[w] / maxSize, 1.) + 0.5);
        int nx = (int)(fmax(cs[0] / maxSize, 1.) + 0.5);
        int ny = (int)(fmax(cs[1] / maxSize, 1.) + 0.5);
        int nz = (int)(fmax(cs[2] / maxSize, 1.) + 0.5);
        nv *= 2;
        nw *= 2;
        const double scale = 1 / (double)(nv * nw * nx * ny * nz);
        const double charge = cs[v] * cs[w] * scale;
        const double pu1 = cs[u] / 2., pu2 = -pu1;
        const double fourpi = 4.0 * 3.14159265358979323846;
        double B[3] = {0, 0, 0};
        double pole[3];
        for (int i = 0; i < nv; i++) {
            pole[v] = -(cs[v] / 2.) + cs[v] / (double)(2 * nv) + (double)i * (cs[v] / (double)nv);
            for (int j = 0; j < nw; j++) {
                pole[w] = -(cs[w] / 2.) + cs[w] / (double)(2 * nw) + (double)j * (cs[w] / (double)nw);
                for (int a = 0; a < nx; a++) {
                    double rx = R[0] - cs[0] / 2. + cs[0] / (double)(2 * nx) + (cs[0] / (double)nx) * (double)a;
                    for (int b = 0; b < ny; b++) {
                        double ry = R[1] - cs[1] / 2. + cs[1] / (double)(2 * ny) + (cs[1] / (double)ny) * (double)b;
                        for (int c = 0; c < nz; c++) {
                            double rz = R[2] - cs[2] / 2. + cs[2] / (double)(2 * nz) + (cs[2] / (double)nz) * (double)c;
                            pole[u] = pu1;
                            double X0 = rx - pole[0], Y0 = ry - pole[1], Z0 = rz - pole[2];
                            double rr = sqrt(X0 * X0 + Y0 * Y0 + Z0 * Z0);
                            double qr = charge / (fourpi * rr * rr * rr);
                            double bx = X0 * qr, by = Y0 * qr, bz = Z0 * qr;
                            pole[u] = pu2;
                            X0 = rx - pole[0]; Y0 = ry - pole[1]; Z0 = rz - pole[2];
                            rr = sqrt(X0 * X0 + Y0 * Y0 + Z0 * Z0);
                            qr = -charge / (fourpi * rr * rr * rr);
                            B[0] += (bx + X0 * qr);
                            B[1] += (by + Y0 * qr);
                            B[2] += (bz + Z0 * qr);
                        }
                    }
                }
            }
        }
        const int xw = wrap_i(x, A.size[0]), yw = wrap_i(y, A.size[1]), zw = wrap_i(z, A.size[2]);
        const long long NL = (long long)A.size[0] * A.size[1] * A.size[2];
        const long long idx = ((long long)xw * A.size[1] + yw) * A.size[2] + zw;
        for (int dd = 0; dd < 3; dd++) {
            int q = sym_q(s, dd);
            if (q < 0) continue;
            if (A.accumulate) atomicAdd(A.K + q * NL + idx, B[dd]);
            else A.K[q * NL + idx] = B[dd];
        }
    }
}

// ---------------------------------------------------------------- Newell tensor
// The demag tensor of uniformly magnetised rectangular cells from the closed forms of
// Newell, Williams & Dunlop, J. Geophys. Res. 98, 9551 (1993): with V = d0 d1 d2,
//   N_aa(X) = 1/(4 pi V) sum_{i,j,k in -1,0,1} c_i c_j c_k f(X_a + i d_a, X_b + j d_b, X_c + k d_c)
//   N_ab(X) = the same sum over g,  c_0 = 2, c_{+-1} = -1,
// f and g as in that paper (eqs. 27 and 32 there).  The 27-term difference of f and g
// cancels catastrophically with distance (terms grow as R^3, the result falls as R^-3),
// so it is used only within RHO_NEAR cell sizes; beyond that the tensor is the cell-cell
// average of the point-dipole tensor, N_ab(X) = 1/V int prod_k (d_k - |s_k|)
// (delta_ab |r|^2 - 3 r_a r_b) / (4 pi |r|^5) ds with r = X + s, by tensor-product
// Gauss-Legendre quadrature of the tent weights (Q points per half axis: 6 below 16,
// 4 below 32, 3 beyond, in units of the largest cell edge).  Against the closed form
// evaluated in 80-bit long double the far field is within 1e-12 relative of each
// element at the switch distance.  Everything is FP64, in units of the largest cell
// edge (the tensor is scale-free).  K = -N: the convolution kernel gives H = K * M.
constexpr double RHO_NEAR = 8.0;

__host__ __device__ __forceinline__ double newell_f(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    double r = (2.0 * x2 - y2 - z2) * R / 6.0;
    if (x2 + z2 > 0) r += 0.5 * y * (z2 - x2) * asinh(y / sqrt(x2 + z2));
    if (x2 + y2 > 0) r += 0.5 * z * (y2 - x2) * asinh(z / sqrt(x2 + y2));
    if (x != 0) r -= x * y * z * atan(y * z / (x * R));
    return r;
}

__host__ __device__ __forceinline__ double newell_g(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    double r = -x * y * R / 3.0;
    if (x2 + y2 > 0) r += x * y * z * asinh(z / sqrt(x2 + y2));
    if (y2 + z2 > 0) r += y / 6.0 * (3.0 * z2 - y2) * asinh(x / sqrt(y2 + z2));
    if (x2 + z2 > 0) r += x / 6.0 * (3.0 * z2 - x2) * asinh(y / sqrt(x2 + z2));
    if (z != 0) r -= z * z2 / 6.0 * atan(x * y / (z * R));
    if (y != 0) r -= 0.5 * z * y2 * atan(x * z / (y * R));
    if (x != 0) r -= 0.5 * z * x2 * atan(y * z / (x * R));
    return r;
}

// 27-point second difference of f (G = false) or g (G = true) at (a, b, c), spacings (da, db, dc)
template <bool G>
__host__ __device__ double newell_diff(double a, double b, double c, double da, double db, double dc) {
    double s = 0;
    for (int i = -1; i <= 1; i++) {
        const double ci = i == 0 ? 2.0 : -1.0;
        for (int j = -1; j <= 1; j++) {
            const double cj = j == 0 ? 2.0 : -1.0;
            for (int k = -1; k <= 1; k++) {
                const double ck = k == 0 ? 2.0 : -1.0;
                const double x = a + i * da, y = b + j * db, z = c + k * dc;
                s += ci * cj * ck * (G ? newell_g(x, y, z) : newell_f(x, y, z));
            }
        }
    }
    return s / (4.0 * 3.14159265358979323846 * da * db * dc);
}

// Gauss-Legendre nodes and weights on [-1, 1], Q = 3, 4, 6 (positive half; symmetric)
__constant__ double GL_X3[2] = {0.0, 0.7745966692414833770};
__constant__ double GL_W3[2] = {0.8888888888888888889, 0.5555555555555555556};
__constant__ double GL_X4[2] = {0.3399810435848562648, 0.8611363115940525752};
__constant__ double GL_W4[2] = {0.6521451548625461427, 0.3478548451374538574};
__constant__ double GL_X6[3] = {0.2386191860831969086, 0.6612093864662645137, 0.9324695142031520278};
__constant__ double GL_W6[3] = {0.4679139345726910473, 0.3607615730481386076, 0.1713244923791703450};

// the 2Q tent-weighted nodes of one axis: s = +-d xi, w = d^2 (1 - xi) w_xi, xi = Gauss
// node mapped to [0, 1]
__device__ int tent_nodes(int Q, double d, double* s, double* w) {
    int n = 0;
    const int half = (Q + 1) / 2;
    for (int h = 0; h < half; h++) {
        const double x = Q == 3 ? GL_X3[h] : Q == 4 ? GL_X4[h] : GL_X6[h];
        const double wx = Q == 3 ? GL_W3[h] : Q == 4 ? GL_W4[h] : GL_W6[h];
        const int signs = (x == 0.0) ? 1 : 2;  // the centre node of odd Q appears once
        for (int sg = 0; sg < signs; sg++) {
            const double t = sg ? -x : x;          // node on [-1, 1]
            const double xi = 0.5 * (t + 1.0);      // on [0, 1]
            const double wi = 0.5 * wx * d * d * (1.0 - xi);
            s[n] = d * xi;  w[n] = wi;  n++;
            s[n] = -d * xi; w[n] = wi;  n++;
        }
    }
    return n;
}

// cell-averaged dipole tensor: N[6] (00 11 22 12 02 01)
__device__ void dipole_avg(double X0, double X1, double X2, const double* d, int Q, double* N) {
    double s0[12], w0[12], s1[12], w1[12], s2[12], w2[12];
    const int n0 = tent_nodes(Q, d[0], s0, w0);
    const int n1 = tent_nodes(Q, d[1], s1, w1);
    const int n2 = tent_nodes(Q, d[2], s2, w2);
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < n0; i++) {
        const double r0 = X0 + s0[i];
        for (int j = 0; j < n1; j++) {
            const double r1 = X1 + s1[j];
            const double w01 = w0[i] * w1[j];
            for (int k = 0; k < n2; k++) {
                const double r2 = X2 + s2[k];
                const double rr = r0 * r0 + r1 * r1 + r2 * r2;
                const double ir = rsqrt(rr);
                const double ir2 = ir * ir;
                const double wk = w01 * w2[k] * ir2 * ir2 * ir;  // w / |r|^5
                a[0] += wk * (rr - 3.0 * r0 * r0);
                a[1] += wk * (rr - 3.0 * r1 * r1);
                a[2] += wk * (rr - 3.0 * r2 * r2);
                a[3] += wk * (-3.0 * r1 * r2);
                a[4] += wk * (-3.0 * r0 * r2);
                a[5] += wk * (-3.0 * r0 * r1);
            }
        }
    }
    const double c = 1.0 / (4.0 * 3.14159265358979323846 * d[0] * d[1] * d[2]);
    for (int q = 0; q < 6; q++) N[q] = a[q] * c;
}

struct NewellArgs {
    int size[3];
    double d[3];           // cell size in units of the largest edge
    int x1, y1, z1;
    int nx_, ny_, nz_;
    double* K;             // [6][L0][L1][L2]: 00 11 22 12 02 01
    int accumulate;
};

__global__ void newell_kernel(NewellArgs A) {
    const long long total = (long long)A.nx_ * A.ny_ * A.nz_;
    for (long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x; gi < total;
         gi += (long long)gridDim.x * blockDim.x) {
        const int x = A.x1 + (int)(gi / ((long long)A.ny_ * A.nz_));
        const long long r = gi % ((long long)A.ny_ * A.nz_);
        const int y = A.y1 + (int)(r / A.nz_);
        const int z = A.z1 + (int)(r % A.nz_);
        const double* d = A.d;
        const double X0 = x * d[0], X1 = y * d[1], X2 = z * d[2];
        const double rho = sqrt(X0 * X0 + X1 * X1 + X2 * X2);
        double N[6];
        if (rho < RHO_NEAR) {
            N[0] = newell_diff<false>(X0, X1, X2, d[0], d[1], d[2]);
            N[1] = newell_diff<false>(X1, X0, X2, d[1], d[0], d[2]);
            N[2] = newell_diff<false>(X2, X1, X0, d[2], d[1], d[0]);
            N[3] = newell_diff<true>(X1, X2, X0, d[1], d[2], d[0]);
            N[4] = newell_diff<true>(X0, X2, X1, d[0], d[2], d[1]);
            N[5] = newell_diff<true>(X0, X1, X2, d[0], d[1], d[2]);
        } else {
            dipole_avg(X0, X1, X2, d, rho < 16.0 ? 6 : rho < 32.0 ? 4 : 3, N);
        }
        const int xw = wrap_i(x, A.size[0]), yw = wrap_i(y, A.size[1]), zw = wrap_i(z, A.size[2]);
        const long long NL = (long long)A.size[0] * A.size[1] * A.size[2];
        const long long idx = ((long long)xw * A.size[1] + yw) * A.size[2] + zw;
        for (int q = 0; q < 6; q++) {
            if (A.accumulate) atomicAdd(A.K + q * NL + idx, -N[q]);
            else A.K[q * NL + idx] = -N[q];
        }
    }
}

__global__ void maxabs_kernel(const double* a, long long n, unsigned long long* out) {
    double m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// real part of the transformed component, one octant, scaled, as float
__global__ void extract_octant_kernel(const double2* spec, int L0, int L1, int hp, int kd0, int kd1, int kd2,
                                      double scale, float* out) {
    const long long n = (long long)kd0 * kd1 * kd2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int kx = (int)(i % kd2);
        long long r = i / kd2;
        int ky = (int)(r % kd1);
        int kz = (int)(r / kd1);
        out[i] = (float)(spec[((long long)kz * L1 + ky) * hp + kx].x * scale);
    }
}

#define CK(...)                                                                                 \
    do {                                                                                        \
        cudaError_t e_ = (__VA_ARGS__);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            snprintf(err, errlen, "%s: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(e_), __FILE__, __LINE__); \
            goto fail;                                                                          \
        }                                                                                       \
    } while (0)

// Real-space FP64 tensor K[6][L0][L1][L2] (00 11 22 12 02 01, device, caller-allocated)
// on `st`: kind 0 = Kernel_Arne (kernel_magnetostatic.go:30-181, `accuracy`), kind 1 =
// Newell.  Entries beyond the reference's index ranges (the Nyquist planes) stay zero.
int fill_demag_tensor(const int L[3], const double cell[3], const int pbc[3], int kind, int accuracy, double* K,
                      cudaStream_t st) {
    const long long NL = (long long)L[0] * L[1] * L[2];
    int x1 = -(L[0] - 1) / 2, x2 = L[0] / 2 - 1;
    int y1 = -(L[1] - 1) / 2, y2 = L[1] / 2 - 1;
    int z1 = -(L[2] - 1) / 2, z2 = L[2] / 2 - 1;
    if (L[0] == 1 && pbc[0] == 0) x2 = 0;
    x1 *= (pbc[0] + 1); x2 *= (pbc[0] + 1);
    y1 *= (pbc[1] + 1); y2 *= (pbc[1] + 1);
    z1 *= (pbc[2] + 1); z2 *= (pbc[2] + 1);
    const int accumulate = (pbc[0] || pbc[1] || pbc[2]) ? 1 : 0;
    if (cudaMemsetAsync(K, 0, sizeof(double) * 6 * NL, st) != cudaSuccess) return MM_ERR_CUDA;
    const long long cells = (long long)(x2 - x1 + 1) * (y2 - y1 + 1) * (z2 - z1 + 1);
    if (kind == 1) {
        NewellArgs A;
        const double lam = fmax(cell[0], fmax(cell[1], cell[2]));
        for (int i = 0; i < 3; i++) { A.size[i] = L[i]; A.d[i] = cell[i] / lam; }
        A.x1 = x1; A.y1 = y1; A.z1 = z1;
        A.nx_ = x2 - x1 + 1; A.ny_ = y2 - y1 + 1; A.nz_ = z2 - z1 + 1;
        A.K = K;
        A.accumulate = accumulate;
        const int blocks = (int)std::min<long long>((cells + 127) / 128, 148LL * 64);
        newell_kernel<<<blocks, 128, 0, st>>>(A);
    } else {
        ArneArgs A;
        for (int i = 0; i < 3; i++) { A.size[i] = L[i]; A.cs[i] = cell[i]; }
        A.x1 = x1; A.y1 = y1; A.z1 = z1;
        A.nx_ = x2 - x1 + 1; A.ny_ = y2 - y1 + 1; A.nz_ = z2 - z1 + 1;
        A.accuracy = (double)(accuracy > 0 ? accuracy : 6);
        A.Lmin = fmin(cell[0], fmin(cell[1], cell[2]));
        A.accumulate = accumulate;
        A.K = K;
        const long long total = 3 * cells;
        const int blocks = (int)std::min<long long>((total + 127) / 128, 148LL * 64);
        kernel_arne_kernel<<<blocks, 128, 0, st>>>(A);
    }
    return cudaGetLastError() == cudaSuccess ? MM_OK : MM_ERR_CUDA;
}

// Builds khat [6][kd0][kd1][kd2] (FP32, device, caller-allocated) and nz[6].
int build_demag_kernel(const int L[3], const double cell[3], const int pbc[3], int kind, int accuracy, float* khat,
                       const int kd[3], int nz[6], cudaStream_t st, char* err, int errlen) {
    const long long NL = (long long)L[0] * L[1] * L[2];
    const int M = L[2] / 2;
    const int hp = M + 1;
    double* K = nullptr;
    double2* spec = nullptr;
    unsigned long long* dmax = nullptr;
    unsigned long long hmax[7];
    int rc = MM_ERR_CUDA;
    {
        CK(cudaMalloc(&K, sizeof(double) * 6 * NL));
        if (fill_demag_tensor(L, cell, pbc, kind, accuracy, K, st) != MM_OK) {
            snprintf(err, errlen, "demag tensor kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            goto fail;
        }
        CK(cudaMalloc(&dmax, sizeof(unsigned long long) * 7));
        CK(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long) * 7, st));
        for (int q = 0; q < 6; q++) maxabs_kernel<<<296, 256, 0, st>>>(K + q * NL, NL, dmax + q);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hmax, dmax, sizeof(unsigned long long) * 6, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double cmax[6], gmax = 0;
        for (int q = 0; q < 6; q++) {
            memcpy(&cmax[q], &hmax[q], sizeof(double));
            gmax = fmax(gmax, cmax[q]);
        }
        // maxwell_convolution.go:412-418: a component is zero if its max is below
        // 1e-5 of the largest element of the whole tensor
        for (int q = 0; q < 6; q++) nz[q] = (gmax > 0 && cmax[q] / gmax >= 1e-5) ? 1 : 0;
        CK(cudaMalloc(&spec, sizeof(double2) * (size_t)L[0] * L[1] * hp));
        const double scale = 1.0 / (double)NL;
        const long long oct = (long long)kd[0] * kd[1] * kd[2];
        for (int q = 0; q < 6; q++) {
            if (!nz[q]) {
                CK(cudaMemsetAsync(khat + q * oct, 0, sizeof(float) * oct, st));
                continue;
            }
            PP none = {nullptr, nullptr, 0};
            CK(launch_xfwd<double2, double>(M, K + q * NL, none, nullptr, spec, L[0] * L[1], L[0], L[1], L[1], L[2],
                                            L[2], hp, nullptr, nullptr, 0, st));
            if (L[1] > 1)
                CK(launch_colfft<double2>(L[1], -1, spec, hp, L[0], (long long)L[1] * hp, hp, L[1], L[1], nullptr,
                                          nullptr, 0, st));
            if (L[0] > 1)
                CK(launch_colfft<double2>(L[0], -1, spec, hp, L[1], hp, (long long)L[1] * hp, L[0], L[0], nullptr,
                                          nullptr, 0, st));
            extract_octant_kernel<<<296, 256, 0, st>>>(spec, L[0], L[1], hp, kd[0], kd[1], kd[2], scale,
                                                       khat + q * oct);
            CK(cudaGetLastError());
        }
        CK(cudaStreamSynchronize(st));
        rc = MM_OK;
    }
fail:
    if (K) cudaFree(K);
    if (spec) cudaFree(spec);
    if (dmax) cudaFree(dmax);
    return rc;
}


// Exch6NgbrKernel (kernel_exchange.go:102-123), module demagexch: the 6-neighbour
// Laplacian as a convolution kernel on the padded grid, written in the reference's
// order (centre, then the +-1 neighbours along x, y, z with wrapped indices,
// kernel.go:19-27; along a dimension of size 1 the neighbour writes overwrite the
// centre) and rounded to float as the reference stores it.  Its FP64 transform (real
// part / prod L, one octant) goes to kex[kd0][kd1][kd2]; it is the same for xx, yy, zz.
int build_exchange_kernel(const int L[3], const double cell[3], float* kex, const int kd[3], cudaStream_t st,
                          char* err, int errlen) {
    const long long NL = (long long)L[0] * L[1] * L[2];
    const int M = L[2] / 2;
    const int hp = M + 1;
    double* K = nullptr;
    double2* spec = nullptr;
    int rc = MM_ERR_CUDA;
    {
        // host list of (index, value), later writes replacing earlier ones
        std::vector<std::pair<long long, double>> w;
        auto put = [&](int x, int y, int z, double v) {
            const long long idx = ((long long)wrap_i(x, L[0]) * L[1] + wrap_i(y, L[1])) * L[2] + wrap_i(z, L[2]);
            for (auto& e : w)
                if (e.first == idx) { e.second = v; return; }
            w.push_back({idx, v});
        };
        const double hx = cell[0] * cell[0], hy = cell[1] * cell[1], hz = cell[2] * cell[2];
        put(0, 0, 0, (float)(-2 / hx - 2 / hy - 2 / hz));
        put(+1, 0, 0, (float)(1 / hx));
        put(-1, 0, 0, (float)(1 / hx));
        put(0, +1, 0, (float)(1 / hy));
        put(0, -1, 0, (float)(1 / hy));
        put(0, 0, +1, (float)(1 / hz));
        put(0, 0, -1, (float)(1 / hz));
        CK(cudaMalloc(&K, sizeof(double) * NL));
        CK(cudaMemsetAsync(K, 0, sizeof(double) * NL, st));
        for (auto& e : w) CK(cudaMemcpyAsync(K + e.first, &e.second, sizeof(double), cudaMemcpyHostToDevice, st));
        CK(cudaMalloc(&spec, sizeof(double2) * (size_t)L[0] * L[1] * hp));
        PP none = {nullptr, nullptr, 0};
        CK(launch_xfwd<double2, double>(M, K, none, nullptr, spec, L[0] * L[1], L[0], L[1], L[1], L[2], L[2], hp,
                                        nullptr, nullptr, 0, st));
        if (L[1] > 1)
            CK(launch_colfft<double2>(L[1], -1, spec, hp, L[0], (long long)L[1] * hp, hp, L[1], L[1], nullptr, nullptr,
                                      0, st));
        if (L[0] > 1)
            CK(launch_colfft<double2>(L[0], -1, spec, hp, L[1], hp, (long long)L[1] * hp, L[0], L[0], nullptr, nullptr,
                                      0, st));
        extract_octant_kernel<<<296, 256, 0, st>>>(spec, L[0], L[1], hp, kd[0], kd[1], kd[2], 1.0 / (double)NL, kex);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));  // the host list must outlive the copies
        rc = MM_OK;
    }
fail:
    if (K) cudaFree(K);
    if (spec) cudaFree(spec);
    return rc;
}

// khat = kd + c * kex on the diagonal components (mod_demagexchange.go:145-157 with the
// Ms factor applied by the convolution passes: c = 2 Aex / (mu0 Ms^2)), kd elsewhere.
__global__ void combine_dex_kernel(const float* kd, const float* kex, long long oct, double c, float* khat) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 6 * oct;
         i += (long long)gridDim.x * blockDim.x) {
        const long long q = i / oct;
        khat[i] = q < 3 ? (float)((double)kd[i] + c * (double)kex[i - q * oct]) : kd[i];
    }
}

int combine_dex(const float* kd, const float* kex, long long oct, double c, float* khat, cudaStream_t st) {
    combine_dex_kernel<<<296, 256, 0, st>>>(kd, kex, oct, c, khat);
    return cudaGetLastError() == cudaSuccess ? MM_OK : MM_ERR_CUDA;
}

}  // namespace mm
