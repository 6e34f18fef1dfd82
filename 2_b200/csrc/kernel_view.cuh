// Symmetric demag kernel lookup shared by the convolution passes (conv.cu) and the fused
// single-layer evaluation (rhs.cu).
#pragma once
#include "mm_internal.h"

namespace mm {
// The six components of the transformed kernel at (kz, ky, kx) of the full half
// spectrum, from the stored octant.
__device__ __forceinline__ void kernel_at(const KernelView& K, int kz, int ky, int kx, float out[6]) {
    float sz = 1.f, sy = 1.f;
    if (kz > (K.L0 >> 1)) { kz = K.L0 - kz; sz = -1.f; }
    if (ky > (K.L1 >> 1)) { ky = K.L1 - ky; sy = -1.f; }
    const int cs = K.kd0 * K.kd1 * K.kd2;
    const int idx = (kz * K.kd1 + ky) * K.kd2 + kx;
    // real-space K_sd is odd along axes s and d (s != d), so its transform flips sign
    // under k -> L-k along those axes; diagonal components are even.
    const float sg[6] = {1.f, 1.f, 1.f, sy, sz, sz * sy};
#pragma unroll
    for (int q = 0; q < 6; q++) out[q] = K.nz[q] ? sg[q] * __ldg(K.k + q * cs + idx) : 0.f;
}
}  // namespace mm
