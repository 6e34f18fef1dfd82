// noalloc.cu -- an entry point that allocates no device memory.
//
// mm_average computes <m> with block partial sums kept in its plan's workspace, which
// mm_plan_create allocates.  Some callers cannot allocate device memory at all: code
// running while a CUDA stream is being captured into a graph (cudaMalloc is not a
// capturable operation), engines whose device memory is owned by another allocator
// that has reserved the whole GPU (a Go array pool, a framework's caching allocator),
// or host code that must not block on the allocator.  mm_average_noalloc serves them:
// the caller passes the magnetisation and a 3-double output, and the partial sums live
// in a fixed file-scope device array (every GPU that loads this library holds it, 192
// KB, until the process exits).
#include <cstdio>
#include <mutex>

#include "mm_internal.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_CELLS_PER_THREAD = 8;
constexpr int NA_CELLS_PER_BLOCK = NA_THREADS * NA_CELLS_PER_THREAD;  // 2048
constexpr int NA_MAX_BLOCKS = 8192;
constexpr long long NA_MAX_CELLS = (long long)NA_CELLS_PER_BLOCK * NA_MAX_BLOCKS;  // 16,777,216
constexpr int NA_MAX_DEVICES = 64;

// per-block compensated partials: (sum, compensation) for each of the 3 components
static __device__ __align__(256) float g_na_partials[NA_MAX_BLOCKS * 6];

std::mutex g_na_mu;
float* g_na_ptr[NA_MAX_DEVICES] = {};

__device__ __forceinline__ void na_add(float& s, float& c, float v) {
    const float t = s + v;
    if (fabsf(s) >= fabsf(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
}

// Block b sums cells [b*2048, (b+1)*2048) of each component and writes its partials;
// every partial the finish kernel reads is written by this call, so nothing needs clearing.
__global__ void __launch_bounds__(NA_THREADS) na_partial_kernel(const float* __restrict__ m, long long N,
                                                                float* __restrict__ partials) {
    float s[3] = {0.f, 0.f, 0.f}, c[3] = {0.f, 0.f, 0.f};
    const long long base = (long long)blockIdx.x * NA_CELLS_PER_BLOCK;
#pragma unroll
    for (int j = 0; j < NA_CELLS_PER_THREAD; j++) {
        const long long i = base + j * NA_THREADS + threadIdx.x;
        if (i < N) {
#pragma unroll
            for (int q = 0; q < 3; q++) na_add(s[q], c[q], m[q * N + i]);
        }
    }
    __shared__ float sh[6][NA_THREADS];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        sh[2 * q][threadIdx.x] = s[q];
        sh[2 * q + 1][threadIdx.x] = c[q];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int q = threadIdx.x;
        float fs = 0.f, fc = 0.f;
        for (int t = 0; t < NA_THREADS; t++) {
            na_add(fs, fc, sh[2 * q][t]);
            fc += sh[2 * q + 1][t];
        }
        partials[blockIdx.x * 6 + 2 * q] = fs;
        partials[blockIdx.x * 6 + 2 * q + 1] = fc;
    }
}

// One thread per component sums the block partials serially (at most 8192, in block
// order): a few microseconds at the largest size, and deterministic.
__global__ void na_finish_kernel(const float* __restrict__ partials, int nblocks, long long N, double* out) {
    if (threadIdx.x >= 3) return;
    const int q = threadIdx.x;
    float fs = 0.f, fc = 0.f;
    for (int b = 0; b < nblocks; b++) {
        na_add(fs, fc, partials[b * 6 + 2 * q]);
        fc += partials[b * 6 + 2 * q + 1];
    }
    out[q] = ((double)fs + (double)fc) / (double)N;
}

// Device address of the scratch array on the current device, looked up once per device
// (the array's name is a host-side stand-in in host code, not a device address).  The
// cache is keyed by device number, so it assumes the runtime's primary context on each
// device and no cudaDeviceReset between calls: after a reset the module is loaded again
// and the cached address is stale.
int na_scratch(float** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return MM_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
        float* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_na_partials) != cudaSuccess || !p) return MM_ERR_CUDA;
        g_na_ptr[dev] = p;
    }
    *out = g_na_ptr[dev];
    return MM_OK;
}

}  // namespace

// <m> of a magnetisation without any device allocation.
//   m     : device, SoA float32, 3 x ncell (components contiguous, internal order)
//   ncell : 1 .. 16,777,216 cells (2048 cells per block x 8192 blocks of scratch);
//           larger sizes return MM_ERR_ARG
//   out   : device, 3 doubles: sum_i m_c[i] / ncell, compensated FP32 partial sums
// Asynchronous on `stream`.  The first call on a device looks up the scratch array's
// device address (cudaGetSymbolAddress) and should come before any stream capture on
// that device; the address is kept per device number (primary context, no
// cudaDeviceReset in between).  A CUDA error left pending by earlier work is reported,
// not attributed to this call's launches.  All calls share the one scratch array and it
// keeps the last call's contents, so calls that overlap on the GPU (different streams,
// or host threads without ordering) race: order them on one stream.
extern "C" MM_API int mm_average_noalloc(const float* m, long long ncell, double* out, mm_stream stream) {
    if (!m || !out) return mm::report_error(MM_ERR_ARG, "mm_average_noalloc: null m or out");
    if (ncell < 1 || ncell > NA_MAX_CELLS)
        return mm::report_error(MM_ERR_ARG,
                                "mm_average_noalloc: ncell must be in 1..16777216 (the fixed scratch array holds "
                                "8192 blocks of 2048 cells); use mm_average with a plan for larger grids");
    char msg[256];
    // an error the caller left pending would otherwise be read back after our launches
    // and reported as theirs: name it and stop
    const cudaError_t prior = cudaGetLastError();
    if (prior != cudaSuccess) {
        snprintf(msg, sizeof msg, "mm_average_noalloc: a CUDA error was pending before the call: %s",
                 cudaGetErrorString(prior));
        return mm::report_error(MM_ERR_CUDA, msg);
    }
    float* partials = nullptr;
    int rc = na_scratch(&partials);
    if (rc != MM_OK) return mm::report_error(rc, "mm_average_noalloc: cudaGetSymbolAddress of the scratch array failed");
    const int nblocks = (int)((ncell + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK);
    cudaStream_t st = (cudaStream_t)stream;
    na_partial_kernel<<<nblocks, NA_THREADS, 0, st>>>(m, ncell, partials);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        na_finish_kernel<<<1, 32, 0, st>>>(partials, nblocks, ncell, out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "mm_average_noalloc: launch failed: %s", cudaGetErrorString(e));
        return mm::report_error(MM_ERR_CUDA, msg);
    }
    return MM_OK;
}
