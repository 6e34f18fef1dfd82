// am12.cu -- device kernels of solver/am12 (solve_am01.go:46-301).
//
// One attempt of the reference's Step loop: explicit Euler start y = y0 + h dy0, an
// implicit-Euler predictor solved by fixed-point iteration (y <- y0 + h f(y)), a
// trapezoidal corrector solved the same way (y <- y0 + h/2 (f(y) + dy0)), and the
// predictor-corrector difference as the error that sets the next dt.  Each iteration's
// convergence test needs the max-norm of the update, so the loop is unrolled to its
// maximum length (6 iterations) and every kernel after a converged or failed test is a
// no-op (am_skip in the control block); the host never synchronises inside a step.
//
// Error norm of an update a -> b (solve_am01.go:129-137):
//   sqrt( sum_c (max|a_c - b_c| / (abs_err + max|b_c| rel_err))^2 / 3 ).
#include "mm_internal.h"

namespace mm {

enum { AM_BDF = 0, AM_TRAP = 1, AM_DIFF = 2 };

__device__ __forceinline__ double am_norm(const DevCtl* c) {
    double t = 0;
    for (int q = 0; q < 3; q++) {
        const double d = (double)__uint_as_float(c->am_red[q]);
        const double b = (double)__uint_as_float(c->am_red[3 + q]);
        const double r = d / (c->am_abs_err + b * c->am_rel_err);
        t += r * r;
    }
    return sqrt(t) / sqrt(3.0);
}

// Start of an attempt (one thread per simulation).  The step-level counters restart
// when the attempt opens a new step (tries == 0).
__global__ void am_begin_kernel(DevCtl* ctl, int nsim) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nsim; b += gridDim.x * blockDim.x) {
        DevCtl* c = ctl + b;
        if (c->done) continue;
        if (c->tries == 0) {
            c->am_iterations = 0;
            c->badsteps = 0;    // badsteps counts this step only (solve_am01.go:50)
            c->am_try = 0;
            c->evals++;         // the evaluation of dy0 at the start of the step
        }
        c->attempts++;
        c->evals++;             // the evaluation at the explicit Euler point
        c->am_skip = 0;
        c->am_phase = 0;
        c->am_iter = 0;
        c->am_er = 0.1;         // maxIterErr
        c->am_iterations++;     // solve_am01.go:96
        for (int q = 0; q < 6; q++) c->am_red[q] = 0u;
    }
}

// One fixed-point update (mode AM_BDF or AM_TRAP) of the iterate y in place, or the
// final predictor-corrector difference (AM_DIFF, y1 = the predictor, nothing written),
// with the max |y - b| and max |b| per component accumulated into the control block.
__global__ void __launch_bounds__(256) am_update_kernel(PP y0p, PP yp, const float* __restrict__ dy,
                                                        const float* __restrict__ dy0, const float* __restrict__ y1,
                                                        DevCtl* ctl, long long N, long long bstride, int mode) {
    DevCtl* c = ctl + blockIdx.y;
    if (c->done || c->am_skip) return;
    const int cur = c->cur;
    const long long off = blockIdx.y * bstride;
    const float* y0 = y0p.get(cur) + off;
    float* y = yp.get(cur) + off;
    const float h = (float)c->h;
    float md[3] = {0.f, 0.f, 0.f}, mb[3] = {0.f, 0.f, 0.f};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const long long k = q * N + i;
            float b;
            if (mode == AM_BDF) b = y0[k] + h * dy[off + k];
            else if (mode == AM_TRAP) b = y0[k] + 0.5f * h * (dy[off + k] + dy0[off + k]);
            else b = y1[off + k];
            const float a = y[k];
            md[q] = fmaxf(md[q], fabsf(a - b));
            mb[q] = fmaxf(mb[q], fabsf(b));
            if (mode != AM_DIFF) y[k] = b;
        }
    }
    __shared__ float s[6][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        for (int o = 16; o > 0; o >>= 1) {
            md[q] = fmaxf(md[q], __shfl_xor_sync(0xffffffffu, md[q], o));
            mb[q] = fmaxf(mb[q], __shfl_xor_sync(0xffffffffu, mb[q], o));
        }
        if (lane == 0) { s[q][w] = md[q]; s[3 + q][w] = mb[q]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        float v = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) v = fmaxf(v, s[threadIdx.x][k]);
        atomicMax(&c->am_red[threadIdx.x], __float_as_uint(v));
    }
}

// Convergence test after an update (one thread per simulation): target error reached,
// or the iteration diverges / runs out (solve_am01.go:143-160).
__global__ void am_test_kernel(DevCtl* ctl, int nsim, int predictor) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nsim; b += gridDim.x * blockDim.x) {
        DevCtl* c = ctl + b;
        if (c->done || c->am_skip) continue;
        const double err = am_norm(c);
        const double a = err / c->am_er;
        c->am_alpha = a;
        if (predictor) c->am_alpha_bdf = a;
        c->am_er = err;
        c->am_iter++;
        c->am_iterations++;
        for (int q = 0; q < 6; q++) c->am_red[q] = 0u;
        if (err <= 0.1) {
            c->am_phase = 1;
            c->am_skip = 1;
        } else if (a >= 1.0 || c->am_iter > 5) {
            c->am_phase = 2;
            c->am_skip = 1;
        } else {
            c->evals++;  // the RHS at the new iterate follows
        }
    }
}

// After a loop: a failed iteration abandons the attempt with a smaller dt
// (solve_am01.go:162-175, 229-240); a converged one opens the next loop.
__global__ void am_between_kernel(DevCtl* ctl, int nsim, int predictor) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nsim; b += gridDim.x * blockDim.x) {
        DevCtl* c = ctl + b;
        if (c->done || c->am_phase == 3) continue;
        if (c->am_phase == 2) {
            if (c->am_try == 10 - 1) {
                c->status = MM_ERR_NOT_CONVERGED;
                c->done = 1;
                continue;
            }
            const double dt = c->dt;
            c->dt = c->am_alpha > 0.6 ? dt * sqrt(0.6 / c->am_alpha) : 0.5 * dt;
            c->h = c->dt * c->gamma;
            if (predictor) c->am_restrict = 1;
            c->tries++;
            c->am_phase = 3;  // abandoned; am_skip stays set
            continue;
        }
        c->am_phase = 0;
        c->am_skip = 0;
        c->am_iter = 0;
        c->am_er = 0.1;
        for (int q = 0; q < 6; q++) c->am_red[q] = 0u;
    }
}

// End of an attempt: the predictor-corrector error sets dt; accept or retry
// (solve_am01.go:242-298).
__global__ void am_final_kernel(DevCtl* ctl, int nsim) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nsim; b += gridDim.x * blockDim.x) {
        DevCtl* c = ctl + b;
        if (c->done || c->am_phase == 3) continue;
        const double err = am_norm(c);
        for (int q = 0; q < 6; q++) c->am_red[q] = 0u;
        const double dt = c->dt;
        const bool bad = err > 1.0;
        if (bad) c->badsteps++;
        c->err = err;
        double nd = dt * sqrt(0.8 / err);
        if (c->am_restrict) {
            nd = fmin(nd, dt * sqrt(0.6 / c->am_alpha_bdf));
            c->am_restrict = 0;
        }
        if (nd < c->mindt) nd = c->mindt;
        if (nd > c->maxdt) nd = c->maxdt;
        c->dt = nd;
        c->h = nd * c->gamma;
        if (c->tq_bits) c->maxtorque = sqrt((double)__uint_as_float(c->tq_bits)) * c->gamma;
        c->tq_bits = 0u;
        if (!bad || nd == c->mindt) {
            if (err > c->peakerr) c->peakerr = err;
            c->t += dt;
            c->step++;
            c->noise_step++;
            c->cur ^= 1;
            c->tries = 0;
            if (c->t >= c->t_end) c->done = 1;
            if (c->step >= c->step_end) c->done = 1;
        } else {
            if (c->am_try > 10) {
                c->status = MM_ERR_NOT_CONVERGED;
                c->done = 1;
            }
            c->am_try++;
            c->tries++;
        }
    }
}

// y1 = y or dy = dybuf inside an attempt (skipped with the loop)
__global__ void am_copy_kernel(PP src, PP dst, const DevCtl* ctl, long long n3) {
    const DevCtl* c = ctl + blockIdx.y;
    if (c->done || c->am_skip) return;
    const long long off = blockIdx.y * n3;
    const float* s = src.get(c->cur) + off;
    float* d = dst.get(c->cur) + off;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
        d[i] = s[i];
}

// normalize.cu:14-42 on a device-resolved buffer: the pull of m before each RHS
// evaluation.  skip as for the evaluations (1: when retrying, 2: with the loop); 0 always
// runs (between runs, when the simulations are done).
__global__ void am_normalize_kernel(PP mp, const float* msat_mask, const DevCtl* ctl, long long N, long long bstride,
                                    long long mask_bstride, int skip) {
    const DevCtl* c = ctl + blockIdx.y;
    if (skip != 0 && (c->done || (skip == 1 && c->tries > 0) || (skip == 2 && c->am_skip))) return;
    float* m = mp.get(c->cur) + blockIdx.y * bstride;
    const float* msk = msat_mask ? msat_mask + blockIdx.y * mask_bstride : nullptr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const float norm = msk ? msk[i] : 1.0f;
        const float x = m[i], y = m[N + i], z = m[2 * N + i];
        const float mn = sqrtf(x * x + y * y + z * z);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        m[i] = x * sc;
        m[N + i] = y * sc;
        m[2 * N + i] = z * sc;
    }
}

// ---------------------------------------------------------------- launchers
static unsigned ctl_blocks(int nsim) { return (unsigned)((nsim + 127) / 128); }

cudaError_t am_begin(DevCtl* ctl, int nsim, cudaStream_t st) {
    am_begin_kernel<<<ctl_blocks(nsim), 128, 0, st>>>(ctl, nsim);
    return cudaGetLastError();
}
cudaError_t am_update(PP y0, PP y, const float* dy, const float* dy0, const float* y1, DevCtl* ctl, long long N,
                      int nsim, int bps, int mode, cudaStream_t st) {
    am_update_kernel<<<dim3((unsigned)bps, (unsigned)nsim), 256, 0, st>>>(y0, y, dy, dy0, y1, ctl, N, 3 * N, mode);
    return cudaGetLastError();
}
cudaError_t am_test(DevCtl* ctl, int nsim, int predictor, cudaStream_t st) {
    am_test_kernel<<<ctl_blocks(nsim), 128, 0, st>>>(ctl, nsim, predictor);
    return cudaGetLastError();
}
cudaError_t am_between(DevCtl* ctl, int nsim, int predictor, cudaStream_t st) {
    am_between_kernel<<<ctl_blocks(nsim), 128, 0, st>>>(ctl, nsim, predictor);
    return cudaGetLastError();
}
cudaError_t am_final(DevCtl* ctl, int nsim, cudaStream_t st) {
    am_final_kernel<<<ctl_blocks(nsim), 128, 0, st>>>(ctl, nsim);
    return cudaGetLastError();
}
cudaError_t am_copy(PP src, PP dst, const DevCtl* ctl, long long n3, int nsim, int bps, cudaStream_t st) {
    am_copy_kernel<<<dim3((unsigned)bps, (unsigned)nsim), 256, 0, st>>>(src, dst, ctl, n3);
    return cudaGetLastError();
}
cudaError_t am_normalize(PP m, const float* msat_mask, const DevCtl* ctl, long long N, long long mask_bstride, int nsim,
                         int bps, int skip, cudaStream_t st) {
    am_normalize_kernel<<<dim3((unsigned)bps, (unsigned)nsim), 256, 0, st>>>(m, msat_mask, ctl, N, 3 * N, mask_bstride,
                                                                              skip);
    return cudaGetLastError();
}

}  // namespace mm
