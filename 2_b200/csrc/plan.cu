// plan.cu -- plan object, time stepper and the fused-tier C-ABI (include/mm_b200.h).
//
// A plan owns every device buffer the hot path needs (spectrum, demag kernel octant,
// Runge-Kutta stages, control block, reduction partials), allocated once at
// mm_plan_create: nothing is allocated in a step (the reference allocates per call in
// maxwell_convolution.go:251 and solve_heun.go:47).
//
// Time stepping follows Solver.Step (src/mumax/engine/solver.go:14-17).  Each step
// attempt is a fixed sequence of launches whose pointers are resolved on the device
// from the control block (accepted-state ping-pong, retry and done flags), so attempts
// can be queued back to back, or replayed from a CUDA graph, without a host round trip.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fft.cuh"
#include "mm_internal.h"

namespace mm {
int build_demag_kernel(const int L[3], const double cell[3], const int pbc[3], int accuracy, float* khat,
                       const int kd[3], int nz[6], cudaStream_t st, char* err, int errlen);
}

using namespace mm;

static thread_local std::string g_err;
static int set_err(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}
namespace mm {
// lets other translation units report through mm_last_error()
int report_error(int code, const char* msg) { return set_err(code, "%s", msg); }
}  // namespace mm

#define CUCHK(...)                                                                                            \
    do {                                                                                                      \
        cudaError_t e_ = (__VA_ARGS__);                                                                               \
        if (e_ != cudaSuccess) return set_err(MM_ERR_CUDA, "%s: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

static const double PI = 3.14159265358979323846264338327950288;
static const double MU0 = 4.0 * PI * 1e-7;
static const double KB = 1.380650424E-23;
static const double MUB = 9.2740091523E-24;
static const double QE = 1.60217646E-19;
static const double HBAR = 1.054571726E-34;

// ---------------------------------------------------------------- device helpers
__global__ void normalize_kernel(float* m, const float* msat_mask, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        float norm = msat_mask ? msat_mask[i] : 1.0f;
        float x = m[i], y = m[N + i], z = m[2 * N + i];
        float mn = sqrtf(x * x + y * y + z * z);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        m[i] = x * sc;
        m[N + i] = y * sc;
        m[2 * N + i] = z * sc;
    }
}

// next = normalise(base + h * sum_j a_j K_j); h from the control block.
struct CombineArgs {
    PP base, next;
    int nk;
    PP kp[MM_MAXK];
    double ak[MM_MAXK];
    const float* msat_mask;
    long long N;
    DevCtl* ctl;
};

__global__ void combine_kernel(CombineArgs A) {
    const DevCtl* ctl = A.ctl;
    if (ctl->done) return;
    const int cur = ctl->cur;
    const float* base = A.base.get(cur);
    float* next = A.next.get(cur);
    const float* kp[MM_MAXK];
    float ak[MM_MAXK];
#pragma unroll
    for (int j = 0; j < MM_MAXK; j++) {
        kp[j] = j < A.nk ? A.kp[j].get(cur) : nullptr;
        ak[j] = j < A.nk ? (float)(A.ak[j] * ctl->h) : 0.f;
    }
    const long long N = A.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        float x = base[i], y = base[N + i], z = base[2 * N + i];
#pragma unroll
        for (int j = 0; j < MM_MAXK; j++) {
            if (j >= A.nk) break;
            x += ak[j] * kp[j][i];
            y += ak[j] * kp[j][N + i];
            z += ak[j] * kp[j][2 * N + i];
        }
        float norm = A.msat_mask ? A.msat_mask[i] : 1.0f;
        float mn = sqrtf(x * x + y * y + z * z);
        float sc = (norm == 0.0f) ? 0.0f : 1.0f;
        sc = (mn != 0.0f) ? sc / mn : 0.0f;
        next[i] = x * sc;
        next[N + i] = y * sc;
        next[2 * N + i] = z * sc;
    }
}

// Step controller of solve_rk12.go:156-210, generalised to error order q (RK12: q=1).
// Runs on one thread after the last evaluation of an attempt.
__global__ void controller_kernel(DevCtl* c, int adaptive, int q, int fsal, int nevals, int first_skippable) {
    if (c->done) return;
    c->attempts++;
    c->evals += nevals - ((first_skippable && c->tries > 0) ? 1 : 0);
    const double dt_used = c->dt;
    bool accept = true;
    if (adaptive) {
        const double err = (double)__uint_as_float(c->err_bits) * c->h;
        c->err = err;
        const double maxErr = c->maxerr;
        const bool bad = err > maxErr;
        if (bad) c->badsteps++;
        if ((!bad || c->tries == 10 - 1) && err > c->peakerr) c->peakerr = err;
        double factor = bad ? pow(maxErr / err, 1.0 / (q + 2)) : pow(maxErr / err, 1.0 / (q + 1));
        factor *= c->headroom;
        if (factor > 1.5) factor = 1.5;
        if (factor < 0.1) factor = 0.1;
        double newDt = dt_used * factor;
        if (newDt < c->mindt) newDt = c->mindt;
        if (newDt > c->maxdt) newDt = c->maxdt;
        c->dt = newDt;
        accept = !bad || newDt == c->mindt;
        if (!accept) {
            if (c->tries > 10) {
                c->status = MM_ERR_NOT_CONVERGED;
                c->done = 1;
            }
            c->tries++;
        }
    }
    c->err_bits = 0u;
    if (accept) {
        c->t += dt_used;
        c->step++;
        c->noise_step++;
        c->cur ^= 1;
        c->tries = 0;
        if (fsal) {
            c->fsal_valid = 1;
            c->maxtorque = sqrt((double)__uint_as_float(c->tq_bits)) * c->gamma;
            if (c->torque_thr > 0 && c->maxtorque < c->torque_thr) c->done = 1;
        }
        if (c->t >= c->t_end) c->done = 1;
        if (c->step >= c->step_end) c->done = 1;
    }
    if (!fsal && c->tq_bits) c->maxtorque = sqrt((double)__uint_as_float(c->tq_bits)) * c->gamma;
    c->tq_bits = 0u;
    if (c->status != MM_OK) c->done = 1;
    c->h = c->dt * c->gamma;
}

// run_until_smaller for non-FSAL solvers: the torque k0 of the current state is known
// after the first evaluation of an attempt (api.go:122-131 checks before each step).
__global__ void torque_check_kernel(DevCtl* c) {
    if (c->done) return;
    if (c->tries == 0) {
        c->maxtorque = sqrt((double)__uint_as_float(c->tq_bits)) * c->gamma;
        if (c->torque_thr > 0 && c->maxtorque < c->torque_thr) c->done = 1;
    }
    c->tq_bits = 0u;
}

// deterministic compensated finish of the block partials of the energy terms
__global__ void energy_finish_kernel(const float* red, int nblocks, double* out) {
    if (threadIdx.x >= 4) return;
    const int q = threadIdx.x;
    double s = 0.0;  // partial pairs are folded in fixed block order
    float fs = 0.f, fc = 0.f;
    for (int b = 0; b < nblocks; b++) {
        float v = red[b * 8 + 2 * q];
        float t = fs + v;
        if (fabsf(fs) >= fabsf(v)) fc += (fs - t) + v;
        else fc += (v - t) + fs;
        fs = t;
        fc += red[b * 8 + 2 * q + 1];
    }
    s = (double)fs + (double)fc;
    out[q] = s;
}

// compensated per-component sums of the state (for <m>)
__global__ void sum3_kernel(const float* m, long long N, float* red) {
    float s[3] = {0.f, 0.f, 0.f}, c[3] = {0.f, 0.f, 0.f};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        for (int q = 0; q < 3; q++) {
            float v = m[q * N + i];
            float t = s[q] + v;
            if (fabsf(s[q]) >= fabsf(v)) c[q] += (s[q] - t) + v;
            else c[q] += (v - t) + s[q];
            s[q] = t;
        }
    }
    __shared__ float sh[6][256];
    for (int q = 0; q < 3; q++) { sh[2 * q][threadIdx.x] = s[q]; sh[2 * q + 1][threadIdx.x] = c[q]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        int q = threadIdx.x;
        float fs = 0.f, fc = 0.f;
        for (int t = 0; t < blockDim.x; t++) {
            float v = sh[2 * q][t];
            float tt = fs + v;
            if (fabsf(fs) >= fabsf(v)) fc += (fs - tt) + v;
            else fc += (v - tt) + fs;
            fs = tt;
            fc += sh[2 * q + 1][t];
        }
        red[blockIdx.x * 8 + 2 * q] = fs;
        red[blockIdx.x * 8 + 2 * q + 1] = fc;
    }
}

// ---------------------------------------------------------------- plan
struct mm_plan_s {
    int device = 0;
    mm_problem prob;
    ConvGeom g;
    FieldParams P;
    bool demag = false;
    float* khat = nullptr;
    float2* tw = nullptr;            // FP32 twiddle table exp(-2 pi i k / 4096)
    KernelView kv;
    float2* S = nullptr;
    // solver state
    int solver = -1;
    float* Y[2] = {nullptr, nullptr};
    float* K1[2] = {nullptr, nullptr};
    float* Kst[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    float* Ma = nullptr;
    float* Mb = nullptr;
    float* Mtmp = nullptr;
    DevCtl* ctl = nullptr;
    DevCtl* ctl_host = nullptr;
    float* red = nullptr;
    int red_blocks = 0;
    double* dres = nullptr;
    unsigned int* tq = nullptr;
    bool state_set = false;
    bool run_until = false;
    long long launches = 0;          // kernels enqueued by this plan (graph replays counted per node)
    int graph_nodes = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_solver = -1;
    bool graph_run_until = false;
    long long bytes = 0;
};

static int dalloc(mm_plan p, void** ptr, size_t bytes) {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) return set_err(MM_ERR_CUDA, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    p->bytes += (long long)bytes;
    return MM_OK;
}

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fill_params(mm_plan p) {
    const mm_problem& q = p->prob;
    FieldParams& P = p->P;
    memset(&P, 0, sizeof P);
    P.demag = q.demag;
    P.exchange = q.exchange;
    P.anis = q.anis;
    P.zeeman = q.zeeman;
    P.thermal = q.thermal && q.temp != 0.0;
    P.zhangli = q.zhangli;
    P.slonczewski = q.slonczewski;
    for (int i = 0; i < 3; i++) { P.n[i] = q.n[i]; P.pbc[i] = q.pbc[i]; }
    P.N = (long long)q.n[0] * q.n[1] * q.n[2];
    P.msat = (float)q.msat;
    P.ex_pre = (float)(2.0 * q.aex / (MU0 * q.msat));
    for (int i = 0; i < 3; i++) P.cinv2[i] = (float)(1.0 / ((double)q.cell[i] * (double)q.cell[i]));
    P.alpha = (float)q.alpha;
    for (int i = 0; i < 3; i++) P.hz[i] = (float)(q.bext[i] / MU0);
    P.kmul = (float)(2.0 * q.ku / (MU0 * q.msat));
    for (int i = 0; i < 3; i++) P.anisu[i] = (float)q.anisu[i];
    P.therm_num = (float)(q.alpha * KB * 2.0 * q.temp);
    P.therm_den = MU0 * (q.cell[0] * q.cell[1] * q.cell[2]) * q.gamma * q.msat;
    P.seed = q.seed;
    P.zl_pre = (float)(q.zl_pol * MUB / (QE * q.msat));
    P.xi = (float)q.xi;
    for (int i = 0; i < 3; i++) {
        P.jmul[i] = (float)q.j[i];
        P.c12inv[i] = 1.0f / (12.0f * (float)q.cell[i]);
        P.p[i] = (float)q.p[i];
    }
    const double beta = HBAR * q.gamma / (MU0 * QE * q.msat);
    P.sl_beta_prime = (float)(q.sl_pol * beta);
    P.sl_pre_fld = (float)(beta * q.eps_prime);
    P.lambda = (float)q.lambda;
    P.t_fl = (float)q.t_fl;
    P.inv_gamma = (float)(1.0 / q.gamma);
    P.msat_mask = q.msat_mask;
    P.aex_mask = q.aex_mask;
    P.alpha_mask = q.alpha_mask;
    P.ku_mask = q.ku_mask;
    for (int i = 0; i < 3; i++) {
        P.anisu_mask[i] = q.anisu_mask[i];
        P.bext_mask[i] = q.bext_mask[i];
        P.j_mask[i] = q.j_mask[i];
        P.p_mask[i] = q.p_mask[i];
    }
    P.temp_mask = q.temp_mask;
    P.xi_mask = q.xi_mask;
    P.zl_pol_mask = q.zl_pol_mask;
    P.sl_pol_mask = q.sl_pol_mask;
    P.lambda_mask = q.lambda_mask;
    P.eps_prime_mask = q.eps_prime_mask;
    P.t_fl_mask = q.t_fl_mask;
}

static int read_ctl(mm_plan p, cudaStream_t st);
static int write_ctl(mm_plan p, cudaStream_t st);

static void free_graph(mm_plan p) {
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
}

extern "C" MM_API const char* mm_last_error(void) { return g_err.c_str(); }
extern "C" MM_API const char* mm_version(void) { return "mm_b200 0.1 (sm_100a)"; }

extern "C" MM_API int mm_plan_create(const mm_problem* prob, mm_plan* out) {
    if (!prob || !out) return set_err(MM_ERR_ARG, "null argument");
    *out = nullptr;
    for (int i = 0; i < 3; i++) {
        if (prob->n[i] < 1) return set_err(MM_ERR_ARG, "grid size must be >= 1");
        if (!(prob->cell[i] > 0)) return set_err(MM_ERR_ARG, "cell size must be > 0");
    }
    if (!(prob->msat != 0.0)) return set_err(MM_ERR_ARG, "Msat multiplier must be non-zero");
    if (!(prob->gamma != 0.0)) return set_err(MM_ERR_ARG, "gamma should be non-zero");
    mm_plan p = new mm_plan_s();
    cudaGetDevice(&p->device);
    p->prob = *prob;
    ConvGeom& g = p->g;
    for (int i = 0; i < 3; i++) {
        g.n[i] = prob->n[i];
        g.L[i] = (prob->n[i] > 1 && prob->pbc[i] == 0) ? 2 * prob->n[i] : prob->n[i];
    }
    g.N = (long long)g.n[0] * g.n[1] * g.n[2];
    fill_params(p);
    p->demag = prob->demag != 0;
    int rc = MM_OK;
    if (p->demag) {
        // Kernel_Arne's sanity checks (kernel_magnetostatic.go:36-45)
        if (!(g.L[1] > 1 && g.L[2] > 1 && g.L[1] % 2 == 0 && g.L[2] % 2 == 0 && (g.L[0] == 1 || g.L[0] % 2 == 0))) {
            delete p;
            return set_err(MM_ERR_ARG, "demag needs even padded sizes > 1 in y and x (got %d %d %d)", g.L[0], g.L[1],
                           g.L[2]);
        }
        if (!pow2(g.L[0]) || !pow2(g.L[1]) || !pow2(g.L[2]) || g.L[2] > 4096 || g.L[1] > 4096 || g.L[0] > 4096) {
            delete p;
            return set_err(MM_ERR_ARG, "demag transform sizes must be powers of two <= 4096 (got %d %d %d)", g.L[0],
                           g.L[1], g.L[2]);
        }
        g.M = g.L[2] / 2;
        g.h = g.M + 1;
        g.hp = (g.h + 3) & ~3;
        g.kd[0] = g.L[0] / 2 + 1;
        g.kd[1] = g.L[1] / 2 + 1;
        g.kd[2] = g.L[2] / 2 + 1;
        const long long oct = (long long)g.kd[0] * g.kd[1] * g.kd[2];
        if ((rc = dalloc(p, (void**)&p->khat, sizeof(float) * 6 * oct))) { delete p; return rc; }
        if ((rc = dalloc(p, (void**)&p->tw, sizeof(float2) * mmfft::TWN))) { mm_plan_destroy(p); return rc; }
        {
            std::vector<float2> h(mmfft::TWN);
            mmfft::make_twiddle_table(h.data());
            if (cudaMemcpy(p->tw, h.data(), sizeof(float2) * mmfft::TWN, cudaMemcpyHostToDevice) != cudaSuccess) {
                mm_plan_destroy(p);
                return set_err(MM_ERR_CUDA, "twiddle table upload failed");
            }
        }
        if ((rc = dalloc(p, (void**)&p->S, sizeof(float2) * 3 * (size_t)g.n[0] * g.L[1] * g.hp))) {
            mm_plan_destroy(p);
            return rc;
        }
        cudaStream_t st;
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        char err[512] = {0};
        int nz[6];
        rc = build_demag_kernel(g.L, prob->cell, prob->pbc, prob->demag_accuracy, p->khat, g.kd, nz, st, err,
                                sizeof err);
        cudaStreamDestroy(st);
        if (rc != MM_OK) {
            mm_plan_destroy(p);
            return set_err(rc, "demag kernel: %s", err);
        }
        p->kv.k = p->khat;
        p->kv.kd0 = g.kd[0];
        p->kv.kd1 = g.kd[1];
        p->kv.kd2 = g.kd[2];
        p->kv.L0 = g.L[0];
        p->kv.L1 = g.L[1];
        for (int q = 0; q < 6; q++) p->kv.nz[q] = nz[q];
    }
    const size_t vb = sizeof(float) * 3 * (size_t)g.N;
    void** bufs[] = {(void**)&p->Y[0], (void**)&p->Y[1], (void**)&p->K1[0], (void**)&p->K1[1], (void**)&p->Ma,
                     (void**)&p->Mb, (void**)&p->Mtmp};
    for (auto b : bufs)
        if ((rc = dalloc(p, b, vb))) { mm_plan_destroy(p); return rc; }
    for (int i = 0; i < 6; i++)
        if ((rc = dalloc(p, (void**)&p->Kst[i], vb))) { mm_plan_destroy(p); return rc; }
    if ((rc = dalloc(p, (void**)&p->ctl, sizeof(DevCtl)))) { mm_plan_destroy(p); return rc; }
    if (cudaMallocHost(&p->ctl_host, sizeof(DevCtl)) != cudaSuccess) {
        mm_plan_destroy(p);
        return set_err(MM_ERR_CUDA, "cudaMallocHost failed");
    }
    p->red_blocks = std::max(p->demag ? xinv_blocks(g.M, g.n[0] * g.n[1]) : 0, local_blocks(g.N));
    p->red_blocks = std::max(p->red_blocks, 148 * 4);
    if ((rc = dalloc(p, (void**)&p->red, sizeof(float) * 8 * p->red_blocks))) { mm_plan_destroy(p); return rc; }
    if ((rc = dalloc(p, (void**)&p->dres, sizeof(double) * 8))) { mm_plan_destroy(p); return rc; }
    if ((rc = dalloc(p, (void**)&p->tq, sizeof(unsigned int) * 4))) { mm_plan_destroy(p); return rc; }
    DevCtl c;
    memset(&c, 0, sizeof c);
    c.t_end = 1e300;
    c.step_end = (1LL << 62);
    c.maxerr = 1.0 / 2000;
    c.mindt = 1e-38;
    c.maxdt = 1e38;
    c.headroom = 0.8;
    c.dt = 1e-15;
    c.gamma = prob->gamma;
    c.h = c.dt * c.gamma;
    c.done = 1;
    if (cudaMemcpy(p->ctl, &c, sizeof c, cudaMemcpyHostToDevice) != cudaSuccess) {
        mm_plan_destroy(p);
        return set_err(MM_ERR_CUDA, "ctl init failed");
    }
    *out = p;
    return MM_OK;
}

extern "C" MM_API int mm_plan_destroy(mm_plan p) {
    if (!p) return MM_OK;
    free_graph(p);
    void* bufs[] = {p->khat, p->tw, p->S, p->Y[0], p->Y[1], p->K1[0], p->K1[1], p->Ma, p->Mb, p->Mtmp, p->ctl,
                    p->red, p->dres, p->tq};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (int i = 0; i < 6; i++)
        if (p->Kst[i]) cudaFree(p->Kst[i]);
    if (p->ctl_host) cudaFreeHost(p->ctl_host);
    delete p;
    return MM_OK;
}

extern "C" MM_API int mm_plan_set_problem(mm_plan p, const mm_problem* prob) {
    if (!p || !prob) return set_err(MM_ERR_ARG, "null argument");
    for (int i = 0; i < 3; i++)
        if (prob->n[i] != p->prob.n[i] || prob->cell[i] != p->prob.cell[i] || prob->pbc[i] != p->prob.pbc[i])
            return set_err(MM_ERR_ARG, "geometry of a plan cannot change");
    if ((prob->demag != 0) != p->demag) return set_err(MM_ERR_ARG, "demag on/off cannot change after plan creation");
    if (!(prob->msat != 0.0) || !(prob->gamma != 0.0)) return set_err(MM_ERR_ARG, "Msat and gamma must be non-zero");
    p->prob = *prob;
    fill_params(p);
    free_graph(p);
    // gamma is part of h = dt*gamma on the device
    int rc = read_ctl(p, 0);
    if (rc) return rc;
    p->ctl_host->gamma = prob->gamma;
    p->ctl_host->h = p->ctl_host->dt * prob->gamma;
    p->ctl_host->fsal_valid = 0;
    return write_ctl(p, 0);
}

extern "C" MM_API int mm_plan_kernel_nonzero(mm_plan p, int out6[6]) {
    if (!p || !out6) return set_err(MM_ERR_ARG, "null argument");
    for (int q = 0; q < 6; q++) out6[q] = p->demag ? p->kv.nz[q] : 0;
    return MM_OK;
}

extern "C" MM_API long long mm_plan_device_bytes(mm_plan p) { return p ? p->bytes : 0; }

// the register z-multiply applies when z is zero-padded (L0 = 2 N0) with N0 <= 16
static bool zreg_ok(const ConvGeom& g) {
    const int n0 = g.n[0];
    return g.L[0] == 2 * n0 && (n0 == 1 || n0 == 2 || n0 == 4 || n0 == 8 || n0 == 16);
}

// ---------------------------------------------------------------- one evaluation
// Launches the convolution passes (if demag) and the epilogue for one StageOp.
static int launch_eval(mm_plan p, const StageOp& op, DevCtl* ctl, int skip_retry, float* const* dbg,
                       long long noise_step, double dt_thermal, float* red, unsigned int* tq_out, cudaStream_t st,
                       int* nblocks_out) {
    const ConvGeom& g = p->g;
    EpiArgs A;
    memset(&A, 0, sizeof A);
    A.P = p->P;
    A.op = op;
    A.ctl = ctl;
    A.noise_step = noise_step;
    A.dt_thermal = dt_thermal;
    bool terms = op.want_energy != 0;
    for (int i = 0; i < 6; i++) {
        A.dbg[i] = dbg ? dbg[i] : nullptr;
        if (A.dbg[i]) terms = true;
    }
    A.red = red;
    A.tq_out = tq_out;
    A.skip_retry = skip_retry;
    int nb = 0;
    if (p->demag) {
        const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
        const int L0 = g.L[0], L1 = g.L[1];
        const long long plane = (long long)L1 * g.hp;
        CUCHK(launch_xfwd<float2, float>(g.M, nullptr, op.m_in, p->P.msat_mask, p->S, 3 * n0 * n1, n0, n1, L1, n2,
                                         n2, g.hp, p->tw, ctl, skip_retry, st));
        const float scale = (float)p->prob.msat;
        if (L0 == 1) {
            CUCHK(launch_colmul(L1, p->S, p->kv, g.h, 1, plane, 0, g.hp, n1, 1, scale, p->tw, ctl, skip_retry, st));
        } else {
            CUCHK(launch_colfft<float2>(L1, -1, p->S, g.h, 3 * n0, plane, g.hp, n1, L1, p->tw, ctl, skip_retry, st));
            if (zreg_ok(g))
                CUCHK(launch_zmul_reg(n0, p->S, p->kv, L1, g.h, g.hp, (long long)n0 * plane, plane, scale, p->tw, ctl,
                                      skip_retry, st));
            else
                CUCHK(launch_colmul(L0, p->S, p->kv, g.h, L1, (long long)n0 * plane, g.hp, plane, n0, 0, scale, p->tw,
                                    ctl, skip_retry, st));
            CUCHK(launch_colfft<float2>(L1, +1, p->S, g.h, 3 * n0, plane, g.hp, L1, n1, p->tw, ctl, skip_retry, st));
        }
        CUCHK(launch_xinv_epi(g.M, p->S, g.hp, L1, p->tw, A, terms, st, &nb));
        p->launches += (L0 == 1) ? 3 : 5;
    } else {
        CUCHK(launch_local_epi(A, terms, st, &nb));
        p->launches += 1;
    }
    if (nblocks_out) *nblocks_out = nb;
    return MM_OK;
}

static PP fixed(float* q) { return PP{q, nullptr, 0}; }
static PP cur_of(float* const* q) { return PP{q[0], q[1], 1}; }
static PP oth_of(float* const* q) { return PP{q[0], q[1], 2}; }
static PP none() { return PP{nullptr, nullptr, 0}; }

static StageOp op_blank() {
    StageOp o;
    memset(&o, 0, sizeof o);
    o.kcur = -1;
    o.ecur = -1;
    return o;
}

extern "C" MM_API int mm_fields(mm_plan p, const float* m, long long noise_step, double dt_thermal, float* h_demag,
                                float* h_ex, float* h_anis, float* h_zee, float* h_therm, float* h_eff,
                                mm_stream stream) {
    if (!p || !m) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    StageOp op = op_blank();
    op.m_in = fixed(const_cast<float*>(m));
    float* dbg[6] = {h_demag, h_ex, h_anis, h_zee, h_therm, h_eff};
    return launch_eval(p, op, nullptr, 0, dbg, noise_step, dt_thermal, nullptr, nullptr, st, nullptr);
}

static int normalize_launch(mm_plan p, float* m, cudaStream_t st) {
    int b = local_blocks(p->g.N);
    normalize_kernel<<<b, 256, 0, st>>>(m, p->P.msat_mask, p->g.N);
    CUCHK(cudaGetLastError());
    return MM_OK;
}

extern "C" MM_API int mm_torque(mm_plan p, float* m, long long noise_step, double dt_thermal, float* torque,
                                mm_stream stream) {
    if (!p || !m || !torque) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = normalize_launch(p, m, st);
    if (rc) return rc;
    StageOp op = op_blank();
    op.m_in = fixed(m);
    op.k_out = fixed(torque);
    return launch_eval(p, op, nullptr, 0, nullptr, noise_step, dt_thermal, nullptr, nullptr, st, nullptr);
}

// ---------------------------------------------------------------- solvers
// Butcher tableaux.  Bogacki-Shampine 3(2) and Dormand-Prince 5(4), both FSAL.
static const double BS_A[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {0, 0.75, 0, 0}, {2. / 9, 1. / 3, 4. / 9, 0}};
static const double BS_E[4] = {2. / 9 - 7. / 24, 1. / 3 - 1. / 4, 4. / 9 - 1. / 3, -1. / 8};
static const double DP_A[7][7] = {
    {0, 0, 0, 0, 0, 0, 0},
    {1. / 5, 0, 0, 0, 0, 0, 0},
    {3. / 40, 9. / 40, 0, 0, 0, 0, 0},
    {44. / 45, -56. / 15, 32. / 9, 0, 0, 0, 0},
    {19372. / 6561, -25360. / 2187, 64448. / 6561, -212. / 729, 0, 0, 0},
    {9017. / 3168, -355. / 33, 46732. / 5247, 49. / 176, -5103. / 18656, 0, 0},
    {35. / 384, 0, 500. / 1113, 125. / 192, -2187. / 6784, 11. / 84, 0}};
static const double DP_E[7] = {35. / 384 - 5179. / 57600, 0, 500. / 1113 - 7571. / 16695,
                               125. / 192 - 393. / 640, -2187. / 6784 + 92097. / 339200,
                               11. / 84 - 187. / 2100, -1. / 40};

static int launch_combine(mm_plan p, PP base, PP next, int nk, const PP* kp, const double* ak, cudaStream_t st) {
    CombineArgs A;
    memset(&A, 0, sizeof A);
    A.base = base;
    A.next = next;
    A.nk = 0;
    for (int j = 0; j < nk; j++) {
        if (ak[j] == 0.0) continue;
        A.kp[A.nk] = kp[j];
        A.ak[A.nk] = ak[j];
        A.nk++;
    }
    A.msat_mask = p->P.msat_mask;
    A.N = p->g.N;
    A.ctl = p->ctl;
    combine_kernel<<<local_blocks(p->g.N), 256, 0, st>>>(A);
    CUCHK(cudaGetLastError());
    p->launches++;
    return MM_OK;
}

// Enqueues one step attempt of the configured solver (no host synchronisation).
static int enqueue_attempt(mm_plan p, cudaStream_t st) {
    DevCtl* ctl = p->ctl;
    int rc;
    const int s = p->solver;
    if (s == MM_EULER || s == MM_HEUN || s == MM_RK12) {
        // eval k0 at the accepted state
        StageOp o0 = op_blank();
        o0.m_in = cur_of(p->Y);
        o0.k_out = fixed(p->Kst[0]);
        o0.want_tq = 1;
        if (s == MM_EULER) {
            o0.do_combine = 1;
            o0.base_is_cur = 1;
            o0.next = oth_of(p->Y);
            o0.nk = 1;
            o0.kcur = 0;
            o0.kp[0] = fixed(p->Kst[0]);
            o0.ak[0] = 1.0;
        } else if (s == MM_HEUN) {
            o0.do_combine = 1;
            o0.base_is_cur = 1;
            o0.next = fixed(p->Ma);
            o0.nk = 1;
            o0.kcur = 0;
            o0.kp[0] = fixed(p->Kst[0]);
            o0.ak[0] = 1.0;
        }
        const int skip = (s == MM_RK12) ? 1 : 0;
        if ((rc = launch_eval(p, o0, ctl, skip, nullptr, 0, 0, nullptr, nullptr, st, nullptr))) return rc;
        if (p->run_until) {
            torque_check_kernel<<<1, 1, 0, st>>>(ctl);
            CUCHK(cudaGetLastError());
            p->launches++;
        }
        if (s == MM_RK12) {
            // Euler predictor from the saved k0 (solve_rk12.go:133), also on retries
            PP kp[1] = {fixed(p->Kst[0])};
            double ak[1] = {1.0};
            if ((rc = launch_combine(p, cur_of(p->Y), fixed(p->Ma), 1, kp, ak, st))) return rc;
        }
        if (s == MM_HEUN || s == MM_RK12) {
            // corrector: y = y_pred + h/2 k1 - h/2 k0 (solve_rk12.go:154, solve_heun.go:63)
            StageOp o1 = op_blank();
            o1.m_in = fixed(p->Ma);
            o1.do_combine = 1;
            o1.base_is_cur = 1;
            o1.next = oth_of(p->Y);
            o1.nk = 2;
            o1.kcur = 0;
            o1.kp[0] = none();
            o1.ak[0] = 0.5;
            o1.kp[1] = fixed(p->Kst[0]);
            o1.ak[1] = -0.5;
            if (s == MM_RK12) {
                o1.ne = 2;
                o1.ecur = 0;
                o1.ep[0] = none();
                o1.ek[0] = 1.0;
                o1.ep[1] = fixed(p->Kst[0]);
                o1.ek[1] = -1.0;
            }
            if ((rc = launch_eval(p, o1, ctl, 0, nullptr, 0, 0, nullptr, nullptr, st, nullptr))) return rc;
        }
        controller_kernel<<<1, 1, 0, st>>>(ctl, s == MM_RK12 ? 1 : 0, 1, 0, s == MM_EULER ? 1 : 2, s == MM_RK12);
        CUCHK(cudaGetLastError());
        p->launches++;
        return MM_OK;
    }
    // RK23 / RK45 (FSAL): K1[cur] = f(Y[cur]) is valid
    const bool dp = (s == MM_RK45);
    const int S = dp ? 7 : 4;
    auto A = [&](int i, int j) { return dp ? DP_A[i][j] : BS_A[i][j]; };
    const double* E = dp ? DP_E : BS_E;
    // k-buffer of stage j: stage 0 = K1[cur], stages 1..S-2 = Kst[j-1], stage S-1 = K1[other]
    auto kbuf = [&](int j) -> PP {
        if (j == 0) return cur_of(p->K1);
        if (j == S - 1) return oth_of(p->K1);
        return fixed(p->Kst[j - 1]);
    };
    // stage-state buffer of stage i (1..S-1): alternate Ma/Mb, the last is Y[other]
    auto mbuf = [&](int i) -> PP {
        if (i == S - 1) return oth_of(p->Y);
        return fixed((i & 1) ? p->Ma : p->Mb);
    };
    {
        PP kp[1] = {kbuf(0)};
        double ak[1] = {A(1, 0)};
        if ((rc = launch_combine(p, cur_of(p->Y), mbuf(1), 1, kp, ak, st))) return rc;
    }
    for (int i = 1; i < S; i++) {
        StageOp o = op_blank();
        o.m_in = mbuf(i);
        o.k_out = kbuf(i);
        if (i + 1 < S) {
            o.do_combine = 1;
            o.base = cur_of(p->Y);
            o.next = mbuf(i + 1);
            o.nk = 0;
            for (int j = 0; j <= i; j++) {
                double a = A(i + 1, j);
                if (a == 0.0) continue;
                if (j == i) o.kcur = o.nk;
                o.kp[o.nk] = (j == i) ? none() : kbuf(j);
                o.ak[o.nk] = a;
                o.nk++;
            }
        } else {
            o.want_tq = 1;
            o.ne = 0;
            for (int j = 0; j < S; j++) {
                if (E[j] == 0.0) continue;
                if (j == i) o.ecur = o.ne;
                o.ep[o.ne] = (j == i) ? none() : kbuf(j);
                o.ek[o.ne] = E[j];
                o.ne++;
            }
        }
        if ((rc = launch_eval(p, o, ctl, 0, nullptr, 0, 0, nullptr, nullptr, st, nullptr))) return rc;
    }
    controller_kernel<<<1, 1, 0, st>>>(ctl, 1, dp ? 4 : 2, 1, S - 1, 0);
    CUCHK(cudaGetLastError());
    p->launches++;
    return MM_OK;
}

static int read_ctl(mm_plan p, cudaStream_t st) {
    CUCHK(cudaMemcpyAsync(p->ctl_host, p->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    return MM_OK;
}
static int write_ctl(mm_plan p, cudaStream_t st) {
    CUCHK(cudaMemcpyAsync(p->ctl, p->ctl_host, sizeof(DevCtl), cudaMemcpyHostToDevice, st));
    CUCHK(cudaStreamSynchronize(st));
    return MM_OK;
}

extern "C" MM_API int mm_solver_init(mm_plan p, int solver, double dt, double mindt, double maxdt, double maxerr) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    if (solver < MM_EULER || solver > MM_RK45) return set_err(MM_ERR_ARG, "unknown solver %d", solver);
    if (!(dt > 0) || !(mindt > 0) || !(maxdt > 0) || !(maxerr > 0)) return set_err(MM_ERR_ARG, "dt, mindt, maxdt, maxerr must be > 0");
    p->solver = solver;
    free_graph(p);
    int rc = read_ctl(p, 0);
    if (rc) return rc;
    DevCtl& c = *p->ctl_host;
    c.dt = dt;
    c.mindt = mindt;
    c.maxdt = maxdt;
    c.maxerr = maxerr;
    c.headroom = 0.8;
    c.gamma = p->prob.gamma;
    c.h = dt * c.gamma;
    c.fsal_valid = 0;
    c.tries = 0;
    c.status = MM_OK;
    return write_ctl(p, 0);
}

extern "C" MM_API int mm_set_state(mm_plan p, const float* m, int from_host, mm_stream stream) {
    if (!p || !m) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    float* dst = p->Y[p->ctl_host->cur];
    CUCHK(cudaMemcpyAsync(dst, m, sizeof(float) * 3 * p->g.N, from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
    if ((rc = normalize_launch(p, dst, st))) return rc;
    p->ctl_host->fsal_valid = 0;
    p->state_set = true;
    return write_ctl(p, st);
}

extern "C" MM_API int mm_get_state(mm_plan p, float* m, int to_host, mm_stream stream) {
    if (!p || !m) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    CUCHK(cudaMemcpyAsync(m, p->Y[p->ctl_host->cur], sizeof(float) * 3 * p->g.N,
                          to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
    CUCHK(cudaStreamSynchronize(st));
    return MM_OK;
}

extern "C" MM_API int mm_set_time(mm_plan p, double t, double dt) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    int rc = read_ctl(p, 0);
    if (rc) return rc;
    p->ctl_host->t = t;
    if (dt > 0) {
        p->ctl_host->dt = dt;
        p->ctl_host->h = dt * p->ctl_host->gamma;
    }
    return write_ctl(p, 0);
}

extern "C" MM_API int mm_set_thermal_dt(mm_plan p, double dt_thermal) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    int rc = read_ctl(p, 0);
    if (rc) return rc;
    p->ctl_host->dt_thermal = dt_thermal;
    return write_ctl(p, 0);
}

// FSAL solvers need f(Y[cur]) before the first attempt.
static int ensure_fsal(mm_plan p, cudaStream_t st) {
    if (p->solver != MM_RK23 && p->solver != MM_RK45) return MM_OK;
    if (p->ctl_host->fsal_valid) return MM_OK;
    // a standalone evaluation with the control block (done = 0 at this point)
    StageOp o = op_blank();
    o.m_in = cur_of(p->Y);
    o.k_out = cur_of(p->K1);
    o.want_tq = 1;
    int rc = launch_eval(p, o, p->ctl, 0, nullptr, 0, 0, nullptr, nullptr, st, nullptr);
    if (rc) return rc;
    if ((rc = read_ctl(p, st))) return rc;
    float tqv;
    memcpy(&tqv, &p->ctl_host->tq_bits, sizeof tqv);
    p->ctl_host->maxtorque = sqrt((double)tqv) * p->ctl_host->gamma;
    p->ctl_host->tq_bits = 0;
    p->ctl_host->fsal_valid = 1;
    return write_ctl(p, st);
}

static int capture_attempt(mm_plan p) {
    if (p->graph && p->graph_solver == p->solver && p->graph_run_until == p->run_until) return MM_OK;
    free_graph(p);
    cudaStream_t cs;
    CUCHK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t gr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { cudaStreamDestroy(cs); return set_err(MM_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e)); }
    const long long before = p->launches;
    int rc = enqueue_attempt(p, cs);
    p->graph_nodes = (int)(p->launches - before);
    p->launches = before;
    e = cudaStreamEndCapture(cs, &gr);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) return set_err(MM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&p->graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) { p->graph = nullptr; return set_err(MM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e)); }
    p->graph_solver = p->solver;
    p->graph_run_until = p->run_until;
    return MM_OK;
}

extern "C" MM_API int mm_queue_attempts(mm_plan p, int attempts, mm_stream stream) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    if (p->solver < 0) return set_err(MM_ERR_STATE, "no solver: call mm_solver_init");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = capture_attempt(p);
    if (rc) return rc;
    for (int a = 0; a < attempts; a++) CUCHK(cudaGraphLaunch(p->graph, st));
    p->launches += (long long)attempts * p->graph_nodes;
    return MM_OK;
}

// Runs attempts until the device sets `done`.  The host only polls the control block
// between batches of queued attempts.
static int drive(mm_plan p, cudaStream_t st, long long max_attempts) {
    int batch = 4;
    long long launched = 0;
    for (;;) {
        int rc = mm_queue_attempts(p, batch, (mm_stream)st);
        if (rc) return rc;
        launched += batch;
        if ((rc = read_ctl(p, st))) return rc;
        const DevCtl& c = *p->ctl_host;
        if (c.status == MM_ERR_NAN) return set_err(MM_ERR_NAN, "NaN in the torque at step %lld", c.step);
        if (c.status != MM_OK) return set_err(c.status, "solver cannot converge after 10 bad steps (step %lld)", c.step);
        if (c.done) return MM_OK;
        if (max_attempts > 0 && launched >= max_attempts) return set_err(MM_ERR_TIMEOUT, "attempt limit reached");
        if (batch < 64) batch *= 2;
    }
}

static int start_run(mm_plan p, cudaStream_t st, double t_end, long long step_end, double thr) {
    if (p->solver < 0) return set_err(MM_ERR_STATE, "no solver: call mm_solver_init");
    if (!p->state_set) return set_err(MM_ERR_STATE, "no state: call mm_set_state");
    int rc = read_ctl(p, st);
    if (rc) return rc;
    DevCtl& c = *p->ctl_host;
    c.done = 0;
    c.status = MM_OK;
    c.tries = 0;
    c.t_end = t_end;
    c.step_end = step_end;
    c.torque_thr = thr;
    c.err_bits = 0;
    c.tq_bits = 0;
    c.gamma = p->prob.gamma;
    c.h = c.dt * c.gamma;
    p->run_until = thr > 0;
    if ((rc = write_ctl(p, st))) return rc;
    if ((rc = ensure_fsal(p, st))) return rc;
    if (thr > 0 && (p->solver == MM_RK23 || p->solver == MM_RK45)) {
        if ((rc = read_ctl(p, st))) return rc;
        if (p->ctl_host->maxtorque < thr) {
            p->ctl_host->done = 1;
            return write_ctl(p, st);
        }
    }
    return MM_OK;
}

static int finish_run(mm_plan p, cudaStream_t st) {
    int rc = read_ctl(p, st);
    if (rc) return rc;
    p->ctl_host->done = 1;
    p->ctl_host->t_end = 1e300;
    p->ctl_host->step_end = (1LL << 62);
    p->ctl_host->torque_thr = 0;
    p->run_until = false;
    return write_ctl(p, st);
}

extern "C" MM_API int mm_run(mm_plan p, double duration, mm_stream stream) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    const double t0 = p->ctl_host->t;
    if (!(t0 < t0 + duration)) return MM_OK;
    if ((rc = start_run(p, st, t0 + duration, (1LL << 62), 0))) return rc;
    rc = drive(p, st, 0);
    int rc2 = finish_run(p, st);
    return rc ? rc : rc2;
}

extern "C" MM_API int mm_steps(mm_plan p, long long n, mm_stream stream) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    if (n <= 0) return MM_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    const long long s0 = p->ctl_host->step;
    if ((rc = start_run(p, st, 1e300, s0 + n, 0))) return rc;
    rc = drive(p, st, 0);
    int rc2 = finish_run(p, st);
    return rc ? rc : rc2;
}

extern "C" MM_API int mm_step(mm_plan p, mm_stream stream) { return mm_steps(p, 1, stream); }

extern "C" MM_API int mm_run_until_maxtorque(mm_plan p, double thr, long long max_steps, mm_stream stream) {
    if (!p) return set_err(MM_ERR_ARG, "null plan");
    if (!(thr > 0)) return set_err(MM_ERR_ARG, "threshold must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    const long long s0 = p->ctl_host->step;
    if ((rc = start_run(p, st, 1e300, max_steps > 0 ? s0 + max_steps : (1LL << 62), thr))) return rc;
    rc = drive(p, st, 0);
    int rc2 = finish_run(p, st);
    return rc ? rc : rc2;
}

extern "C" MM_API int mm_get_stats(mm_plan p, mm_stats* out, mm_stream stream) {
    if (!p || !out) return set_err(MM_ERR_ARG, "null argument");
    int rc = read_ctl(p, (cudaStream_t)stream);
    if (rc) return rc;
    const DevCtl& c = *p->ctl_host;
    out->t = c.t;
    out->dt = c.dt;
    out->err = c.err;
    out->peakerr = c.peakerr;
    out->maxtorque = c.maxtorque;
    out->step = c.step;
    out->badsteps = c.badsteps;
    out->attempts = c.attempts;
    out->evals = c.evals;
    out->status = c.status;
    out->done = c.done;
    return MM_OK;
}

// ---------------------------------------------------------------- reductions of the state
extern "C" MM_API int mm_maxtorque(mm_plan p, double* out, mm_stream stream) {
    if (!p || !out) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    CUCHK(cudaMemsetAsync(p->tq, 0, sizeof(unsigned int), st));
    StageOp o = op_blank();
    o.m_in = fixed(p->Y[p->ctl_host->cur]);
    o.k_out = fixed(p->Mtmp);
    o.want_tq = 1;
    if ((rc = launch_eval(p, o, nullptr, 0, nullptr, p->ctl_host->noise_step,
                          p->ctl_host->dt_thermal > 0 ? p->ctl_host->dt_thermal : p->ctl_host->dt, nullptr, p->tq,
                          st, nullptr)))
        return rc;
    unsigned int bits = 0;
    CUCHK(cudaMemcpyAsync(&bits, p->tq, sizeof bits, cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    float v;
    memcpy(&v, &bits, sizeof v);
    *out = sqrt((double)v) * p->prob.gamma;
    return MM_OK;
}

extern "C" MM_API int mm_average(mm_plan p, double out[3], mm_stream stream) {
    if (!p || !out) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    const int nb = std::min(p->red_blocks, 148 * 2);
    sum3_kernel<<<nb, 256, 0, st>>>(p->Y[p->ctl_host->cur], p->g.N, p->red);
    CUCHK(cudaGetLastError());
    energy_finish_kernel<<<1, 32, 0, st>>>(p->red, nb, p->dres);
    CUCHK(cudaGetLastError());
    double r[4];
    CUCHK(cudaMemcpyAsync(r, p->dres, sizeof r, cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    for (int c = 0; c < 3; c++) out[c] = r[c] / (double)p->g.N;
    return MM_OK;
}

extern "C" MM_API int mm_energy(mm_plan p, double out[5], mm_stream stream) {
    if (!p || !out) return set_err(MM_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    StageOp o = op_blank();
    o.m_in = fixed(p->Y[p->ctl_host->cur]);
    o.want_energy = 1;
    // thermal noise does not enter the energy terms
    int nb = 0;
    if ((rc = launch_eval(p, o, nullptr, 0, nullptr, 0, 1.0, p->red, nullptr, st, &nb))) return rc;
    energy_finish_kernel<<<1, 32, 0, st>>>(p->red, nb, p->dres);
    CUCHK(cudaGetLastError());
    double r[4];
    CUCHK(cudaMemcpyAsync(r, p->dres, sizeof r, cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    const mm_problem& q = p->prob;
    const double V = q.cell[0] * q.cell[1] * q.cell[2];
    out[0] = q.zeeman ? -V * r[0] * q.msat : 0.0;
    out[1] = q.exchange ? -0.5 * V * MU0 * r[1] * q.msat : 0.0;
    out[2] = q.demag ? -0.5 * V * MU0 * r[2] * q.msat : 0.0;
    out[3] = q.anis ? -0.5 * V * MU0 * r[3] * q.msat : 0.0;
    out[4] = out[0] + out[1] + out[2] + out[3];
    return MM_OK;
}

extern "C" MM_API long long mm_plan_launch_count(mm_plan p) { return p ? p->launches : 0; }

// Times each pass of one right-hand-side evaluation (at the accepted state, result
// discarded) with CUDA events recorded on the launching stream between the passes;
// ms_out[i] = average duration of pass i over `reps` evaluations.  Pass order:
// 3-D: xfwd, y fwd, z mul, y inv, x inv + epilogue; 2-D: xfwd, y mul, x inv + epilogue;
// no demag: epilogue only.
extern "C" MM_API int mm_profile_eval(mm_plan p, int reps, double* ms_out, int* npass, mm_stream stream) {
    if (!p || !ms_out || !npass || reps < 1) return set_err(MM_ERR_ARG, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = read_ctl(p, st);
    if (rc) return rc;
    const ConvGeom& g = p->g;
    StageOp op = op_blank();
    op.m_in = fixed(p->Y[p->ctl_host->cur]);
    op.k_out = fixed(p->Mtmp);
    EpiArgs A;
    memset(&A, 0, sizeof A);
    A.P = p->P;
    A.op = op;
    const int np = p->demag ? (g.L[0] == 1 ? 3 : 5) : 1;
    *npass = np;
    std::vector<cudaEvent_t> ev(np + 1);
    for (auto& e : ev) CUCHK(cudaEventCreate(&e));
    std::vector<double> acc(np, 0.0);
    for (int r = -1; r < reps; r++) {  // r = -1: untimed warm-up evaluation
        int k = 0;
        CUCHK(cudaEventRecord(ev[k++], st));
        int nb = 0;
        if (p->demag) {
            const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
            const int L0 = g.L[0], L1 = g.L[1];
            const long long plane = (long long)L1 * g.hp;
            const float scale = (float)p->prob.msat;
            CUCHK(launch_xfwd<float2, float>(g.M, nullptr, op.m_in, p->P.msat_mask, p->S, 3 * n0 * n1, n0, n1, L1,
                                             n2, n2, g.hp, p->tw, nullptr, 0, st));
            CUCHK(cudaEventRecord(ev[k++], st));
            if (L0 == 1) {
                CUCHK(launch_colmul(L1, p->S, p->kv, g.h, 1, plane, 0, g.hp, n1, 1, scale, p->tw, nullptr, 0, st));
                CUCHK(cudaEventRecord(ev[k++], st));
            } else {
                CUCHK(launch_colfft<float2>(L1, -1, p->S, g.h, 3 * n0, plane, g.hp, n1, L1, p->tw, nullptr, 0, st));
                CUCHK(cudaEventRecord(ev[k++], st));
                if (zreg_ok(g))
                    CUCHK(launch_zmul_reg(n0, p->S, p->kv, L1, g.h, g.hp, (long long)n0 * plane, plane, scale, p->tw,
                                          nullptr, 0, st));
                else
                    CUCHK(launch_colmul(L0, p->S, p->kv, g.h, L1, (long long)n0 * plane, g.hp, plane, n0, 0, scale,
                                        p->tw, nullptr, 0, st));
                CUCHK(cudaEventRecord(ev[k++], st));
                CUCHK(launch_colfft<float2>(L1, +1, p->S, g.h, 3 * n0, plane, g.hp, L1, n1, p->tw, nullptr, 0, st));
                CUCHK(cudaEventRecord(ev[k++], st));
            }
            CUCHK(launch_xinv_epi(g.M, p->S, g.hp, L1, p->tw, A, false, st, &nb));
        } else {
            CUCHK(launch_local_epi(A, false, st, &nb));
        }
        CUCHK(cudaEventRecord(ev[k++], st));
        CUCHK(cudaEventSynchronize(ev[np]));
        if (r < 0) continue;
        for (int i = 0; i < np; i++) {
            float ms = 0.f;
            CUCHK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            acc[i] += ms;
        }
    }
    for (int i = 0; i < np; i++) ms_out[i] = acc[i] / reps;
    for (auto& e : ev) cudaEventDestroy(e);
    return MM_OK;
}

// Geometry of the plan's transform: L[3], M, h, hp, kd[3], nonzero kernel components.
extern "C" MM_API int mm_plan_geometry(mm_plan p, int* out12) {
    if (!p || !out12) return set_err(MM_ERR_ARG, "bad argument");
    const ConvGeom& g = p->g;
    int v[12] = {g.L[0], g.L[1], g.L[2], g.M, g.h, g.hp, g.kd[0], g.kd[1], g.kd[2], 0, 0, 0};
    int nzc = 0;
    for (int q = 0; q < 6; q++) nzc += p->demag ? p->kv.nz[q] : 0;
    v[9] = nzc;
    v[10] = p->demag ? 1 : 0;
    memcpy(out12, v, sizeof v);
    return MM_OK;
}
