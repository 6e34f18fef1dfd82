// mm_internal.h -- internal structures shared by the kernels and the host runtime.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mm_b200.h"

namespace mm {

// Spectrum layout (the half-spectrum buffer that the convolution passes work in):
//   S[((c*N0 + z)*L1 + y)*hp + kx],  c in 0..2, z < N0, y < L1, kx < h = L2/2+1
// Only z < N0 rows exist: the z transform is done forward, multiplied and inverted
// inside one pass, so the padded z half never reaches HBM.
struct ConvGeom {
    int n[3];     // grid (internal order)
    int L[3];     // padded sizes
    int M;        // L2/2 : complex length of the row transform
    int h;        // L2/2 + 1 : stored half-spectrum columns
    int hp;       // row pitch of S in complex elements
    int kd[3];    // stored kernel octant: L0/2+1, L1/2+1, L2/2+1
    long long N;  // cells
};

// Device-side control block of the time stepper.  One per simulation; all kernels of an
// attempt read their simulation's block, the controller kernel writes it.  Every decision (accept/reject,
// dt, done) is made on the device so that attempts can be queued without host syncs.
struct DevCtl {
    double t, dt;            // time of the accepted state, dt for the next attempt
    double t_end;            // stop when t >= t_end
    long long step_end;      // stop when step >= step_end
    double maxerr, mindt, maxdt, headroom;
    double err, peakerr;     // last error estimate, all-time max of accepted errors
    double torque_thr;       // stop when maxtorque < torque_thr (<= 0: off)
    double maxtorque;        // gamma * max|tau| of the last evaluated derivative
    double gamma;
    double h;                // dt * gamma used by the current attempt
    unsigned int err_bits;   // max |sum e_j k_j| over cells/components (float bits)
    unsigned int tq_bits;    // max |tau|^2 over cells (float bits)
    int cur;                 // which ping-pong state holds the accepted state
    int done;                // 1: target reached -> kernels are no-ops
    int tries;               // rejected attempts of the current step
    int status;              // MM_OK, MM_ERR_NOT_CONVERGED, MM_ERR_NAN
    int fsal_valid;          // derivative buffer K1[cur] holds f(Y[cur])
    int pad0;
    long long step, badsteps, attempts, evals;
    long long noise_step;    // thermal noise counter (advanced once per accepted step)
    double dt_thermal;       // > 0: fixed dt for the thermal scale (cutoff_dt), else dt
    // autotabulate on the device (notify_tabulate.go:23-28): after an accepted step with
    // t - count*period >= period a record is due (tab_pending), written by the record
    // kernels of the same attempt into this simulation's rows
    double tab_period;       // <= 0: off
    long long tab_count;     // records due so far (the reference's count)
    long long tab_lost;      // records that found the buffer full
    int tab_n, tab_cap;      // rows written since the last read, capacity
    int tab_pending;
    int save_pending;        // autosave (notify_autosave.go:25-31): a state copy is due
    double save_period;      // <= 0: off
    double save_start;       // time autosave was turned on
    long long save_count, save_lost;
    int save_n, save_cap;    // states held since the last read, capacity
    // solver/am12 (solve_am01.go:46-301), see am12.cu
    double am_abs_err, am_rel_err;   // m_maxAbsError, m_maxRelError
    double am_er;            // error of the previous fixed-point iteration
    double am_alpha;         // convergence ratio of the last iteration
    double am_alpha_bdf;     // last predictor ratio (kept across steps)
    long long am_iterations; // iterations of the current step (bdf_iterations)
    int am_iter;             // iterations of the current loop
    int am_phase;            // loop state: 0 running, 1 converged, 2 failed
    int am_skip;             // the remaining kernels of the loop / attempt do nothing
    int am_restrict;         // limit the next dt by the predictor ratio
    int am_try;              // bad steps of this step (the reference's try)
    unsigned int am_red[6];  // max |y - yb| and max |yb| per component (float bits)
};

// Written by the controller after every attempt: what the host polls between batches.
struct CtlSummary {
    int active;              // simulations not done
    int status;              // first non-OK status among the simulations, else MM_OK
    int bad_sim;             // the simulation that set it
    int pad;
    long long step;          // step counter of bad_sim
    long long max_left;      // max over active simulations of step_end - step
};

// Scalars that may differ between the simulations of a batched plan (multipliers in
// SI units, pre-folded as the reference's updaters fold them on the host).
struct SimScalars {
    float msat;                 // Msat multiplier (A/m)
    float ex_pre;               // 2 Aex/(mu0 Msat)
    float alpha;
    float hz[3];                // B_ext/mu0 (A/m)
    float kmul;                 // 2 Ku/(mu0 Msat)
    float anisu[3];
    float therm_num;            // alpha * kB * 2 * T
    float zl_pre;               // P muB/(e Msat)
    float sl_beta_prime, sl_pre_fld;
    float jmul[3];              // current density multiplier (A/m^2)
    double therm_den;           // mu0 * V * gamma * Msat  (dt applied on device)
    unsigned long long seed;    // thermal Philox key
};

// Parameters of the effective field and torque, device pointers for masks
// (NULL = uniform 1), multipliers in SI units, internal axis order.
//
// Batched plans hold nsim simulations of one geometry.  Every per-cell array is laid
// out [sim][component][z][y][x] (sim stride 3N floats); kernels take the simulation
// from blockIdx.y.  Masks are shared (mask_bstride 0) or per simulation (N).
struct FieldParams {
    int demag, exchange, anis, zeeman, thermal, zhangli, slonczewski;
    int n[3];
    int pbc[3];
    long long N;
    SimScalars s;               // single-simulation scalars (sims == NULL)
    const SimScalars* sims;     // per-simulation scalars (device), or NULL
    long long bstride;          // 3N: floats between simulations in per-cell arrays
    long long mask_bstride;     // 0 (shared masks) or N
    float cinv2[3];             // 1/cell^2
    float xi;
    float c12inv[3];            // 1/(12 cell)
    float lambda, t_fl;
    float p[3];
    float inv_gamma;
    const float *msat_mask, *aex_mask, *alpha_mask, *ku_mask;
    const float *anisu_mask[3], *bext_mask[3], *j_mask[3];
    const float *temp_mask, *xi_mask, *zl_pol_mask;
    const float *p_mask[3];
    const float *sl_pol_mask, *lambda_mask, *eps_prime_mask, *t_fl_mask;
    // SetPointwise time tables (device, rows t v0 v1 v2): 0 = B_ext (T), 1 = j (A/m^2)
    struct TimeTable {
        const double* rows;
        int n;
        int pad;
    } tab[2];
};

// Selects which of the two ping-pong buffers is read/written, from ctl->cur:
// sel==0: fixed pointer p0; sel==1: the accepted side (p0 if cur==0 else p1);
// sel==2: the other side.  Resolved on the device so that attempts can be queued
// (or captured in a CUDA graph) without knowing whether earlier attempts were accepted.
struct PP {
    float* p0;
    float* p1;
    int sel;
    __host__ __device__ float* get(int cur) const {
        return sel == 0 ? p0 : (sel == 1 ? (cur ? p1 : p0) : (cur ? p0 : p1));
    }
};

// What the fused epilogue does with the derivative k it has just computed at a cell:
//   k_out[cell] = k
//   next[cell]  = normalise(B + h * sum_j ak[j] * K_j[cell])   (if do_combine)
//                 B = base[cell], or the evaluated state itself when base_is_cur;
//                 the term j == kcur uses k from registers
//   err        <- max over cells/components of |sum_j ek[j] * K_j[cell]|   (if ne > 0)
//   tq         <- max |k|^2                                               (if want_tq)
#define MM_MAXK 8
struct StageOp {
    PP m_in;
    PP k_out;
    int do_combine;
    int base_is_cur;
    PP base;
    PP next;
    int nk;
    int kcur;
    PP kp[MM_MAXK];
    double ak[MM_MAXK];
    int ne;
    int ecur;
    PP ep[MM_MAXK];
    double ek[MM_MAXK];
    int want_tq;
    int want_energy;
    int skip_if_retry;   // 1: skip when retrying (k0 of RK12/Heun/AM12); 2: skip while am_skip
    int pad;
    double c_time;       // the evaluation is at t + c_time * dt (time tables)
};

// Symmetric demag kernel in k-space, stored for one octant only:
// k[q][kz][ky][kx], kz <= L0/2, ky <= L1/2, kx <= L2/2; q = xx yy zz yz xz xy.
struct KernelView {
    const float* k;
    int kd0, kd1, kd2;
    int L0, L1;
    int nz[6];
};

// A Runge-Kutta stage state next = normalise(base + h * sum_j ak[j] * kp[j]) per cell, with
// the Msat mask as norm map (combine_kernel in plan.cu; combine_rows_kernel in rhs.cu also
// writes the state's R2C rows).
struct CombineArgs {
    PP base, next;
    int nk;
    PP kp[MM_MAXK];
    double ak[MM_MAXK];
    const float* msat_mask;
    long long N;
    long long bstride, mask_bstride;
    DevCtl* ctl;
    int no_norm;  // leave the result unnormalised (the AM12 Euler start)
};

// Arguments of the fused epilogue (rhs.cu).
struct EpiArgs {
    FieldParams P;
    StageOp op;
    DevCtl* ctl;               // NULL for a standalone evaluation
    long long noise_step;      // standalone thermal sample
    double dt_thermal;         // standalone thermal dt
    float* dbg[6];             // optional per-term outputs: demag, ex, anis, zee, therm, eff
    float* red;                // energy block partials [sim][block][8]
    unsigned int* tq_out;      // standalone max |k|^2 per simulation (float bits), may be NULL
    int skip_retry;
    long long spec_bstride;    // complex elements between simulations in the spectrum
    double t_eval;             // time of a standalone evaluation (time tables)
    // Row transform of the next stage state (four-step epilogue with op.do_combine only):
    // when fwd is set, the epilogue also writes the R2C rows of next (times the Msat mask
    // if fwd_mask) into fwd, the spectrum rows it has read, so that the next evaluation
    // starts at its column pass.
    float2* fwd;
    int fwd_mask;
    int fwd_pad;
};

#ifdef __CUDACC__
// skip_retry: 1 = the kernel belongs to a retried attempt's reusable first evaluation
// (skipped when tries > 0); 2 = an evaluation inside an AM12 fixed-point loop (skipped
// once the loop has ended or the attempt was abandoned)
__device__ __forceinline__ bool conv_skip(const DevCtl* ctl, int skip_retry) {
    return ctl && (ctl->done || (skip_retry == 1 && ctl->tries > 0) || (skip_retry == 2 && ctl->am_skip));
}
#endif

// ---- launchers (conv.cu, rhs.cu)
// Every launcher runs nsim simulations (gridDim.y = nsim); *_bstride are the element
// strides between simulations, ctl (if not NULL) points to nsim control blocks, and
// sim_scale (if not NULL) gives the demag scale per simulation.  `tile` (-1, 0, +1)
// selects the autotuner's variant of the rows or columns per block of the four-step
// row, column and epilogue passes (0 = default).
template <typename V, typename S>
cudaError_t launch_xfwd(int M, const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                        int in_pitch, int n_in, int hp, const float2* tw, const DevCtl* ctl, int skip_retry,
                        cudaStream_t st, int nsim = 1, long long in_bstride = 0, long long out_bstride = 0,
                        long long mask_bstride = 0, int tile = 0);
template <typename V>
cudaError_t launch_colfft(int L, int sign, V* S, int ncols, int nouter, long long outer_stride,
                          long long line_stride, int n_in, int n_out, const float2* tw, const DevCtl* ctl,
                          int skip_retry, cudaStream_t st, int nsim = 1, long long sim_stride = 0, int tile = 0);
cudaError_t launch_colmul(int L, float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                          long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                          const float2* tw, const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim = 1,
                          long long sim_stride = 0, const float* sim_scale = nullptr, int tile = 0);
cudaError_t launch_zmul_reg(int P, float2* S, const KernelView& K, int L1, int h, int hp, long long comp_stride,
                            long long zstride, float scale, const float2* tw, const DevCtl* ctl, int skip_retry,
                            cudaStream_t st, int nsim = 1, long long sim_stride = 0,
                            const float* sim_scale = nullptr);
cudaError_t launch_xinv_epi(int M, const float2* S, int hp, int L1, const float2* tw, const EpiArgs& A, bool terms,
                            cudaStream_t st, int* nblocks, int nsim = 1, int tile = 0);
cudaError_t launch_local_epi(const EpiArgs& A, bool terms, cudaStream_t st, int* nblocks, int nsim = 1);
// fused single-layer evaluation (rhs.cu): convolution and epilogue in one launch, one
// block per simulation; fused2d_ok tells whether a geometry is served
bool fused2d_ok(const int n[3]);
cudaError_t launch_fused2d(const float* in_mask, long long mask_bstride, const KernelView& K, float scale,
                           const float* sim_scale, const float2* tw, const EpiArgs& A, cudaStream_t st, int* nblocks,
                           int nsim);
// solver/am12 (am12.cu)
cudaError_t am_begin(DevCtl* ctl, int nsim, cudaStream_t st);
cudaError_t am_update(PP y0, PP y, const float* dy, const float* dy0, const float* y1, DevCtl* ctl, long long N,
                      int nsim, int bps, int mode, cudaStream_t st);
cudaError_t am_test(DevCtl* ctl, int nsim, int predictor, cudaStream_t st);
cudaError_t am_between(DevCtl* ctl, int nsim, int predictor, cudaStream_t st);
cudaError_t am_final(DevCtl* ctl, int nsim, cudaStream_t st);
cudaError_t am_copy(PP src, PP dst, const DevCtl* ctl, long long n3, int nsim, int bps, cudaStream_t st);
cudaError_t am_normalize(PP m, const float* msat_mask, const DevCtl* ctl, long long N, long long mask_bstride, int nsim,
                         int bps, int skip, cudaStream_t st);
int xinv_blocks(int M, int n0n1);
// mixed-radix passes (mixed.cu) for lengths that are not powers of two; the launchers of
// conv.cu and rhs.cu hand those lengths to them.  Their twiddle tables must have been
// prepared (mr_prepare, mixed.cuh) on the device for M and 2M, L1 and L0.
template <typename V, typename S>
cudaError_t launch_mr_xfwd(int M, const S* in, PP pp, const float* mask, V* out, int nrows, int Z, int Y, int Yout,
                           int in_pitch, int n_in, int hp, const DevCtl* ctl, int skip_retry, cudaStream_t st,
                           int nsim, long long in_bstride, long long out_bstride, long long mask_bstride);
template <typename V>
cudaError_t launch_mr_colfft(int L, int sign, V* S, int ncols, int nouter, long long outer_stride,
                             long long line_stride, int n_in, int n_out, const DevCtl* ctl, int skip_retry,
                             cudaStream_t st, int nsim, long long sim_stride);
cudaError_t launch_mr_colmul(int L, float2* S, const KernelView& K, int ncols, int nouter, long long comp_stride,
                             long long outer_stride, long long line_stride, int n_in, int kaxis, float scale,
                             const DevCtl* ctl, int skip_retry, cudaStream_t st, int nsim, long long sim_stride,
                             const float* sim_scale);
// whether the C2R + epilogue pass for row length M can also write the R2C rows of the
// next stage state (EpiArgs::fwd)
bool epi_r2c_supported(int M);
// combine_rows_kernel: the stage state of A (normalised, A.no_norm = 0) and its R2C rows
// into the spectrum S (times the Msat mask when fwd_mask), for M with epi_r2c_supported(M)
cudaError_t launch_combine_rows(int M, const CombineArgs& A, const int n[3], float2* S, int hp, int L1,
                                long long spec_bstride, const float2* tw, int fwd_mask, int nsim, cudaStream_t st);
int report_error(int code, const char* msg);  // sets mm_last_error()
int local_blocks(long long N, int nsim = 1);

}  // namespace mm
