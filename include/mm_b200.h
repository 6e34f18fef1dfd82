/* mm_b200.h -- C-ABI of the B200-native micromagnetic hot path (fused tier).
 *
 * Plain C: pointers, sizes and status codes; no torch types.  All arrays are SoA
 * float32, one contiguous block per component, C order [z][y][x] in the reference's
 * INTERNAL axis order (Z,Y,X) = (0,1,2) (src/mumax/gpu/array.go:120-130,
 * src/mumax/engine/api.go:13,44).  Device pointers unless stated otherwise.
 *
 * Which reference interface each entry point replaces:
 *   mm_plan_create        MaxwellPlan.init/EnableDemag/loadDipoleKernel/LoadKernel
 *                         (src/mumax/modules/maxwell_convolution.go:72-100,112-120,176-192,313-410)
 *                         + Kernel_Arne (src/mumax/modules/kernel_magnetostatic.go:30-181);
 *                         with demag_exchange, module demagexch's kernel chain
 *                         (mod_demagexchange.go:26-205, kernel_exchange.go:102-123)
 *   mm_fields             the H_eff SumUpdater and its parents: MaxwellPlan.UpdateB
 *                         (maxwell_convolution.go:222-309), exch6Updater (mod_exchange6.go:40-51),
 *                         UniaxialAnisUpdater (mod_uniaxialanisotropy.go:44-57), zeeman
 *                         (mod_zeeman.go:23-31, update_sum.go:29-75), TempBrownUpdater
 *                         (mod_temperature.go:71-134)
 *   mm_torque             torqueUpdater (mod_llg.go:59-70) + AddTermUpdater of zzt/stt
 *                         (update_addterm.go:26-40, mod_zhang-li.go:50-70, mod_slonczewski.go:56-99)
 *   mm_solver_init/mm_step/mm_run/mm_steps/mm_run_until_maxtorque
 *                         Solver.Step (src/mumax/engine/solver.go:14-17): solver/rk12
 *                         (solve_rk12.go:91-214), euler (solve_euler.go:22-50), heun
 *                         (solve_heun.go:27-79), am12 (solve_am01.go:46-301);
 *                         Engine.Run/Steps (engine.go:489-524);
 *                         API.Run_Until_Smaller (api.go:122-131).  rk23/rk45 are new.
 *   mm_maxtorque          MaxNormUpdater (update_reduce.go:103-108, reductor.go:173-186)
 *   mm_average            AverageUpdater (update_reduce.go:47-69)
 *   mm_energy             EnergyUpdater/SDotUpdater (mod_energy.go:24-95, update_sdot.go:36-62)
 *   mm_plan_create_batch, mm_batch_*, mm_ensemble_*
 *                         many independent simulations per launch; the reference runs one
 *                         simulation per engine (engine.go:22-40), so a batch replaces nsim
 *                         engines, each with its own Solver.Step, stepped side by side.
 */
#ifndef MM_B200_H
#define MM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define MM_API __declspec(dllexport)
#else
#define MM_API __attribute__((visibility("default")))
#endif

/* status codes (0 = ok, negative = error class) */
enum {
    MM_OK = 0,
    MM_ERR_ARG = -1,           /* invalid argument / unsupported size */
    MM_ERR_CUDA = -2,          /* CUDA runtime error */
    MM_ERR_NOT_CONVERGED = -3, /* more than 10 rejected attempts in one step (solve_rk12.go:205) */
    MM_ERR_NAN = -4,           /* NaN in the state (quant.go:427-432) */
    MM_ERR_STATE = -5,         /* call out of order (no solver, no state, ...) */
    MM_ERR_TIMEOUT = -6,       /* a bounded device wait gave up */
    MM_ERR_RANGE = -7          /* time outside a SetPointwise table (update_pointwise.go:66) */
};

/* demag tensor kinds (mm_problem.demag_tensor) */
enum { MM_TENSOR_ARNE = 0, MM_TENSOR_NEWELL = 1 };

/* solvers */
enum { MM_EULER = 0, MM_HEUN = 1, MM_RK12 = 2, MM_RK23 = 3, MM_RK45 = 4, MM_AM12 = 5 };

/* Problem description.  Multipliers in SI units; masks are DEVICE float arrays of
 * n0*n1*n2 values multiplying the multiplier (NULL = uniform 1), exactly the
 * MASK-quantity convention of the reference (common_func.h:298-301). */
typedef struct mm_problem {
    int n[3];          /* cells, internal order (Z,Y,X) */
    double cell[3];    /* cell size (m), internal order */
    int pbc[3];        /* periodic flags, internal order */
    int demag, exchange, anis, zeeman, thermal, zhangli, slonczewski; /* terms on/off */
    int demag_accuracy;                  /* Kernel_Arne accuracy (6 for module demag) */
    double msat, aex, alpha, gamma;      /* A/m, J/m, -, m/As */
    double bext[3];                      /* T */
    double ku, anisu[3];                 /* J/m^3, unit vector */
    double temp;                         /* K */
    unsigned long long seed;             /* thermal Philox key */
    double j[3];                         /* A/m^2 */
    double zl_pol, xi;                   /* Zhang-Li polarisation, non-adiabaticity */
    double p[3], sl_pol, lambda, eps_prime, t_fl; /* Slonczewski */
    const float *msat_mask, *aex_mask, *alpha_mask, *ku_mask;
    const float *anisu_mask[3], *bext_mask[3], *j_mask[3];
    const float *temp_mask, *xi_mask, *zl_pol_mask;
    const float *p_mask[3];
    const float *sl_pol_mask, *lambda_mask, *eps_prime_mask, *t_fl_mask;
    /* 1: module demagexch (mod_demagexchange.go:26-205): the exchange field is folded into
     * the demag kernel (Ms K_demag + 2Aex/(mu0 Ms) Laplacian, kernel_exchange.go:102-123)
     * and computed by the same convolution of m; the 6-neighbour stencil term is off.
     * Needs demag = 1, a uniform Aex (no aex_mask) and nsim = 1. */
    int demag_exchange;
    /* MM_TENSOR_ARNE (0): Kernel_Arne face-charge integration (kernel_magnetostatic.go:
     * 30-181), the reference's only tensor.  MM_TENSOR_NEWELL (1): the closed forms of
     * Newell, Williams & Dunlop (1993) in FP64 within 8 cell sizes, the cell-averaged
     * dipole tensor by Gauss quadrature beyond.  No counterpart in the reference. */
    int demag_tensor;
} mm_problem;

/* Scalars of one simulation of a batched plan (the multipliers of Msat, Aex, alpha, B_ext,
 * Ku1, anisU, Temp and the thermal seed); everything else comes from the mm_problem. */
typedef struct mm_sim {
    double msat, aex, alpha;             /* A/m, J/m, - */
    double bext[3];                      /* T */
    double ku, anisu[3];                 /* J/m^3, unit vector */
    double temp;                         /* K */
    unsigned long long seed;             /* thermal Philox key */
} mm_sim;

typedef struct mm_stats {
    double t, dt, err, peakerr, maxtorque;
    long long step, badsteps, attempts, evals;
    int status, done;
    long long iterations;  /* solver/am12: fixed-point iterations of the last step */
} mm_stats;

typedef struct mm_plan_s* mm_plan;
typedef struct mm_ensemble_s* mm_ensemble;
typedef struct CUstream_st* mm_stream; /* cudaStream_t; NULL = legacy default stream */

/* Last error message of the calling thread ("" if none). */
MM_API const char* mm_last_error(void);
MM_API const char* mm_version(void);

/* Builds the plan: geometry, demag tensor (FP64 on the GPU), its transform, and all
 * workspaces; nothing is allocated after this call.  Runs on the current device. */
MM_API int mm_plan_create(const mm_problem* prob, mm_plan* out);
MM_API int mm_plan_destroy(mm_plan plan);
/* A plan of nsim independent simulations of one geometry (grid, cell, pbc, terms, demag
 * tensor).  Per-cell arrays (state, fields, torque) hold nsim blocks of 3 x N floats,
 * simulation-major.  sims[nsim] gives each simulation's scalars; NULL takes them all from
 * prob.  Masks in prob hold N values shared by all simulations (masks_per_sim = 0) or
 * nsim x N values (masks_per_sim = 1).  Each simulation has its own time step, accept /
 * reject decisions and stop condition; all run in the same kernel launches.  With demag,
 * nsim > 1 needs 8 <= padded L2 <= 2048.  mm_plan_create(prob) = (prob, 1, NULL, 0). */
MM_API int mm_plan_create_batch(const mm_problem* prob, int nsim, const mm_sim* sims, int masks_per_sim,
                                mm_plan* out);
MM_API int mm_plan_nsim(mm_plan plan);
/* Tile shapes of the FFT passes, picked at plan creation by the autotuner (timed field
 * evaluations; MM_AUTOTUNE=0 in the environment keeps the defaults).  tiles[0]: rows per
 * block of the R2C row pass, tiles[1]: columns per block of the column passes, tiles[2]:
 * rows per block of the C2R + stencil/torque epilogue, each as a shift of the default
 * (-1 = half, 0 = default, +1 = double; tiles[2] in {-1, 0}); tiles[3]: 1 = the fused
 * single-layer evaluation (one launch per evaluation, one block per simulation, the half
 * spectrum in shared memory; films with n0 = 1, N1 <= 64, N2 in 32..128).  eval_us (may
 * be NULL): the timed evaluation with the chosen tiles (0 if not tuned).  Results do not
 * depend on the tiles (energies up to the order of their block partial sums). */
MM_API int mm_plan_tiles(mm_plan plan, int tiles[4], double* eval_us);
MM_API int mm_plan_set_tiles(mm_plan plan, const int tiles[4]);
/* Tuning runs made in this process (the autotuner keeps each plan shape's result per
 * device and reuses it for later plans of that shape; no counterpart in the reference). */
MM_API long long mm_autotune_runs(void);
/* Real-space demag tensor in FP64 on the GPU, the function Kernel_Arne
 * (kernel_magnetostatic.go:30-181) computes on the host: out[6][L0][L1][L2] (device,
 * caller-allocated; components 00 11 22 12 02 01 of the internal axes, K = -N so that
 * H = K * M), for the padded sizes L, cell sizes and periodic flags of a plan; kind
 * MM_TENSOR_ARNE (with `accuracy`, 6 for module demag) or MM_TENSOR_NEWELL.  Entries
 * outside the reference's index ranges (the Nyquist planes) are zero.  Async on stream. */
MM_API int mm_demag_tensor(const int L[3], const double cell[3], const int pbc[3], int kind, int accuracy,
                           double* out, mm_stream stream);

/* The plan's transformed demag tensor, one octant: out[6][kd0][kd1][kd2] (host, may be
 * NULL to query kd), components xx yy zz yz xz xy in internal axis order, scaled by
 * 1/(L0 L1 L2) like the reference's fftKern (maxwell_convolution.go:576-612); the other
 * octants follow by symmetry (even along every axis for the diagonal, odd along s and d
 * for K_sd).  For demagexch plans this is the demag part alone. */
MM_API int mm_plan_demag_kernel(mm_plan plan, float* out, int kd[3]);
/* Replaces the per-simulation scalars of a batched plan. */
MM_API int mm_batch_set_sims(mm_plan plan, const mm_sim* sims);
/* Replaces multipliers/masks/terms of an existing plan (same grid, cell, pbc). */
MM_API int mm_plan_set_problem(mm_plan plan, const mm_problem* prob);
/* Non-zero demag tensor components (xx yy zz yz xz xy, internal order). */
MM_API int mm_plan_kernel_nonzero(mm_plan plan, int out6[6]);
/* Bytes of device memory held by the plan. */
MM_API long long mm_plan_device_bytes(mm_plan plan);

/* Per-term fields at m (which is used as given, not normalised).  Any output may be
 * NULL.  noise_step selects the thermal noise sample, dt_thermal its dt. */
MM_API int mm_fields(mm_plan plan, const float* m, long long noise_step, double dt_thermal,
                     float* h_demag, float* h_ex, float* h_anis, float* h_zee, float* h_therm,
                     float* h_eff, mm_stream stream);
/* Torque array tau/gamma (+ spin-transfer terms / gamma) at normalise(m); m is
 * normalised in place first, as pulling "m" does in the reference. */
MM_API int mm_torque(mm_plan plan, float* m, long long noise_step, double dt_thermal,
                     float* torque, mm_stream stream);

/* ---- time stepping: the plan owns the state; all control runs on the device ---- */
MM_API int mm_solver_init(mm_plan plan, int solver, double dt, double mindt, double maxdt,
                          double maxerr);
/* solver/am12 error tolerances m_maxAbsError, m_maxRelError (defaults 1e-4, 1e-3). */
MM_API int mm_solver_am12_tolerances(mm_plan plan, double abs_err, double rel_err);
MM_API int mm_set_state(mm_plan plan, const float* m, int from_host, mm_stream stream);
MM_API int mm_get_state(mm_plan plan, float* m, int to_host, mm_stream stream);
MM_API int mm_set_time(mm_plan plan, double t, double dt);
MM_API int mm_set_thermal_dt(mm_plan plan, double dt_thermal);
/* One accepted step (retries included). */
MM_API int mm_step(mm_plan plan, mm_stream stream);
/* Steps until t >= t_start + duration (Engine.Run). */
MM_API int mm_run(mm_plan plan, double duration, mm_stream stream);
/* Exactly n accepted steps (Engine.Steps). */
MM_API int mm_steps(mm_plan plan, long long n, mm_stream stream);
/* Steps until maxtorque = gamma*max|tau| < thr (run_until_smaller("maxtorque", thr)). */
MM_API int mm_run_until_maxtorque(mm_plan plan, double thr, long long max_steps, mm_stream stream);
/* Queue `attempts` step attempts with no host synchronisation (CUDA-graph replay). */
MM_API int mm_queue_attempts(mm_plan plan, int attempts, mm_stream stream);
MM_API int mm_get_stats(mm_plan plan, mm_stats* out, mm_stream stream);

/* ---- reductions of the current state ---- */
MM_API int mm_maxtorque(mm_plan plan, double* out, mm_stream stream);
MM_API int mm_average(mm_plan plan, double out[3], mm_stream stream);
/* E_zeeman, E_ex, E_demag, E_anis, E (J) -- compensated FP32 sums. */
MM_API int mm_energy(mm_plan plan, double out[5], mm_stream stream);

/* <m> without any device allocation, for callers that cannot allocate device memory
 * (code inside a CUDA stream capture, engines whose device memory belongs to another
 * allocator, host code that must not block on the allocator).  No counterpart in the
 * reference.  m: device SoA float32 3 x ncell; out: device, 3 doubles (sum m_c / ncell).
 * ncell is limited to 16,777,216 (MM_ERR_ARG beyond): the block partials live in a fixed
 * 192 KB file-scope device array held by every GPU that loads the library.  The first
 * call on a device looks up that array's address and should precede any stream capture;
 * calls share the array, so calls that overlap on the GPU race. */
MM_API int mm_average_noalloc(const float* m, long long ncell, double* out, mm_stream stream);

/* run_until_maxtorque with one threshold per simulation (thr[nsim]); each simulation
 * stops, and stays frozen, once its own maxtorque falls below its threshold. */
MM_API int mm_batch_run_until_maxtorque(mm_plan plan, const double* thr, long long max_steps, mm_stream stream);

/* ---- time-dependent inputs: SetPointwise (api.go:172-190, update_pointwise.go:30-88) ----
 * A table of npoints rows (t, v0, v1, v2), internal component order, times
 * non-decreasing, makes B_ext (MM_TABLE_BEXT, T) or j (MM_TABLE_J, A/m^2) a piecewise
 * linear function of time that the kernels evaluate on the device at every stage time
 * (t + c dt), replacing the multiplier.  As in the reference the value is 0 at or before
 * the first time and a time past the last row is an error (MM_ERR_RANGE).  npoints = 0
 * removes the table; otherwise npoints >= 2.  Standalone evaluations (mm_fields,
 * mm_torque, reductions) use simulation 0's time. */
enum { MM_TABLE_BEXT = 0, MM_TABLE_J = 1 };
MM_API int mm_set_table(mm_plan plan, int quantity, int npoints, const double* rows);

/* ---- autotabulate on the device (AutoTabulate, notify_tabulate.go:23-28) ----
 * After every accepted step with t - count*period >= period, the step's own launches
 * append a row (t, <m>_0, <m>_1, <m>_2 (internal order), maxtorque, dt, step, 0) to the
 * simulation's device table: no host synchronisation.  capacity rows per simulation;
 * period <= 0 turns it off.  mm_tabulate_read copies all tables to out
 * [nsim][capacity][8] (host), the rows written per simulation to counts[nsim] and the
 * rows that found the table full to lost[nsim] (may be NULL), and empties the tables.
 * maxtorque is that of the new state for RK23/RK45 and of the previous state otherwise. */
MM_API int mm_tabulate(mm_plan plan, double period, int capacity);
MM_API int mm_tabulate_read(mm_plan plan, double* out, int* counts, long long* lost, mm_stream stream);

/* ---- autosave of m on the device (AutoSave, notify_autosave.go:25-31) ----
 * After every accepted step with (t - t_on) - count*period >= period, the step's own
 * launches copy the new state into the next of `capacity` device slots per simulation
 * (no host synchronisation); t_on is the time of this call.  mm_autosave_read copies the
 * held states to states [nsim][capacity][3N] and their times to times [nsim][capacity]
 * (host), the count per simulation to counts, the states that found the slots full to
 * lost (may be NULL), and frees the slots.  period <= 0 turns it off. */
MM_API int mm_autosave(mm_plan plan, double period, int capacity);
MM_API int mm_autosave_read(mm_plan plan, float* states, double* times, int* counts, long long* lost,
                            mm_stream stream);

/* ---- continuous batching (relaxation pools) ----
 * mm_batch_restart puts new problems into `count` slots idx[] of a batched plan: state
 * m[count][3N] (host if from_host, else device), scalars sims[count] (NULL: keep the
 * slot's), torque thresholds thr[count]; the slots restart at t = 0 with the solver's
 * initial dt while the other slots keep their state; a slot stops after max_steps steps
 * (0: no limit) whether or not it reached its threshold.  Per-simulation masks are the
 * caller's device arrays: write the new slot's values before this call.
 * mm_batch_drive steps until at most target_active simulations are still running. */
MM_API int mm_batch_restart(mm_plan plan, int count, const int* idx, const float* m, int from_host,
                            const mm_sim* sims, const double* thr, long long max_steps, mm_stream stream);
/* Stops the simulations in slots idx[count]: they count as done (state and statistics
 * kept) until mm_batch_restart reuses the slot. */
MM_API int mm_batch_cancel(mm_plan plan, int count, const int* idx, mm_stream stream);
MM_API int mm_batch_drive(mm_plan plan, int target_active, long long max_attempts, mm_stream stream);

/* ---- per-simulation results of a (batched) plan; out arrays have nsim entries ---- */
MM_API int mm_batch_stats(mm_plan plan, mm_stats* out, mm_stream stream);
MM_API int mm_batch_maxtorque(mm_plan plan, double* out, mm_stream stream);
MM_API int mm_batch_average(mm_plan plan, double* out3, mm_stream stream);   /* nsim x 3 */
MM_API int mm_batch_energy(mm_plan plan, double* out5, mm_stream stream);    /* nsim x 5 */

/* ---- ensembles: several plans (e.g. one batched plan per grid size) stepped together,
 * each on its own branch of one CUDA graph that replays `attempts_per_launch` attempts of
 * every plan.  The plans stay owned by the caller and must outlive the ensemble. ---- */
MM_API int mm_ensemble_create(const mm_plan* plans, int nplans, int attempts_per_launch, mm_ensemble* out);
MM_API int mm_ensemble_destroy(mm_ensemble ens);
/* Every simulation of every plan takes n accepted steps. */
MM_API int mm_ensemble_steps(mm_ensemble ens, long long n, mm_stream stream);
/* Every simulation advances by `duration` seconds. */
MM_API int mm_ensemble_run(mm_ensemble ens, double duration, mm_stream stream);
MM_API long long mm_ensemble_launch_count(mm_ensemble ens);

/* ---- output and input formats (host side; ovf/, dump/ and engine/format_dump.go) ----
 * data: host float32 [ncomp][n0][n1][n2] in internal order (ncomp 1 or 3), n and cell
 * internal.  OVF 2.0 (ovf2_output.go:34-161) and OMF 1.0 (omf_output.go:34-206) write
 * one file; a dump frame (dump/writer.go:34-97, format_dump.go:40-62, CRC-64 ISO) is
 * appended to the file.  mm_read_field reads the first field of any of them (data NULL:
 * sizes only), checking the OMF control number and the dump CRC. */
enum { MM_FMT_OVF2_BIN4 = 0, MM_FMT_OVF2_TEXT = 1, MM_FMT_OMF_BIN4 = 2, MM_FMT_OMF_TEXT = 3, MM_FMT_DUMP = 4 };
MM_API int mm_write_field(const char* path, int format, const float* data, int ncomp, const int n[3],
                          const double cell[3], double time, const char* name, const char* unit);
MM_API int mm_read_field(const char* path, float* data, long long capacity, int* ncomp, int n[3], double* time);
/* CRC-64 with the ISO polynomial as Go's hash/crc64 computes it (the dump checksum). */
MM_API uint64_t mm_crc64_iso(const void* data, size_t n);
/* Snapshot of the plan's state without stopping the GPU: copies m to pinned host memory on
 * a side stream once the work queued on `stream` is done (later work on `stream` waits only
 * for that copy), then formats and writes the file on a host thread.  mm_save_wait blocks
 * until every pending snapshot of the plan is on disk and returns the first error. */
MM_API int mm_save_async(mm_plan plan, const char* path, int format, mm_stream stream);
MM_API int mm_save_wait(mm_plan plan);

/* ---- learned warm start: BF16 U-Net kernels (no counterpart in the reference) ----
 * NHWC bf16 tensors addressed as channel views (pixel stride cs, channel offset co);
 * FP32 accumulation; pointers are device pointers.  conv3x3: out = act(bias + W * in),
 * W [Cout][9][Cin] bf16, Cin % 16 == 0 (relu 0/1, bias may be NULL).  wgrad: dW[Cout][9][Cin]
 * += sum over pixels (FP32, atomics).  pool: 2x2 average (backward adds into the input
 * gradient); upsample: nearest 2x (backward sums); relu_bwd zeroes d where out <= 0;
 * mse: masked mean-square error of the first three channels against a float target
 * [P][3] (loss accumulated, gradient written); adam: one Adam step on FP32 master
 * weights with a bf16 copy; flip: the transposed, tap-reversed weights of the data
 * gradient. */
MM_API int mm_nn_conv3x3(const void* in, int in_cs, int in_co, int Cin, const void* W, const float* bias, void* out,
                         int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu, mm_stream st);
/* Iteration limit of the mbarrier waits in the tcgen05 kernels (default 2^26; a
 * negative value restores it).  A wait that runs out sets the kernel's error flag and the
 * block returns after its MMAs in flight are done; a limit of 0 makes every such wait run
 * out at once, which tests use to check that the time-out is reported. */
MM_API int mm_nn_set_wait_limit(long long iterations);
/* tcgen05 weight gradient: dW[Cout][9][Cin] (FP32, accumulated: zero it first) of the 3x3
 * convolution from dY [B*H*W][dy_cs] (channels dy_co..+Cout) and X [B*H*W][x_cs]
 * (channels x_co..+Cin); channel counts, strides and offsets multiples of 8, W <= 256;
 * *err set if an mbarrier wait runs out. */
MM_API int mm_nn_conv3x3_wgrad_tc(const void* dy, int dy_cs, int dy_co, int Cout, const void* x, int x_cs, int x_co,
                                  int Cin, float* dW, int B, int H, int W, int* err, mm_stream st);
/* Kernel behind mm_nn_conv3x3_tc: 0 = one 128-position tile per block (default),
 * 1 = persistent warp-specialised (loader warps, one MMA thread, epilogue warps, two TMEM
 * accumulators).  Same results.  No counterpart in the reference. */
MM_API int mm_nn_set_conv_kernel(int persistent);
/* conv3x3 on the 5th-generation tensor cores (tcgen05.mma, TMEM accumulators); *err
 * (device int) is set if a bounded wait inside the kernel ran out. */
MM_API int mm_nn_conv3x3_tc(const void* in, int in_cs, int in_co, int Cin, const void* W, const float* bias, void* out,
                            int out_cs, int out_co, int Cout, int B, int H, int Wd, int relu, int* err, mm_stream st);
MM_API int mm_nn_conv3x3_wgrad(const void* dy, int dy_cs, int dy_co, int Cout, const void* x, int x_cs, int x_co,
                               int Cin, float* dW, int B, int H, int Wd, mm_stream st);
MM_API int mm_nn_pool(const void* in, int in_cs, int in_co, void* out, int out_cs, int out_co, int C, int B, int Ho,
                      int Wo, int backward, mm_stream st);
MM_API int mm_nn_upsample(const void* in, int in_cs, int in_co, void* out, int out_cs, int out_co, int C, int B,
                          int Hi, int Wi, int backward, mm_stream st);
MM_API int mm_nn_relu_bwd(const void* out, int o_cs, int o_co, void* d, int d_cs, int d_co, int C, long long P,
                          mm_stream st);
/* ReLU backward (relu != 0: d = 0 where out <= 0, in place) and bias gradient
 * db[c] += sum_p d[p][c] in one pass over P pixels of C <= 512 channels (channel counts,
 * strides and offsets multiples of 8). */
MM_API int mm_nn_relu_bias_bwd(const void* out, int o_cs, int o_co, void* d, int d_cs, int d_co, int C, long long P,
                               int relu, float* db, mm_stream st);
MM_API int mm_nn_bias_grad(const void* d, int d_cs, int d_co, int C, long long P, float* db, mm_stream st);
MM_API int mm_nn_mse(const void* out, int o_cs, const float* target, const float* mask, long long P, float norm,
                     void* dout, int d_cs, float* loss, mm_stream st);
MM_API int mm_nn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                      float eps, int t, void* wb, mm_stream st);
MM_API int mm_nn_flip(const void* W, int Cout, int Cin, void* Wt, int Cin_t, int Cout_t, mm_stream st);
/* warm-start input features [nq][P][16] bf16 from masks [nq][P] and prm [nq][8] =
 * (Ms, Aex, Ku1, axis x, axis y, B_x, B_y, 0) in user axes (see unet.py). */
MM_API int mm_nn_features(const float* masks, const float* prm, long long nq, int P, void* out, mm_stream st);
/* initial states [nq][3][P] (internal SoA: m_z, m_y, m_x) = mask * normalised first three
 * output channels (m_x, m_y, m_z) of the network output [nq][P][out_cs]. */
MM_API int mm_nn_output_state(const void* out, int out_cs, const float* masks, long long nq, int P, float* state,
                              mm_stream st);
MM_API int mm_nn_to_bf16(const float* in, long long P, int C, void* out, int o_cs, int o_co, mm_stream st);

/* ---- instrumentation ---- */
/* Kernels this plan has enqueued so far (graph replays counted per kernel node). */
MM_API long long mm_plan_launch_count(mm_plan plan);
/* Average duration (ms) of each pass of one field evaluation, timed with CUDA events
 * on `stream` around each pass; *npass = 5 (3-D), 3 (2-D film) or 1 (no demag). */
MM_API int mm_profile_eval(mm_plan plan, int reps, double* ms_out, int* npass, mm_stream stream);
/* L0 L1 L2, M, h, hp, kd0 kd1 kd2, number of non-zero kernel components, demag flag, 0 */
MM_API int mm_plan_geometry(mm_plan plan, int out12[12]);

#ifdef __cplusplus
}
#endif
#endif /* MM_B200_H */
