#!/usr/bin/env python
"""Benchmark of the micromagnetic hot path (one JSON line on rank 0).

Workload (default): 3-D film with perpendicular anisotropy, 256x256x16 cells of
4x4x2 nm, Ms 1.1e6 A/m, Aex 1.5e-11 J/m, Ku1 5e5 J/m^3 along z, alpha 0.1, m seeded
i.i.d. uniform on the sphere, no applied field, demag + exchange + anisotropy,
adaptive RK23 (max error 1e-5).  A "step" is one accepted solver step (its rejected
attempts included).  Metric: cell-steps/s = cells x accepted steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (torchrun, one process per GPU): independent replicas, one simulation per GPU
with its own seed (weak scaling); no collective in the step.  The reference arm times
the FP64 CPU oracle (a restatement of the reference's discretisation; the reference
itself has no CPU implementation of this path) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "2_b200"))

MU0 = 4e-7 * np.pi

WORKLOAD = dict(
    name="film3d_256x256x16_perp_anis_rk23",
    n=(16, 256, 256),                 # internal (z, y, x)
    cell=(2e-9, 4e-9, 4e-9),
    demag=1, exchange=1, anis=1, zeeman=0,
    msat=1.1e6, aex=1.5e-11, ku=5e5, anisu=(1.0, 0.0, 0.0), alpha=0.1, gamma=2.211e5,
    solver="rk23", maxerr=1e-5, dt0=1e-15,
)


def problem():
    w = WORKLOAD
    return dict(n=w["n"], cell=w["cell"], demag=w["demag"], exchange=w["exchange"], anis=w["anis"],
                zeeman=w["zeeman"], msat=w["msat"], aex=w["aex"], ku=w["ku"], anisu=w["anisu"],
                alpha=w["alpha"], gamma=w["gamma"])


def initial_m(seed):
    n = WORKLOAD["n"]
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(3, N))
    v /= np.linalg.norm(v, axis=0, keepdims=True)
    return v.astype(np.float32).ravel()


# ---------------------------------------------------------------- byte model
def pass_bytes(geo, n, masks=0):
    """Algorithmic HBM bytes of each pass of one standalone field evaluation
    (k written, no stage combine) in this design: only the non-zero half of the
    padded data is stored, the kernel is one octant of nk FP32 components."""
    N0, N1, N2 = n
    N = N0 * N1 * N2
    L0, L1, L2 = geo["L"]
    h = geo["h"]
    oct_ = geo["kd"][0] * geo["kd"][1] * geo["kd"][2]
    kb = 4 * geo["nk"] * oct_
    a = 24 * N0 * N1 * h
    b = 24 * N0 * L1 * h
    if L0 == 1:
        return [("xfwd", 12 * N + 4 * N * masks + a), ("ymul", a + kb + a), ("xinv_epi", a + 12 * N + 12 * N)]
    return [("xfwd", 12 * N + 4 * N * masks + a), ("yfwd", a + b), ("zmul", b + kb + b), ("yinv", b + a),
            ("xinv_epi", a + 12 * N + 12 * N)]


def step_bytes_rk23(geo, n):
    """Algorithmic bytes of one RK23 attempt: start combine + 3 fused evaluations."""
    N = n[0] * n[1] * n[2]
    conv = sum(b for _, b in pass_bytes(geo, n)) - 24 * N   # passes without the epilogue's m read / k write
    ev = conv + 12 * N + 12 * N                               # + read m, write k
    combine0 = 36 * N                                         # Y, K1 -> M1
    e1 = ev + 12 * N + 12 * N                                 # + read Y, write M2
    e2 = ev + 12 * N * 3 + 12 * N                             # + read Y, K1, K2, write Y'
    e3 = ev + 12 * N * 3                                      # + error: read K1, K2, K3
    return combine0 + e1 + e2 + e3


def survey_step_bytes(n, L, evals, extra_per_cell):
    """The fixed minimal-pass byte model of the hot-path specification, per accepted step:
    B_eval = 36N + a + (a+b) + (b + 24 Pc + b) + (b+a) + a for 3-D grids (a = 24 N0 N1 h,
    b = 24 N0 L1 h, Pc = L0 L1 h, h = L2/2+1; full FP32 kernel spectrum), then
    B_step = evals * B_eval + extra_per_cell * N (RK23: 3 evaluations, 132 B/cell for the
    stage combines and the error estimate).  1,397 B per cell-step for the 256x256x16
    film.  It does not depend on how this implementation fuses its passes."""
    N0, N1, N2 = n
    N = N0 * N1 * N2
    L0, L1, L2 = L
    h = L2 // 2 + 1
    a = 24 * N0 * N1 * h
    b = 24 * N0 * L1 * h
    pc = L0 * L1 * h
    if L0 == 1:
        ev = 36 * N + a + (a + 16 * L1 * h + a) + a
    else:
        ev = 36 * N + a + (a + b) + (b + 24 * pc + b) + (b + a) + a
    return evals * ev + extra_per_cell * N


def read_traffic():
    """Per-pass DRAM bytes of one launch (ncu dram__bytes_read.sum + dram__bytes_write.sum),
    from the committed capture summary of this workload, if there is one."""
    path = os.path.join(ROOT, "profiles", "traffic_film3d_256x256x16.txt")
    out = {}
    if os.path.exists(path):
        for ln in open(path):
            f = ln.split("#")[0].split()
            if len(f) == 2:
                out[f[0]] = int(f[1])
    return out


def step_bytes_heun(geo, n):
    """Algorithmic bytes of one Heun step: two fused evaluations; the first also writes the
    predictor, the second reads the saved k0 and writes the corrected state."""
    N = n[0] * n[1] * n[2]
    conv = sum(b for _, b in pass_bytes(geo, n)) - 36 * N   # passes without reading m / writing k
    return 2 * conv + 2 * (12 * N + 12 * N + 12 * N + 12 * N)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU baseline (oracle)
def reference_gpu_baseline(device, ref_steps=10, our_steps=50):
    """The reference's own CUDA kernels on this GPU (oracle/ref_gpu.py: libmumax2 built
    from the reference's sources, driven by a restatement of its Go RK12 loop, cuFFT for
    the transforms) against this repository's fused path with the same solver (RK12,
    the reference's adaptive solver; it has no RK23), configuration and initial state.
    CUDA-event timing of whole steps after 3 warm-up steps; the reference path's host
    syncs are part of its step, as in the reference."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu as R
    from mumax2 import Plan
    if not R.available():
        return {"unavailable": "reference library not built (oracle/build_ref.sh)"}
    w = WORKLOAD
    n = w["n"]
    N = n[0] * n[1] * n[2]
    plan = Plan(problem(), device=device)
    ref = R.RefPath(n, w["cell"], w["msat"], w["aex"], w["alpha"], w["gamma"], w["ku"], w["anisu"],
                    plan.demag_kernel(), dt=w["dt0"], maxerr=w["maxerr"])
    m0 = initial_m(0)
    ref.set_state(m0)
    for _ in range(3):
        ref.step()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s0, e0 = ref.step_count, ref.evals
    a.record()
    for _ in range(ref_steps):
        ref.step()
    b.record()
    torch.cuda.synchronize()
    ref_ms = a.elapsed_time(b)
    ref_evals = (ref.evals - e0) / (ref.step_count - s0)
    del ref
    plan.solver("rk12", dt=w["dt0"], maxerr=w["maxerr"])
    plan.set_state(m0)
    plan.steps(3)
    torch.cuda.synchronize()
    st0 = plan.stats()
    a.record()
    plan.steps(our_steps)
    b.record()
    torch.cuda.synchronize()
    our_ms = a.elapsed_time(b)
    st1 = plan.stats()
    plan.close()
    ref_v = N * ref_steps / (ref_ms * 1e-3)
    our_v = N * our_steps / (our_ms * 1e-3)
    return {"value": ref_v, "unit": "cell-steps/s", "kind": "reference libmumax2 kernels + cuFFT on this GPU",
            "solver": "rk12", "steps": ref_steps, "ms_per_step": ref_ms / ref_steps,
            "evals_per_step": ref_evals,
            "ours_rk12": {"value": our_v, "ms_per_step": our_ms / our_steps, "steps": our_steps,
                          "evals_per_step": (st1["evals"] - st0["evals"]) / our_steps},
            "ours_over_reference": our_v / ref_v}


def cufft_comparator(L, our_eval_ms, reps=20):
    """cuFFT (through torch.fft) as a timing comparator only: the 3-D R2C and C2R of the
    three magnetisation components on the zero-padded volume L, the transforms the
    reference's FFTPlanX runs per field evaluation, against this repository's five passes
    of one evaluation (transforms, kernel multiply and the whole field/torque epilogue).
    CUDA events, 3 warm-up repetitions."""
    import torch
    x = torch.randn(3, *L, device="cuda")
    spec = torch.fft.rfftn(x, dim=(1, 2, 3))
    y = torch.empty_like(x)
    for _ in range(3):
        torch.fft.rfftn(x, dim=(1, 2, 3), out=spec)
        torch.fft.irfftn(spec, s=L, dim=(1, 2, 3), out=y)
    a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize()
    fwd = inv = 0.0
    for _ in range(reps):
        a.record()
        torch.fft.rfftn(x, dim=(1, 2, 3), out=spec)
        b.record()
        torch.fft.irfftn(spec, s=L, dim=(1, 2, 3), out=y)
        c.record()
        torch.cuda.synchronize()
        fwd += a.elapsed_time(b)
        inv += b.elapsed_time(c)
    fwd, inv = fwd / reps, inv / reps
    return {"cufft_r2c_ms": fwd, "cufft_c2r_ms": inv, "cufft_transforms_ms": fwd + inv,
            "ours_eval_ms": our_eval_ms, "cufft_transforms_over_ours_eval": (fwd + inv) / our_eval_ms,
            "padded": list(L), "components": 3}


def cpu_baseline(max_seconds=25.0):
    """FP64 oracle on the host cores: RK23 steps of the same workload (bounded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    w = WORKLOAD
    o = O.Oracle(O.full_desc(**problem()))
    r = O.OracleRun(o, initial_m(0).astype(np.float64), solver=w["solver"], dt=w["dt0"], maxerr=w["maxerr"])
    r.step()   # FSAL start-up evaluation excluded from the sample
    t0 = time.perf_counter()
    steps = 0
    while True:
        r.step()
        steps += 1
        if time.perf_counter() - t0 > max_seconds or steps >= 8:
            break
    dt = time.perf_counter() - t0
    N = w["n"][0] * w["n"][1] * w["n"][2]
    return {"value": N * steps / dt, "unit": "cell-steps/s", "cores": int(O.lib().or_num_threads()),
            "kind": "port", "sample": f"{steps} RK23 steps of the full 256x256x16 workload after one warm-up "
                                      f"step, FP64 oracle with OpenMP ({dt:.1f} s)", "seconds": dt}


def film_config(world):
    """The config object of the film workload, identical in both arms."""
    w = WORKLOAD
    n = w["n"]
    return {"workload": w["name"], "cells": n[0] * n[1] * n[2], "grid_xyz": [n[2], n[1], n[0]],
            "cell_nm": [4, 4, 2], "solver": w["solver"], "maxerr": w["maxerr"], "parallelism": f"replicas{world}",
            "l2": "per-step working set (state, stages, half spectrum, kernel) ~250 MB > 126 MB L2"}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    cb = cpu_baseline(max_seconds=min(120.0, 15.0 * max(1, args.steps)))
    line = {"impl": "reference", "metric": "cell-steps/s", "value": cb["value"], "unit": "cell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": film_config(world),
            "cpu_baseline": {k: cb[k] for k in ["value", "unit", "cores", "kind", "sample"]},
            "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def e2e_pipelined(plan, host_in, device, steps=20, jobs=2):
    """End-to-end rate of independent jobs through the C-ABI with host buffers: each job
    uploads its input state from pinned host memory (mm_set_state from the host), takes
    one step (mm_step) and downloads the resulting state (mm_get_state to the host).
    `jobs` plans of the same workload (`plan` and jobs-1 more) run the jobs from their own
    host threads and streams, so that the copies of one job overlap the steps of the
    others (the two copy directions and the kernels use separate engines).  Device time
    from the first to the last event on the streams."""
    import ctypes as C
    import torch
    from mumax2 import Plan
    from mumax2 import _native as nat
    w = WORKLOAD
    L = nat.lib()
    plans = [plan]
    for _ in range(jobs - 1):
        q = Plan(problem(), device=device)
        q.solver(w["solver"], dt=w["dt0"], maxerr=w["maxerr"])
        plans.append(q)
    streams = [torch.cuda.Stream() for _ in plans]
    outs = [torch.empty_like(host_in).pin_memory() for _ in plans]

    def job(k, n):
        h, st = plans[k].h, C.c_void_p(streams[k].cuda_stream)
        for _ in range(n):
            nat.check(L.mm_set_state(h, C.c_void_p(host_in.data_ptr()), 1, st))
            nat.check(L.mm_step(h, st))
            nat.check(L.mm_get_state(h, C.c_void_p(outs[k].data_ptr()), 1, st))

    for k in range(jobs):   # warm-up: graph capture of each plan on its stream
        job(k, 2)
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(jobs)]
    for k in range(jobs):
        ev[k][0].record(streams[k])
    per = steps // jobs
    th = [threading.Thread(target=job, args=(k, per)) for k in range(jobs)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for k in range(jobs):
        ev[k][1].record(streams[k])
    torch.cuda.synchronize()
    t0 = min(range(jobs), key=lambda k: ev[0][0].elapsed_time(ev[k][0]))   # the earliest start
    ms = max(ev[t0][0].elapsed_time(ev[k][1]) for k in range(jobs))
    for q in plans[1:]:
        q.close()
    return {"ms": ms, "steps": jobs * per, "jobs": jobs}


# ---------------------------------------------------------------- replicas
def aggregate(ms_local, cells, steps, world, dist=None, device=None):
    """Whole-job throughput of `world` independent replicas: the slowest rank's device
    time (max over ranks) bounds the job; every rank advanced `cells` by `steps`."""
    ms = ms_local
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([ms_local], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, cells * steps * world / (ms / 1e3)


def replica_seed(rank):
    """Each replica integrates its own random initial state."""
    return 1000 + rank


# ---------------------------------------------------------------- ensemble workload
def ensemble_bench(args, rank, world, local_rank, dist, emit=True):
    """2048 independent thermal simulations of five grid sizes, one batched plan per size,
    all stepped from one CUDA graph (stochastic Heun, fixed 50 fs).  A step advances every
    simulation by one Heun step; value = total cells x steps / device time.  Beside it:
    the same simulations run one at a time (a sample of one per grid size) and their <m>
    against the batched run.  With N > 1 ranks the 2048 simulations are split into
    contiguous cell-balanced blocks, one per rank (strong scaling, no collective while
    stepping), and the per-simulation <m> are gathered to rank 0 at the end."""
    import ctypes as C
    import torch
    from mumax2 import Ensemble, Plan
    from mumax2 import _native as nat
    from mumax2 import workloads as W
    if world > 1:
        # the same ensemble on every rank, a contiguous cell-balanced block of it per rank
        classes, shard = W.ensemble_shard(args.nsim, seed=0, rank=rank, world=world)
    else:
        classes, shard = W.ensemble(nsim=args.nsim, seed=0), (0, args.nsim)
    plans, states = [], []
    for c in classes:
        p = Plan(c["problem"], sims=c["sims"], device=local_rank)
        p.solver("heun", dt=W.ENSEMBLE_DT)
        m0 = W.uniform_state(c["n"], c["m0"], len(c["sims"]))
        p.set_state(m0)
        plans.append(p)
        states.append(m0)
    ens = Ensemble(plans, attempts=args.ens_attempts)
    cells = W.cells_of(classes)
    ens.steps(args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = ens.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.steps(args.steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = ens.launch_count() - l0
    ms_max, value = aggregate(ms, cells, args.steps, world, dist, "cuda")
    total_cells = cells
    if dist is not None and world > 1:
        # sharded: the ranks' cells add up to the ensemble's (not world x cells)
        import torch
        t = torch.tensor([float(cells)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        total_cells = int(t.item())
        value = total_cells * args.steps / (ms_max / 1e3)
    step_b = 0
    for c, p in zip(classes, plans):
        step_b += step_bytes_heun(p.geometry(), c["n"]) * len(c["sims"])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = (float(json.load(open(peaks_path))["hbm_gbs"]), "measured") if os.path.exists(peaks_path) \
        else (6650.0, "fallback")
    achieved = step_b * args.steps / (ms / 1e3) / 1e9

    # end to end: states from pinned host memory, the steps, states back to the host
    L = nat.lib()
    hin = [torch.from_numpy(s).pin_memory() for s in states]
    hout = [torch.empty_like(h).pin_memory() for h in hin]
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for p, h in zip(plans, hin):
        nat.check(L.mm_set_state(p.h, C.c_void_p(h.data_ptr()), 1, None))
    ens.steps(args.steps)
    for p, h in zip(plans, hout):
        nat.check(L.mm_get_state(p.h, C.c_void_p(h.data_ptr()), 1, None))
    f1.record()
    torch.cuda.synchronize()
    e2e_ms, e2e_value = aggregate(f0.elapsed_time(f1), cells, args.steps, world, dist, "cuda")
    io_bytes = sum(h.numel() * 4 for h in hin)

    # unbatched comparison: the first simulation of each grid size alone, same inputs
    # and steps (warm-up + timed + end-to-end run), then its <m> against the batch
    avg_b = [p.batch_average() for p in plans]
    gathered = None
    if dist is not None and world > 1:   # per-simulation <m> of every rank to rank 0
        g = W.gather_per_sim(dist, np.concatenate([c["ids"] for c in classes]), np.concatenate(avg_b), args.nsim)
        gathered = None if g is None else int(np.isfinite(g).all(axis=1).sum())
    uni_cells_steps, uni_ms, dm = 0, 0.0, 0.0
    for c, p, m0, ab in zip(classes, plans, states, avg_b):
        q = dict(c["problem"])
        q.update(c["sims"][0])
        s = Plan(q, device=local_rank)
        s.solver("heun", dt=W.ENSEMBLE_DT)
        N = int(np.prod(c["n"]))
        s.set_state(m0[:3 * N])
        s.steps(args.warmup + args.steps)
        s.set_state(m0[:3 * N])
        torch.cuda.synchronize()
        u0 = torch.cuda.Event(enable_timing=True)
        u1 = torch.cuda.Event(enable_timing=True)
        u0.record()
        s.steps(args.steps)
        u1.record()
        torch.cuda.synchronize()
        uni_ms += u0.elapsed_time(u1)
        uni_cells_steps += N * args.steps
        dm = max(dm, float(np.abs(s.average() - ab[0]).max()))
        s.close()
    unbatched = uni_cells_steps / (uni_ms / 1e3)
    if rank == 0:
        line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"thermal_ensemble_{args.nsim}", "simulations": args.nsim,
                           "cells": total_cells, "shard_of_rank0": list(shard),
                           "grids_xyz": [list(g) for g in W.ENSEMBLE_GRIDS_USER],
                           "sims_per_grid": [len(c["sims"]) for c in classes], "cell_nm": [4, 4, 3],
                           "solver": "heun", "dt_fs": 50, "temperature_K": W.ENSEMBLE_TEMP,
                           "attempts_per_graph_launch": args.ens_attempts, "parallelism": f"replicas{world}",
                           "l2": f"working set ~{sum(p.device_bytes() for p in plans) / 1e9:.1f} GB > 126 MB L2"},
                "roofline": {"bound": "hbm", "kernel": "whole Heun step (all passes of all simulations)",
                             "achieved": achieved, "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_step": step_b},
                "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": io_bytes / args.steps,
                        "d2h_bytes_per_step": io_bytes / args.steps, "steps": args.steps},
                "unbatched": {"value": unbatched, "unit": "cell-steps/s",
                              "sample": f"first simulation of each of the {len(classes)} grid sizes, one plan each, "
                                        f"{args.steps} steps", "batched_over_unbatched": value / unbatched,
                              "max_abs_avg_m_diff": dm},
                "gpu_launches": launches, "clocks": clocks}
        if world > 1:
            line["scaling"] = "strong"
            line["per_sim_avg_m_gathered"] = gathered
        if emit:
            print(json.dumps(line), flush=True)
    ens.close()
    for p in plans:
        p.close()
    return line if rank == 0 else None


# ---------------------------------------------------------------- relaxation workload
def relax_bench(args, rank, world, local_rank, dist):
    """Batched plain relaxations: 64x64x1 films with seeded geometry masks and parameters,
    from the cold start (uniform along +x), RK23 with alpha = 1 until each simulation's
    maxtorque / (gamma Ms) < 1e-4.  Two schedules over one plan of --relax-batch slots:
    synchronous batches (a batch waits for its slowest member) and continuous batching
    (a finished slot takes the next problem at once).  value = relaxations / device time
    of the continuous schedule."""
    import torch
    from mumax2 import Plan
    from mumax2 import workloads as W
    B = args.relax_batch
    nb = max(1, args.nsim // B)
    nrel = nb * B
    problem, sims, masks = W.relax_set(nrel, seed=rank)
    n = problem["n"]
    N = int(np.prod(n))
    gamma = problem["gamma"]
    thr_all = np.array([1e-4 * gamma * s["msat"] for s in sims])
    cold1 = W.cold_state(n, 1)
    plan = Plan(problem, masks={"msat": np.concatenate(masks[:B])}, sims=sims[:B], masks_per_sim=True,
                device=local_rank)
    plan.solver("rk23", dt=1e-14, maxerr=args.relax_maxerr)
    if args.profile_only:
        # pass timing of one evaluation and the batched RK23 step, on the plan of B slots
        # and on the 16-slot plan that finishes a pool (cold states, CUDA events)
        out = {}
        for k, p in (("slots%d" % B, plan), ("slots16", None)):
            if p is None:
                p = Plan(problem, masks={"msat": np.concatenate(masks[:16])}, sims=sims[:16], masks_per_sim=True,
                         device=local_rank)
                p.solver("rk23", dt=1e-14, maxerr=args.relax_maxerr)
            k_slots = B if p is plan else 16
            p.set_state(W.cold_state(n, k_slots))
            p.steps(20)
            torch.cuda.synchronize()
            pass_ms = p.profile_eval(args.profile_reps)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            p.steps(300)
            e1.record()
            torch.cuda.synchronize()
            out[k] = {"passes_us": [round(t * 1000, 1) for t in pass_ms], "tiles": p.tiles()[0],
                      "rk23_step_us": round(e0.elapsed_time(e1) / 300 * 1000, 1)}
            if p is not plan:
                p.close()
        plan.close()
        if rank == 0:
            print(json.dumps({"workload": "relax_64x64x1_cold", "profile": out}), flush=True)
        return None
    sampler = ClockSampler(local_rank)
    sampler.start()

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # synchronous batches (batch 0 repeated first as an untimed warm-up)
    sync_ms, sync_steps, sync_conv = 0.0, [], 0
    for k in range(nb + 1):
        j = max(0, k - 1)
        bs = sims[j * B:(j + 1) * B]
        plan.mask_tensor("msat").copy_(torch.from_numpy(np.concatenate(masks[j * B:(j + 1) * B])))
        plan.set_sims(bs)
        plan.solver("rk23", dt=1e-14, maxerr=args.relax_maxerr)
        thr = thr_all[j * B:(j + 1) * B]
        step0 = [s["step"] for s in plan.batch_stats()]
        torch.cuda.synchronize()
        e0, e1 = events()
        e0.record()
        plan.set_state(W.cold_state(n, B))
        plan.batch_run_until_maxtorque(thr, max_steps=args.relax_max_steps)
        e1.record()
        torch.cuda.synchronize()
        if k == 0:
            continue
        sync_ms += e0.elapsed_time(e1)
        st = plan.batch_stats()
        sync_steps += [s["step"] - s0 for s, s0 in zip(st, step0)]
        sync_conv += sum(1 for s, t in zip(st, thr) if s["maxtorque"] < t)

    # continuous batching over the same problems: the relaxation pool of the warm-start
    # evaluation (a finished slot takes the next problem at once; the last relaxations
    # move to a 16-slot drain plan, made here before the timed region)
    from mumax2 import warmstart as WS
    WS._tail_plan(plan, problem, masks[0], sims[0], 16, local_rank, args.relax_maxerr)
    plan.solver("rk23", dt=1e-14, maxerr=args.relax_maxerr)
    cold_all = np.repeat(cold1[None, :], nrel, axis=0)
    refill = max(1, B // 8)   # the pool refills once this many slots are free
    torch.cuda.synchronize()
    e0, e1 = events()
    e0.record()
    res = WS.relax_pool(problem, sims, masks, list(cold_all), thr_all, slots=B, maxerr=args.relax_maxerr,
                        max_steps=args.relax_max_steps, device=local_rank, plan=plan, want_energy=False)
    e1.record()
    torch.cuda.synchronize()
    cont_steps = list(res["steps"])
    cont_conv = int(np.sum(res["maxtorque"] < thr_all))
    worst = float(np.max(res["maxtorque"] / (gamma * np.array([q["msat"] for q in sims]))))
    cont_ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    ms_max, value = aggregate(cont_ms, 1, nrel, world, dist, "cuda")
    _, sync_value = aggregate(sync_ms, 1, nrel, world, dist, "cuda")
    if rank == 0:
        line = {"metric": "relaxations/s", "value": value, "unit": "relaxations/s", "n_gpus": world,
                "steps": nrel, "warmup": 1, "ms_per_step": ms_max / nrel, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "relax_64x64x1_cold", "relaxations": nrel, "slots": B,
                           "refill_per_drive": refill, "grid_xyz": list(W.RELAX_GRID_USER), "cell_nm": [4, 4, 3],
                           "solver": "rk23", "maxerr": args.relax_maxerr, "alpha": 1.0,
                           "start": "cold (uniform +x)",
                           "criterion": "maxtorque / (gamma Ms) < 1e-4 per simulation",
                           "parallelism": f"replicas{world}"},
                "relax": {"schedule": "continuous batching, 16-slot drain plan", "converged": cont_conv,
                          "of": nrel, "steps_mean": float(np.mean(cont_steps)),
                          "steps_max": int(np.max(cont_steps)), "worst_torque_over_gamma_ms": worst,
                          "drive_s": res["drive_s"], "host_s": res["host_s"]},
                "synchronous_batches": {"value": sync_value, "unit": "relaxations/s", "converged": sync_conv,
                                        "steps_mean": float(np.mean(sync_steps)),
                                        "steps_max": int(np.max(sync_steps))},
                "clocks": clocks}
        print(json.dumps(line), flush=True)
    plan.close()


# ---------------------------------------------------------------- single-simulation configs
def single_bench(args, rank, world, local_rank, dist, emit=True):
    """The single-simulation workloads: --workload sp4 (the 128x32x1 film of the SP4
    geometry, RK45, <m> every 10 ps) and --workload wall (the 512x128x1 Neel wall under
    Zhang-Li current, RK45, with the wall position from <m_x> every 10 ps, plus the
    Slonczewski variant on a 128x128x1 disk).
    Latency-bound sizes: the numbers are simulated time and steps per second."""
    import torch
    from mumax2 import Plan
    from mumax2 import workloads as W
    dur = args.duration
    runs = []
    if args.workload == "sp4":
        prob, m0 = W.sp4_film(seed=rank)
        runs.append(("sp4_film_128x32x1_rk45", prob, m0, None))
        dur = dur or 1e-9
    else:
        prob, m0, x0 = W.neel_wall_strip(seed=rank)
        runs.append(("neel_wall_512x128x1_zhangli_rk45", prob, m0, x0))
        # Slonczewski variant: 128x128x1 disk, p = +z (user), lambda 1, current along z
        n = (1, 128, 128)
        yy, xx = np.mgrid[0:128, 0:128]
        disk = (((xx + 0.5 - 64) ** 2 + (yy + 0.5 - 64) ** 2) <= 64 ** 2).astype(np.float32).ravel()
        sprob = dict(n=n, cell=(2e-9, 2e-9, 2e-9), pbc=(0, 0, 0), demag=1, exchange=1, slonczewski=1,
                     msat=8.6e5, aex=1.3e-11, alpha=0.02, gamma=2.211e5, p=(1.0, 0.0, 0.0), sl_pol=0.5,
                     **{"lambda": 1.0}, eps_prime=0.0, t_fl=2e-9, j=(1e11, 0.0, 0.0))
        sm = W.uniform_state(n, (0.1, 0.0, 1.0)).reshape(3, -1) * disk[None, :]
        runs.append(("slonczewski_disk_128x128x1_rk45", (sprob, {"msat": disk}), sm.ravel(), None))
        dur = dur or 5e-9
    out = []
    sampler = ClockSampler(local_rank)
    sampler.start()
    for name, prob, m0, x0 in runs:
        masks = {}
        if isinstance(prob, tuple):
            prob, masks = prob
        plan = Plan(prob, masks=masks, device=local_rank)
        plan.solver("rk45", dt=1e-15, maxerr=1e-5)
        plan.set_state(m0)
        plan.tabulate(1e-11, capacity=int(dur / 1e-11) + 16)
        plan.run(2e-11)       # warm-up: graph capture, first steps
        plan.tabulate_read()
        st0 = plan.stats()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.run(dur)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = plan.stats()
        rows = plan.tabulate_read()[0]
        N = int(np.prod(prob["n"]))
        steps = st["step"] - st0["step"]
        rec = {"workload": name, "cells": N, "simulated_s": dur, "steps": steps, "ms": ms,
               "steps_per_s": steps / (ms / 1e3), "cell_steps_per_s": N * steps / (ms / 1e3),
               "simulated_ns_per_s": dur * 1e9 / (ms / 1e3), "attempts": st["attempts"] - st0["attempts"],
               "avg_m_user_end": [float(v) for v in plan.average()[::-1]], "table_rows": len(rows)}
        if x0 is not None and len(rows) > 4:
            L = prob["n"][2] * prob["cell"][2]
            xw = W.wall_position(rows[:, 3], L)   # internal component 2 = user x
            h = len(rows) // 2
            v = np.polyfit(rows[h:, 0], xw[h:], 1)[0]
            rec.update({"wall_x0_m": x0, "wall_x_end_m": float(xw[-1]), "wall_velocity_m_per_s": float(v)})
        out.append(rec)
        plan.close()
    clocks = sampler.stop()
    if rank == 0:
        first = out[0]
        line = {"metric": "cell-steps/s", "value": first["cell_steps_per_s"], "unit": "cell-steps/s",
                "n_gpus": world, "steps": first["steps"], "warmup": 1, "ms_per_step": first["ms"] / first["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": first["workload"], "solver": "rk45", "maxerr": 1e-5,
                                                "parallelism": f"replicas{world}"},
                "runs": out, "clocks": clocks}
        if emit:
            print(json.dumps(line), flush=True)
        return line
    return None


# ---------------------------------------------------------------- learned warm start
def warmstart_bench(args, rank, world, local_rank, dist, emit=True):
    """The learned warm start: relaxed states of --train problems (plain relax from the cold
    start, continuous batching) train the BF16 U-Net on the GPU; on --nsim held-out problems the
    warm start (network inference + relax) is timed against the cold relax.  value =
    warm relaxations/s (fallbacks to the cold start included).  A warm relax gets the 99th
    percentile of the training relaxations' step counts as its budget."""
    import torch
    from mumax2 import unet as U
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    t0 = time.perf_counter()
    problem, sims, masks, res = WS.generate(args.train, seed=1000 + rank, device=local_rank)
    t_gen = time.perf_counter() - t0
    data = WS.Dataset(problem, sims, masks, res["state"], device=local_rank, mirror=not args.no_mirror)
    t0 = time.perf_counter()
    net, losses = WS.train(data, epochs=args.epochs, batch=256, lr=2e-3, device=local_rank,
                           tcgen05=not args.mma_sync)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    steps_per_epoch = len(data) // 256
    flops = 3 * U.conv_flops(64, 64) * 256 * steps_per_epoch * args.epochs
    _, hs, hm = W.relax_set(args.nsim, seed=5000 + rank)
    sampler = ClockSampler(local_rank)
    sampler.start()
    ev = WS.evaluate(net, problem, hs, hm, device=local_rank, max_steps=WS.step_budget(res["steps"]),
                     longest_first=not args.warm_index_order)
    clocks = sampler.stop()
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = float(json.load(open(peaks_path))["bf16_tflops_sustained"]) if os.path.exists(peaks_path) else 1400.0
    if rank == 0:
        line = {"metric": "relaxations/s", "value": ev["warm_per_s"], "unit": "relaxations/s", "n_gpus": world,
                "steps": ev["relaxations"], "warmup": 0, "ms_per_step": 1e3 / ev["warm_per_s"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32",
                "data": "synthetic",
                "config": {"workload": "relax_64x64x1_warm_start", "held_out": args.nsim, "train": args.train,
                           "epochs": args.epochs, "net": "U-Net 4 levels, 32/64/128/256 channels, 3x3, bf16",
                           "training_set": "relaxed states" + ("" if args.no_mirror else
                                                               " and their x-mirror images"),
                           "conv": "mma.sync" if args.mma_sync else "tcgen05",
                           "parallelism": f"replicas{world}"},
                "warm_vs_cold": ev,
                "training": {"generate_s": t_gen, "train_s": t_train, "loss_first_epoch": losses[0],
                             "loss_last_epoch": losses[-1],
                             "tflops_achieved": flops / t_train / 1e12, "tflops_peak_sustained": peak,
                             "frac": flops / t_train / 1e12 / peak},
                "clocks": clocks}
        if emit:
            print(json.dumps(line), flush=True)
        return line
    return None


def extra_workloads(args, rank, world, local_rank, dist):
    """The other halves of the headline metric, measured in the default run on the same
    GPU after the film: the learned warm start (20,000 training relaxations, 4,096
    held-out problems relaxed cold and warm, batch 256), the thermal ensemble (2048
    simulations of five grid sizes, 200 stochastic Heun steps after 5 warm-up steps) and
    the RK45 single-simulation configurations (SP4 film, Neel wall, Slonczewski disk).
    Each is summarised under its own key; its full line is what --workload prints."""
    import copy
    out = {}
    a = copy.copy(args)
    a.nsim, a.mma_sync = 4096, False
    t0 = time.perf_counter()
    try:
        ws = warmstart_bench(a, rank, world, local_rank, dist, emit=False)
        ev = ws["warm_vs_cold"]
        out["warm_start"] = {
            "workload": "relax_64x64x1_warm_start", "metric": "relaxations/s",
            "warm_per_s": ev["warm_per_s"], "cold_per_s": ev["cold_per_s"], "warm_vs_cold": ev["speedup"],
            "held_out": ev["relaxations"], "train": a.train, "epochs": a.epochs, "batch": 256,
            "cold_steps_mean": ev["cold_steps_mean"], "warm_steps_mean": ev["warm_steps_mean"],
            "warm_steps_incl_fallbacks_mean": ev["warm_steps_incl_fallbacks_mean"],
            "fallbacks": ev["fallbacks"], "final_converged_frac": ev["final_converged_frac"],
            "energy_within_1e-4_frac": ev["energy_within_tol_frac"],
            "criterion": "maxtorque / (gamma Ms) < 1e-4, final energy within 1e-4 relative of the cold relax",
            "training": ws["training"], "clocks": ws["clocks"], "seconds": time.perf_counter() - t0}
    except Exception as ex:  # reported, not fatal
        out["warm_start"] = {"failed": f"{type(ex).__name__}: {ex}"}
    a = copy.copy(args)
    a.nsim, a.steps, a.warmup, a.ens_attempts = 2048, 200, 5, args.ens_attempts
    t0 = time.perf_counter()
    try:
        en = ensemble_bench(a, rank, world, local_rank, dist, emit=False)
        out["ensemble"] = {"workload": en["config"]["workload"], "metric": "cell-steps/s", "value": en["value"],
                           "ms_per_step": en["ms_per_step"], "steps": a.steps, "warmup": a.warmup,
                           "config": en["config"], "roofline": en["roofline"], "e2e": en["e2e"],
                           "unbatched": en["unbatched"], "gpu_launches": en["gpu_launches"],
                           "clocks": en["clocks"], "seconds": time.perf_counter() - t0}
    except Exception as ex:  # reported, not fatal
        out["ensemble"] = {"failed": f"{type(ex).__name__}: {ex}"}
    # the RK45 single-simulation configurations: the SP4 film (1 ns) and the Neel wall under
    # Zhang-Li current with the Slonczewski disk (5 ns each)
    for wl in ("sp4", "wall"):
        a = copy.copy(args)
        a.workload, a.duration = wl, 0.0
        t0 = time.perf_counter()
        try:
            sl = single_bench(a, rank, world, local_rank, dist, emit=False)
            out["rk45_" + wl] = {"metric": "cell-steps/s", "runs": sl["runs"], "clocks": sl["clocks"],
                                 "seconds": time.perf_counter() - t0}
        except Exception as ex:  # reported, not fatal
            out["rk45_" + wl] = {"failed": f"{type(ex).__name__}: {ex}"}
    return out


# ---------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference-kernels-on-this-GPU comparison (RK12) of the film workload")
    ap.add_argument("--profile-reps", type=int, default=10)
    ap.add_argument("--no-extras", action="store_true",
                    help="film3d: leave out the warm-start, ensemble and RK45 measurements of the default line")
    ap.add_argument("--profile-only", action="store_true",
                    help="film3d: only time the passes of one field evaluation (few launches; for ncu "
                         "captures); relax: the passes and the batched RK23 step of the pool's plans")
    ap.add_argument("--workload", default="film3d",
                    choices=["film3d", "ensemble", "relax", "sp4", "wall", "warmstart"],
                    help="film3d: the 256x256x16 RK23 film (default); ensemble: 2048 thermal simulations; "
                         "relax: batched cold relaxations of 64x64x1 films; sp4: the 128x32x1 RK45 film; "
                         "wall: Zhang-Li domain wall and Slonczewski disk; warmstart: the learned warm start")
    ap.add_argument("--train", type=int, default=20000, help="warmstart: training relaxations")
    ap.add_argument("--epochs", type=int, default=40, help="warmstart: training epochs")
    ap.add_argument("--warm-index-order", action="store_true",
                    help="warmstart: start the warm relaxations in index order (not longest first)")
    ap.add_argument("--no-mirror", action="store_true",
                    help="warmstart: train without the mirror-image copies of the relaxed problems")
    ap.add_argument("--mma-sync", action="store_true",
                    help="warmstart: forward and data-gradient convolutions on the mma.sync kernel")
    ap.add_argument("--duration", type=float, default=0.0, help="sp4/wall: simulated time (s)")
    ap.add_argument("--relax-batch", type=int, default=256)
    ap.add_argument("--relax-maxerr", type=float, default=1e-6)
    ap.add_argument("--relax-max-steps", type=int, default=100000)
    ap.add_argument("--nsim", type=int, default=0,
                    help="ensemble: simulations (2048); relax: relaxations (2048); warmstart: held-out problems (4096)")
    ap.add_argument("--ens-attempts", type=int, default=50, help="ensemble: attempts per graph launch")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.workload in ("ensemble", "relax", "sp4", "wall", "warmstart"):
        fn = {"ensemble": ensemble_bench, "relax": relax_bench, "sp4": single_bench, "wall": single_bench,
              "warmstart": warmstart_bench}
        if not args.nsim:
            args.nsim = 4096 if args.workload == "warmstart" else 2048
        fn[args.workload](args, rank, world, local_rank, dist)
        if dist:
            dist.destroy_process_group()
        return

    from mumax2 import Plan
    w = WORKLOAD
    n = w["n"]
    N = n[0] * n[1] * n[2]
    plan = Plan(problem(), device=local_rank)
    tiles, tuned_us = plan.tiles()
    plan.solver(w["solver"], dt=w["dt0"], maxerr=w["maxerr"])
    plan.set_state(initial_m(replica_seed(rank)))
    if args.profile_only:
        geo = plan.geometry()
        pass_ms = plan.profile_eval(args.profile_reps)
        print(json.dumps({"passes": [{"pass": nm, "ms": t, "algorithmic_bytes": b}
                                     for (nm, b), t in zip(pass_bytes(geo, n), pass_ms)]}), flush=True)
        plan.close()
        return
    plan.steps(args.warmup)
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    st0 = plan.stats()
    l0 = plan.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.steps(args.steps)
    e1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    launches = plan.launch_count() - l0
    st1 = plan.stats()
    attempts = st1["attempts"] - st0["attempts"]
    evals = st1["evals"] - st0["evals"]
    ms_max, value = aggregate(ms, N, args.steps, world, dist, "cuda")

    # per-pass timing of one evaluation (CUDA events on the launching stream)
    geo = plan.geometry()
    pass_ms = plan.profile_eval(args.profile_reps)
    pb = pass_bytes(geo, n)
    shares = [x / sum(pass_ms) for x in pass_ms]
    dom = int(np.argmax(pass_ms))
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = pb[dom][1] / (pass_ms[dom] * 1e-3) / 1e9
    traffic = read_traffic().get(pb[dom][0])
    step_b = step_bytes_rk23(geo, n) * attempts / max(1, args.steps)
    step_gbs = step_b * args.steps / (ms / 1e3) / 1e9
    spec_b = survey_step_bytes(n, geo["L"], 3, 132)
    spec_gbs = spec_b * args.steps / (ms / 1e3) / 1e9

    # end-to-end through the C-ABI with host buffers: per step H2D of the state from
    # pinned memory, one mm_step, D2H of the state
    e2e_steps = min(args.steps, 10)
    host_in = torch.from_numpy(plan.get_state()).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    import ctypes as C
    from mumax2 import _native as nat
    L = nat.lib()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(e2e_steps):
        nat.check(L.mm_set_state(plan.h, C.c_void_p(host_in.data_ptr()), 1, None))
        nat.check(L.mm_step(plan.h, None))
        nat.check(L.mm_get_state(plan.h, C.c_void_p(host_out.data_ptr()), 1, None))
    f1.record()
    torch.cuda.synchronize()
    e2e_ms, e2e_value = aggregate(f0.elapsed_time(f1), N, e2e_steps, world, dist, "cuda")
    e2e_pipe = e2e_pipelined(plan, host_in, local_rank, steps=4 * e2e_steps, jobs=4)
    _, e2e_pipe_value = aggregate(e2e_pipe["ms"], N, e2e_pipe["steps"], world, dist, "cuda")

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline()
        except Exception as ex:  # reported, not fatal
            cb = {"value": None, "unit": "cell-steps/s", "cores": None, "kind": "port", "sample": f"failed: {ex}"}
    fc = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        try:
            fc = cufft_comparator(tuple(geo["L"]), sum(pass_ms))
        except Exception as ex:  # reported, not fatal
            fc = {"unavailable": f"failed: {ex}"}
    rg = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        try:
            rg = reference_gpu_baseline(local_rank)
        except Exception as ex:  # reported, not fatal
            rg = {"unavailable": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": film_config(world),
            "tiles": {"chosen": tiles, "tuned_eval_us": tuned_us},
            "roofline": {"bound": "hbm", "kernel": pb[dom][0], "achieved": achieved, "peak": peak,
                         "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": pb[dom][1], "launch_ms": pass_ms[dom]},
            "passes": [{"pass": nm, "ms": t, "share": s, "algorithmic_bytes": b, "gbs": b / (t * 1e-3) / 1e9}
                       for (nm, b), t, s in zip(pb, pass_ms, shares)],
            "step_roofline": {"model": "hot-path specification, minimal-pass model (1,397 B per cell-step here)",
                              "bytes_per_step": spec_b, "achieved_gbs": spec_gbs, "frac": spec_gbs / peak,
                              "design_bytes_per_step": step_b, "design_achieved_gbs": step_gbs,
                              "design_frac": step_gbs / peak},
            "attempts_per_step": attempts / args.steps, "evals_per_step": evals / args.steps,
            "e2e": {"value": e2e_pipe_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 12 * N,
                    "d2h_bytes_per_step": 12 * N, "steps": e2e_pipe["steps"],
                    "how": "independent jobs, each: H2D of its input state from pinned memory, one mm_step, D2H of "
                           "the result; four plans driven by four host threads on their own streams, so that the "
                           "copies of some jobs overlap the steps of the others",
                    "jobs": e2e_pipe["jobs"],
                    "serial": {"value": e2e_value, "steps": e2e_steps,
                               "how": "one plan, one stream: H2D, mm_step, D2H back to back"}},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cb if cb is None else {k: cb[k] for k in ["value", "unit", "cores", "kind", "sample"]},
            "reference_gpu": rg,
            "fft_comparator": fc,
        }
    plan.close()
    if rank == 0 and world == 1 and not args.no_extras:
        line.update(extra_workloads(args, rank, world, local_rank, dist))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
