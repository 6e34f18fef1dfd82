"""Python handle of one fused plan (geometry + parameters + demag kernel + stepper).

Device memory for masks and state lives in torch CUDA tensors (plumbing only); all
computation runs in libmm_b200.so.  Arrays are in the reference's internal axis
order (Z,Y,X), SoA [comp][n0][n1][n2]; a batched plan (`sims` given) holds nsim such
blocks one after the other, [sim][comp][n0][n1][n2].
"""
import ctypes as C

import numpy as np

from . import _native as nat


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("mm_b200 needs a CUDA device (sm_100a); none is available")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Plan:
    """One simulation, or nsim = len(sims) simulations of one geometry when `sims` (a list
    of dicts overriding msat, aex, alpha, bext, ku, anisu, temp, seed) is given.  Masks are
    shared by all simulations unless masks_per_sim, in which case each holds nsim x N."""

    def __init__(self, problem, masks=None, device=0, sims=None, masks_per_sim=False):
        torch = _torch()
        self.torch = torch
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        torch.cuda.set_device(self.device)
        self.problem = dict(problem)
        n = self.problem["n"]
        self.N = int(n[0]) * int(n[1]) * int(n[2])
        self.nsim = len(sims) if sims else 1
        self._masks = {}
        self._mask_ptrs = {}
        self._upload_masks(masks or {})
        self._struct = nat.make_problem(self.problem, self._mask_ptrs)
        h = C.c_void_p()
        if sims:
            self._sims = nat.make_sims(self.problem, sims)
            nat.check(nat.lib().mm_plan_create_batch(C.byref(self._struct), self.nsim, C.cast(self._sims, C.c_void_p),
                                                     1 if masks_per_sim else 0, C.byref(h)))
        else:
            nat.check(nat.lib().mm_plan_create(C.byref(self._struct), C.byref(h)))
        self.h = h
        self._solver = None

    def _upload_masks(self, masks):
        torch = self.torch
        self._masks = {}
        self._mask_ptrs = {}
        for k, v in masks.items():
            if v is None:
                continue
            if k in nat.MASK_VECTORS:
                ts = [None if c is None else torch.as_tensor(np.ascontiguousarray(c, dtype=np.float32).ravel(),
                                                              device=self.device) for c in v]
                self._masks[k] = ts
                self._mask_ptrs[k] = [None if t is None else t.data_ptr() for t in ts]
            else:
                t = torch.as_tensor(np.ascontiguousarray(v, dtype=np.float32).ravel(), device=self.device)
                self._masks[k] = t
                self._mask_ptrs[k] = t.data_ptr()

    def set_problem(self, problem, masks=None):
        self.problem = dict(problem)
        if masks is not None:
            self._upload_masks(masks)
        self._struct = nat.make_problem(self.problem, self._mask_ptrs)
        nat.check(nat.lib().mm_plan_set_problem(self.h, C.byref(self._struct)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            nat.lib().mm_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self, a, count=None):
        """a as a contiguous float32 device tensor of `count` states (default: all of the
        plan's simulations), 3N floats each; any other size is refused here, since the
        library reads exactly that many floats."""
        torch = self.torch
        if isinstance(a, torch.Tensor):
            t = a.to(self.device, torch.float32).contiguous()
        else:
            t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32).ravel(), device=self.device)
        want = 3 * self.N * (self.nsim if count is None else count)
        if t.numel() != want:
            raise ValueError("state array of %d floats, expected %d (%s x 3N, N = %d)"
                             % (t.numel(), want, self.nsim if count is None else count, self.N))
        return t

    def tiles(self):
        """(tiles, eval_us): the autotuned tile shifts of the row, column and epilogue
        passes, the fused single-layer flag, and the timed evaluation with them."""
        t = (C.c_int * 4)()
        us = C.c_double(0.0)
        nat.check(nat.lib().mm_plan_tiles(self.h, t, C.byref(us)))
        return list(t[:]), us.value

    def demag_kernel(self):
        """The transformed demag tensor octant [6][kd0][kd1][kd2] (xx yy zz yz xz xy,
        internal axes), scaled by 1/(L0 L1 L2)."""
        kd = (C.c_int * 3)()
        nat.check(nat.lib().mm_plan_demag_kernel(self.h, None, kd))
        out = np.zeros((6, kd[0], kd[1], kd[2]), dtype=np.float32)
        nat.check(nat.lib().mm_plan_demag_kernel(self.h, out.ctypes.data_as(C.c_void_p), kd))
        return out

    def set_tiles(self, tiles):
        """tiles: [row, column, epilogue] shifts, optionally a fourth entry (fused
        single-layer evaluation, 0/1; 0 if left out)."""
        tiles = list(tiles) + [0] * (4 - len(tiles))
        nat.check(nat.lib().mm_plan_set_tiles(self.h, (C.c_int * 4)(*tiles)))

    def kernel_nonzero(self):
        out = (C.c_int * 6)()
        nat.check(nat.lib().mm_plan_kernel_nonzero(self.h, out))
        return list(out[:])

    def device_bytes(self):
        return nat.lib().mm_plan_device_bytes(self.h)

    def fields(self, m, noise_step=0, dt_thermal=0.0):
        torch = self.torch
        md = self._dev(m)
        out = {k: torch.zeros(3 * self.N * self.nsim, device=self.device)
               for k in ["demag", "ex", "anis", "zee", "therm", "eff"]}
        nat.check(nat.lib().mm_fields(self.h, _ptr(md), noise_step, dt_thermal, _ptr(out["demag"]), _ptr(out["ex"]),
                                      _ptr(out["anis"]), _ptr(out["zee"]), _ptr(out["therm"]), _ptr(out["eff"]), None))
        torch.cuda.synchronize(self.device)
        return out

    def torque(self, m, noise_step=0, dt_thermal=0.0):
        """Returns (torque array tau/gamma incl. STT/gamma, normalised m) as device tensors."""
        torch = self.torch
        md = self._dev(m).clone()
        t = torch.zeros(3 * self.N * self.nsim, device=self.device)
        nat.check(nat.lib().mm_torque(self.h, _ptr(md), noise_step, dt_thermal, _ptr(t), None))
        torch.cuda.synchronize(self.device)
        return t, md

    # ---- stepping
    def solver(self, name="rk12", dt=1e-15, mindt=1e-38, maxdt=1e38, maxerr=1.0 / 2000, abs_err=1e-4, rel_err=1e-3):
        """maxerr: the explicit solvers' error per step; abs_err/rel_err: solver/am12's
        m_maxAbsError and m_maxRelError."""
        nat.check(nat.lib().mm_solver_init(self.h, nat.SOLVERS[name], dt, mindt, maxdt, maxerr))
        if name == "am12":
            nat.check(nat.lib().mm_solver_am12_tolerances(self.h, abs_err, rel_err))
        self._solver = name

    def set_state(self, m):
        md = self._dev(m)
        nat.check(nat.lib().mm_set_state(self.h, _ptr(md), 0, None))

    def get_state(self):
        out = np.zeros(3 * self.N * self.nsim, dtype=np.float32)
        nat.check(nat.lib().mm_get_state(self.h, out.ctypes.data_as(C.c_void_p), 1, None))
        return out

    def set_time(self, t, dt=0.0):
        nat.check(nat.lib().mm_set_time(self.h, t, dt))

    def set_thermal_dt(self, dt):
        nat.check(nat.lib().mm_set_thermal_dt(self.h, dt))

    def step(self):
        nat.check(nat.lib().mm_step(self.h, None))

    def steps(self, n):
        nat.check(nat.lib().mm_steps(self.h, int(n), None))

    def run(self, duration):
        nat.check(nat.lib().mm_run(self.h, float(duration), None))

    def run_until_maxtorque(self, thr, max_steps=0):
        nat.check(nat.lib().mm_run_until_maxtorque(self.h, float(thr), int(max_steps), None))

    def queue_attempts(self, n, stream=None):
        nat.check(nat.lib().mm_queue_attempts(self.h, int(n), stream))

    def stats(self):
        s = nat.MMStats()
        nat.check(nat.lib().mm_get_stats(self.h, C.byref(s), None))
        return {k: getattr(s, k) for k, _ in nat.MMStats._fields_}

    def maxtorque(self):
        v = C.c_double()
        nat.check(nat.lib().mm_maxtorque(self.h, C.byref(v), None))
        return v.value

    def average(self):
        out = (C.c_double * 3)()
        nat.check(nat.lib().mm_average(self.h, out, None))
        return np.array(out[:])

    def energy(self):
        out = (C.c_double * 5)()
        nat.check(nat.lib().mm_energy(self.h, out, None))
        return dict(zip(["E_zeeman", "E_ex", "E_demag", "E_anis", "E"], out[:]))

    # ---- time-dependent inputs
    def set_table(self, quantity, times, values):
        """SetPointwise table of "bext" (T) or "j" (A/m^2): values[i] (internal component
        order) at times[i]; piecewise linear in between, evaluated on the device at every
        stage time.  An empty table removes it."""
        times = np.asarray(times, dtype=np.float64)
        rows = np.zeros((len(times), 4))
        if len(times):
            rows[:, 0] = times
            rows[:, 1:] = np.asarray(values, dtype=np.float64).reshape(-1, 3)
        self._tab = getattr(self, "_tab", {})
        self._tab[quantity] = np.ascontiguousarray(rows.ravel())
        nat.check(nat.lib().mm_set_table(self.h, nat.TABLES[quantity], len(times),
                                         self._tab[quantity].ctypes.data_as(C.c_void_p)))

    # ---- output
    def save_async(self, path, fmt="ovf", options=()):
        """Snapshot of m written to `path` by a host thread while the GPU keeps going."""
        nat.check(nat.lib().mm_save_async(self.h, str(path).encode(), nat.format_code(fmt, options), None))

    def save_wait(self):
        nat.check(nat.lib().mm_save_wait(self.h))

    def autosave(self, period, capacity=16):
        """Copy m on the device every `period` of simulated time (notify_autosave.go)."""
        nat.check(nat.lib().mm_autosave(self.h, float(period), int(capacity)))
        self._save_cap = int(capacity) if period > 0 else getattr(self, "_save_cap", 0)

    def autosave_read(self):
        """States saved since the last read: a list (one per simulation) of
        (times [k], states [k][3N])."""
        cap = max(1, getattr(self, "_save_cap", 0))
        n3 = 3 * self.N
        states = np.zeros((self.nsim, cap, n3), dtype=np.float32)
        times = np.zeros((self.nsim, cap))
        counts = np.zeros(self.nsim, dtype=np.int32)
        lost = np.zeros(self.nsim, dtype=np.int64)
        nat.check(nat.lib().mm_autosave_read(self.h, states.ctypes.data_as(C.c_void_p), times.ctypes.data_as(C.c_void_p),
                                             counts.ctypes.data_as(C.c_void_p), lost.ctypes.data_as(C.c_void_p),
                                             None))
        self.save_lost = lost
        return [(times[b, :counts[b]].copy(), states[b, :counts[b]].copy()) for b in range(self.nsim)]

    # ---- autotabulate on the device
    def tabulate(self, period, capacity=4096):
        """Record (t, <m>, maxtorque, dt, step) on the device every `period` of simulated
        time (no host synchronisation); period <= 0 turns it off."""
        nat.check(nat.lib().mm_tabulate(self.h, float(period), int(capacity)))
        self._tab_cap = int(capacity) if period > 0 else getattr(self, "_tab_cap", 0)

    def tabulate_read(self):
        """Rows recorded since the last read: a list (one per simulation) of arrays
        [rows][8] = (t, <m>_0, <m>_1, <m>_2, maxtorque, dt, step, 0), internal order."""
        cap = max(1, getattr(self, "_tab_cap", 0))
        out = np.zeros((self.nsim, cap, 8))
        counts = np.zeros(self.nsim, dtype=np.int32)
        lost = np.zeros(self.nsim, dtype=np.int64)
        nat.check(nat.lib().mm_tabulate_read(self.h, out.ctypes.data_as(C.c_void_p), counts.ctypes.data_as(C.c_void_p),
                                             lost.ctypes.data_as(C.c_void_p), None))
        self.tab_lost = lost
        return [out[b, :counts[b]].copy() for b in range(self.nsim)]

    # ---- batched plans: one entry per simulation
    def set_sims(self, sims):
        if len(sims) != self.nsim:
            raise ValueError("set_sims needs %d entries, got %d" % (self.nsim, len(sims)))
        self._sims = nat.make_sims(self.problem, sims)
        nat.check(nat.lib().mm_batch_set_sims(self.h, C.cast(self._sims, C.c_void_p)))

    def batch_run_until_maxtorque(self, thr, max_steps=0):
        """Each simulation b steps until its maxtorque < thr[b]."""
        self._thr = np.ascontiguousarray(thr, dtype=np.float64).ravel()
        if self._thr.shape != (self.nsim,):
            raise ValueError("one threshold per simulation needed (%d), got %d" % (self.nsim, self._thr.size))
        nat.check(nat.lib().mm_batch_run_until_maxtorque(self.h, self._thr.ctypes.data_as(C.c_void_p),
                                                         int(max_steps), None))

    def batch_restart(self, idx, m, thr, sims=None, max_steps=0):
        """Put new problems into slots idx (continuous batching): states m [k][3N] (host
        array, or a float32 tensor on this plan's device),
        torque thresholds thr [k], optional scalar dicts sims [k].  Per-simulation masks
        are updated by writing into this plan's mask tensors before the call."""
        idx = np.ascontiguousarray(idx, dtype=np.int32).ravel()
        k = len(idx)
        if hasattr(m, "data_ptr"):   # device tensor [k][3N] float32
            m = self._dev(m, k)
            mp, from_host = C.c_void_p(m.data_ptr()), 0
        else:
            m = np.ascontiguousarray(m, dtype=np.float32).ravel()
            if m.size != 3 * self.N * k:
                raise ValueError("batch_restart: %d floats for %d states of 3N = %d" % (m.size, k, 3 * self.N))
            mp, from_host = m.ctypes.data_as(C.c_void_p), 1
        thr = np.ascontiguousarray(thr, dtype=np.float64).ravel()
        if thr.size != k or (sims is not None and len(sims) != k):
            raise ValueError("batch_restart: one threshold (and one sims entry) per slot")
        sa = nat.make_sims(self.problem, sims) if sims is not None else None
        nat.check(nat.lib().mm_batch_restart(self.h, len(idx), idx.ctypes.data_as(C.c_void_p), mp, from_host,
                                             C.cast(sa, C.c_void_p) if sa is not None else None,
                                             thr.ctypes.data_as(C.c_void_p), int(max_steps), None))

    def batch_cancel(self, idx):
        """Stops the simulations in slots idx (they count as done until restarted)."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        nat.check(nat.lib().mm_batch_cancel(self.h, len(idx), idx.ctypes.data_as(C.c_void_p), None))

    def batch_drive(self, target_active=0, max_attempts=0):
        """Step until at most target_active simulations are still running."""
        nat.check(nat.lib().mm_batch_drive(self.h, int(target_active), int(max_attempts), None))

    def mask_tensor(self, name):
        """The device tensor behind a mask (for in-place slot updates)."""
        return self._masks[name]

    def batch_stats(self):
        arr = (nat.MMStats * self.nsim)()
        nat.check(nat.lib().mm_batch_stats(self.h, C.cast(arr, C.c_void_p), None))
        return [{k: getattr(s, k) for k, _ in nat.MMStats._fields_} for s in arr]

    def batch_maxtorque(self):
        out = np.zeros(self.nsim)
        nat.check(nat.lib().mm_batch_maxtorque(self.h, out.ctypes.data_as(C.c_void_p), None))
        return out

    def batch_average(self):
        out = np.zeros((self.nsim, 3))
        nat.check(nat.lib().mm_batch_average(self.h, out.ctypes.data_as(C.c_void_p), None))
        return out

    def batch_energy(self):
        """nsim x 5: E_zeeman, E_ex, E_demag, E_anis, E."""
        out = np.zeros((self.nsim, 5))
        nat.check(nat.lib().mm_batch_energy(self.h, out.ctypes.data_as(C.c_void_p), None))
        return out

    # ---- instrumentation
    def launch_count(self):
        return nat.lib().mm_plan_launch_count(self.h)

    def profile_eval(self, reps=10):
        out = (C.c_double * 8)()
        npass = C.c_int()
        nat.check(nat.lib().mm_profile_eval(self.h, int(reps), out, C.byref(npass), None))
        return list(out[:npass.value])

    def geometry(self):
        out = (C.c_int * 12)()
        nat.check(nat.lib().mm_plan_geometry(self.h, out))
        v = list(out[:])
        return dict(L=tuple(v[0:3]), M=v[3], h=v[4], hp=v[5], kd=tuple(v[6:9]), nk=v[9], demag=v[10], nsim=v[11])


class Ensemble:
    """Several plans (typically one batched plan per grid size) stepped together from one
    CUDA graph; `attempts` step attempts of every plan per graph launch."""

    def __init__(self, plans, attempts=16):
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p.h.value for p in self.plans])
        h = C.c_void_p()
        nat.check(nat.lib().mm_ensemble_create(arr, len(self.plans), int(attempts), C.byref(h)))
        self.h = h

    def steps(self, n):
        nat.check(nat.lib().mm_ensemble_steps(self.h, int(n), None))

    def run(self, duration):
        nat.check(nat.lib().mm_ensemble_run(self.h, float(duration), None))

    def launch_count(self):
        return nat.lib().mm_ensemble_launch_count(self.h)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            nat.lib().mm_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
