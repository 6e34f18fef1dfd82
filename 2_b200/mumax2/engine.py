"""Quantity/module engine and the script API of MuMax2, for the hot path.

Mirrors, for the per-timestep micromagnetic path only:
  - the Engine with named quantities (src/mumax/engine/engine.go:32-55, quant.go:39-61),
    each a multiplier per component times an optional space-dependent mask
    (MASK quantities, quant.go) or a full array (FIELD quantities);
  - modules registered by name (engine/module.go:46-88) that add quantities and wire
    them into H_eff, torque and the solver (mod_micromag.go, mod_demag.go,
    mod_exchange6.go, mod_llg.go, mod_zeeman.go, mod_uniaxialanisotropy.go,
    mod_temperature.go, mod_zhang-li.go, mod_slonczewski.go, mod_maxtorque.go,
    mod_energy.go, solve_*.go);
  - the user API of src/mumax/engine/api.go (setgridsize, setcellsize, load, setv,
    getv, sets, gets, setmask, setarray, getarray, run, steps, run_until_smaller ...),
    with its x<->z axis swap (api.go:13,44,152) so user scripts keep x,y,z order.
Everything numeric runs in libmm_b200.so through `Plan` (the fused C-ABI); this layer
only keeps names, units and the lazy update semantics of the reference.
"""
import numpy as np

MU0 = 4e-7 * np.pi
GAMMA0 = 2.211e5

# quantity kinds (engine/quant.go)
VALUE, MASK, FIELD = "VALUE", "MASK", "FIELD"


class Quant:
    def __init__(self, name, ncomp, kind, unit="", desc="", value=None):
        self.name = name
        self.ncomp = ncomp
        self.kind = kind
        self.unit = unit
        self.desc = desc
        self.mult = list(value) if value is not None else [0.0] * ncomp  # internal order
        self.mask = None  # internal order (ncomp, n0, n1, n2) float32 or None

    def __repr__(self):
        return f"Quant({self.name}, {self.kind}, mult={self.mult})"


def _file_to_user(a):
    """[ncomp][n0][n1][n2] internal -> user layout [ncomp][x][y][z]."""
    a = np.asarray(a)
    if a.shape[0] == 3:
        a = a[::-1]
    return np.ascontiguousarray(np.transpose(a, (0, 3, 2, 1)))


def _swap_vec(v):
    """User (x,y,z) <-> internal (z,y,x) for vectors (common/index.go:70-85)."""
    v = list(v)
    if len(v) == 3:
        v[0], v[2] = v[2], v[0]
    return v


class Engine:
    SOLVERS = {"solver/euler": "euler", "solver/heun": "heun", "solver/rk12": "rk12", "solver/rk23": "rk23",
               "solver/rk45": "rk45", "solver/am12": "am12"}

    def __init__(self, device=0):
        self.device = device
        self.q = {}
        self.modules = []
        self.size = None     # internal (n0, n1, n2)
        self.cell = None     # internal
        self.periodic = [0, 0, 0]
        self.solver_name = None
        self.plan = None
        self._plan_key = None
        self._dirty_params = True
        self._solver_dirty = True
        self._m = None       # host copy when the plan is not built yet
        self._pointwise = {}  # SetPointwise tables: quantity -> [(t, internal value)]
        self._autotab = None  # (quants, filename, period, header written)
        self._autosave = None  # (quantity, format code, extension, period)
        self.outdir = "."
        self._last_output_t = 0.0
        self._output_id = 0
        self._tables_dirty = False
        for name, unit in [("t", "s"), ("dt", "s"), ("step", "")]:
            self._add(name, 1, VALUE, unit)
        self.q["dt"].mult = [1e-15]

    # ------------------------------------------------------------ quantities
    def _add(self, name, ncomp, kind, unit="", desc="", value=None):
        key = name.lower()
        if key not in self.q:
            self.q[key] = Quant(name, ncomp, kind, unit, desc, value)
        return self.q[key]

    def quant(self, name):
        key = name.lower()
        if key not in self.q:
            raise KeyError(f"no quantity {name!r}; loaded modules: {self.modules}")
        return self.q[key]

    def has(self, name):
        return name.lower() in self.q

    # ------------------------------------------------------------ geometry
    def set_gridsize(self, nx, ny, nz):
        if self.size is not None:
            raise RuntimeError("Grid size already set")
        self.size = (int(nz), int(ny), int(nx))

    def set_cellsize(self, cx, cy, cz):
        if self.cell is not None:
            raise RuntimeError("Cell size already set")
        self.cell = (float(cz), float(cy), float(cx))

    def set_periodic(self, px, py, pz):
        self.periodic = [int(pz), int(py), int(px)]

    @property
    def ncell(self):
        return self.size[0] * self.size[1] * self.size[2]

    # ------------------------------------------------------------ modules
    def load(self, name):
        if name in self.modules:
            return
        loaders = {
            "micromagnetism": self._load_micromag, "demag": self._load_demag, "exchange6": self._load_exchange,
            "demagexch": self._load_demagexch,
            "llg": self._load_llg, "zeeman": self._load_zeeman, "anisotropy/uniaxial": self._load_anis,
            "temperature/brown": self._load_temp, "zhang-li": self._load_zl, "slonczewski": self._load_slon,
            "maxtorque": self._load_maxtorque, "micromag/energy": self._load_energy,
        }
        if name in self.SOLVERS:
            self._load_solver(name)
        elif name in loaders:
            loaders[name]()
        else:
            raise KeyError(f"unknown module {name!r} (this build covers the micromagnetic hot path)")
        self.modules.append(name)

    def _load_magnetization(self):
        self._add("m", 3, FIELD, "", "magnetization")
        self._add("Msat", 1, MASK, "A/m", "saturation magnetization")
        self._add("H_eff", 3, FIELD, "A/m", "effective field")

    def _load_micromag(self):   # mod_micromag.go:22-40
        self._load_magnetization()
        for m in ["demag", "exchange6", "llg", "zeeman", "solver/rk12", "maxtorque"]:
            self.load(m)
        self.quant("dt").mult = [1e-15]
        self.quant("mindt").mult = [1e-15]
        self.quant("m_maxerror").mult = [1.0 / 2000.0]

    def _load_demag(self):
        self._load_magnetization()
        self._add("B", 3, FIELD, "T", "demag field")

    def _load_demagexch(self):  # mod_demagexchange.go:26-78
        self._load_magnetization()
        self._add("Aex", 1, VALUE, "J/m", "exchange coefficient")
        self._add("demag_acc", 1, VALUE, "", "demag field accuracy", [8.0])
        self._add("H_dex", 3, FIELD, "A/m", "demag+exchange field")

    def _load_exchange(self):
        self._load_magnetization()
        self._add("Aex", 1, MASK, "J/m", "exchange coefficient")
        self._add("H_ex", 3, FIELD, "A/m", "exchange field")

    def _load_llg(self):        # mod_llg.go:31-57
        self._load_magnetization()
        self._add("alpha", 1, MASK, "", "damping")
        self._add("gamma", 1, VALUE, "m/As", "gyromag. ratio", [GAMMA0])
        self._add("torque", 3, FIELD, "/s")

    def _load_zeeman(self):
        self._load_magnetization()
        self._add("B_ext", 3, MASK, "T", "externally applied magnetic field")

    def _load_anis(self):
        self._load_magnetization()
        self._add("H_anis", 3, FIELD, "A/m", "uniaxial anisotropy field")
        self._add("Ku", 1, MASK, "J/m3", "uniaxial anisotropy constant K")
        self._add("anisU", 3, MASK, "", "uniaxial anisotropy direction (unit vector)")

    def _load_temp(self):       # mod_temperature.go:25-46
        self.load("llg")
        self._add("Temp", 1, MASK, "K", "temperature")
        self._add("Therm_seed", 1, VALUE, "", "random seed for H_therm")
        self._add("H_therm", 3, FIELD, "A/m", "thermal fluctuating field")
        self._add("cutoff_dt", 1, VALUE, "s", "update thermal field at most once per cutoff_dt")

    def _load_current(self):
        self._add("j", 3, MASK, "A/m2", "current density")

    def _load_zl(self):         # mod_zhang-li.go:25-45
        self.load("llg")
        self._add("xi", 1, MASK, "", "degree of non-adiabaticity", [0.05])
        self._add("polarisation", 1, MASK, "", "polarization degree of the spin-current", [1.0])
        self._load_current()
        self._add("zzt", 3, FIELD, "/s", "Zhang-Li spin transfer torque")

    def _load_slon(self):       # mod_slonczewski.go:25-50
        self.load("llg")
        self._add("t_fl", 1, MASK, "", "free layer thickness")
        self._add("lambda", 1, MASK, "", "scattering control parameter", [1.0])
        self._add("p", 3, MASK, "", "polarization vector")
        self._add("pol", 1, MASK, "", "polarization efficiency", [1.0])
        self._add("epsilon_prime", 1, MASK, "", "field-like term", [0.0])
        self._load_current()
        self._add("stt", 3, FIELD, "/s", "Slonczewski spin transfer torque")

    def _load_maxtorque(self):
        self._add("maxtorque", 1, VALUE, "/s", "Maximum |torque|")

    def _load_energy(self):     # mod_energy.go:24-67
        for n in ["E", "E_zeeman", "E_ex", "E_demag", "E_anis"]:
            self._add(n, 1, VALUE, "J")

    def _load_solver(self, name):  # solve_rk12.go:33-76
        if self.solver_name is not None:
            raise RuntimeError("solver already set")
        self.solver_name = self.SOLVERS[name]
        self._add("mindt", 1, VALUE, "s", "Minimum time step", [1e-38])
        self._add("maxdt", 1, VALUE, "s", "Maximum time step", [1e38])
        self._add("badsteps", 1, VALUE, "", "Number of time steps that had to be re-done")
        self._add("m_error", 1, VALUE, "", "Error/step estimate for m")
        self._add("m_peakerror", 1, VALUE, "", "All-time maximum error/step for m")
        self._add("m_maxerror", 1, VALUE, "", "Maximum error/step for m", [1.0 / 2000.0])
        if self.solver_name == "am12":  # solve_am01.go:316-366
            self._add("bdf_iterations", 1, VALUE, "", "Number of iterations per step")
            self._add("m_maxAbsError", 1, VALUE, "", "Maximum absolute error per step for m", [1e-4])
            self._add("m_maxRelError", 1, VALUE, "", "Maximum relative error per step for m", [1e-3])

    # ------------------------------------------------------------ problem
    def _mult(self, name, default=0.0, comp=0):
        if not self.has(name):
            return default
        return self.quant(name).mult[comp]

    def _problem(self):
        if self.size is None or self.cell is None:
            raise RuntimeError("set the grid size and cell size first")
        has = self.has
        prob = dict(n=self.size, cell=self.cell, pbc=tuple(self.periodic),
                    demag=int("demag" in self.modules or "micromagnetism" in self.modules
                              or "demagexch" in self.modules),
                    demag_exchange=int("demagexch" in self.modules),
                    exchange=int(has("Aex")), anis=int(has("Ku")), zeeman=int(has("B_ext")),
                    thermal=int(has("Temp")), zhangli=int("zhang-li" in self.modules),
                    slonczewski=int("slonczewski" in self.modules),
                    msat=self._mult("Msat"), aex=self._mult("Aex"), alpha=self._mult("alpha"),
                    gamma=self._mult("gamma", GAMMA0),
                    bext=tuple(self.quant("B_ext").mult) if has("B_ext") else (0, 0, 0),
                    ku=self._mult("Ku"), anisu=tuple(self.quant("anisU").mult) if has("anisU") else (0, 0, 1),
                    temp=self._mult("Temp"), seed=int(self._mult("Therm_seed")),
                    j=tuple(self.quant("j").mult) if has("j") else (0, 0, 0),
                    zl_pol=self._mult("polarisation", 1.0), xi=self._mult("xi", 0.05),
                    p=tuple(self.quant("p").mult) if has("p") else (0, 0, 1), sl_pol=self._mult("pol", 1.0),
                    eps_prime=self._mult("epsilon_prime"), t_fl=self._mult("t_fl"))
        prob["lambda"] = self._mult("lambda", 1.0)
        if "demagexch" in self.modules:
            prob["demag_accuracy"] = int(self._mult("demag_acc", 8.0))
        masks = {}
        names = {"msat": "Msat", "aex": "Aex", "alpha": "alpha", "ku": "Ku", "temp": "Temp", "xi": "xi",
                 "zl_pol": "polarisation", "sl_pol": "pol", "lambda": "lambda", "eps_prime": "epsilon_prime",
                 "t_fl": "t_fl"}
        for k, qn in names.items():
            if has(qn) and self.quant(qn).mask is not None:
                masks[k] = self.quant(qn).mask.reshape(-1)
        for k, qn in {"anisu": "anisU", "bext": "B_ext", "j": "j", "p": "p"}.items():
            if has(qn) and self.quant(qn).mask is not None:
                mk = self.quant(qn).mask
                masks[k] = [mk[c].reshape(-1) for c in range(3)]
        return prob, masks

    def _ensure_plan(self):
        from .plan import Plan
        prob, masks = self._problem()
        key = (prob["n"], prob["cell"], prob["pbc"], prob["demag"], prob.get("demag_exchange", 0),
               prob.get("demag_accuracy", 6))
        if self.plan is None or self._plan_key != key:
            m = self._state_host()
            if self.plan is not None:
                self.plan.close()
            if self.plan is not None and self._autotab:
                self._drain_tab()
            self.plan = Plan(prob, masks=masks, device=self.device)
            self._plan_key = key
            self._tables_dirty = True
            if self._autotab:
                self.plan.tabulate(self._autotab[2], self.TAB_CAPACITY)
            if self._autosave:
                self.plan.autosave(self._autosave[3], self.SAVE_CAPACITY)
            self._dirty_params = False
            self._solver_dirty = True
            if m is not None:
                self.plan.set_state(m)
                self._m = None
        elif self._dirty_params:
            self.plan.set_problem(prob, masks)
            self._dirty_params = False
        if self._tables_dirty:
            for lname, table in (("b_ext", "bext"), ("j", "j")):
                pts = self._pointwise.get(lname, [])
                self.plan.set_table(table, [t for t, _ in pts], [v for _, v in pts])
            self._tables_dirty = False
        if self._solver_dirty and self.solver_name is not None:
            self.plan.solver(self.solver_name, dt=self.quant("dt").mult[0], mindt=self._mult("mindt", 1e-38),
                             maxdt=self._mult("maxdt", 1e38), maxerr=self._mult("m_maxerror", 1.0 / 2000),
                             abs_err=self._mult("m_maxAbsError", 1e-4), rel_err=self._mult("m_maxRelError", 1e-3))
            st = self.plan.stats()
            self.plan.set_time(self.quant("t").mult[0], self.quant("dt").mult[0])
            del st
            cutoff = self._mult("cutoff_dt")
            if cutoff > 0:
                self.plan.set_thermal_dt(cutoff)
            self._solver_dirty = False
        return self.plan

    def _state_host(self):
        if self.plan is not None:
            return self.plan.get_state()
        return self._m

    def _sync_stats(self):
        st = self.plan.stats()
        self.quant("t").mult = [st["t"]]
        self.quant("dt").mult = [st["dt"]]
        self.quant("step").mult = [float(st["step"])]
        if self.has("badsteps"):
            self.quant("badsteps").mult = [float(st["badsteps"])]
            self.quant("m_error").mult = [st["err"]]
            self.quant("m_peakerror").mult = [st["peakerr"]]
        if self.has("bdf_iterations"):
            self.quant("bdf_iterations").mult = [float(st["iterations"])]

    # ------------------------------------------------------------ API (api.go)
    def setv(self, name, value):
        q = self.quant(name)
        value = [float(v) for v in np.atleast_1d(value)]
        if len(value) != q.ncomp:
            raise ValueError(f"{name} has {q.ncomp} components")
        q.mult = _swap_vec(value)
        lname = name.lower()
        if lname == "m":
            raise ValueError("m is a field: use setarray")
        if lname in ("dt", "mindt", "maxdt", "m_maxerror", "t", "cutoff_dt", "m_maxabserror", "m_maxrelerror"):
            self._solver_dirty = True
        else:
            self._dirty_params = True

    def setpointwise(self, name, time, value):
        """SetPointwise (api.go:172-190): `name` follows a piecewise linear function of
        time through the given (time, value) points, evaluated on the device at every
        solver stage.  Appending a time earlier than the last one starts a new list
        (update_pointwise.go:91-97).  The device path covers B_ext and j."""
        q = self.quant(name)
        lname = name.lower()
        if lname not in ("b_ext", "j"):
            raise NotImplementedError(f"time tables are evaluated on the device for B_ext and j, not {name}")
        value = [float(v) for v in np.atleast_1d(value)]
        if len(value) != q.ncomp:
            raise ValueError(f"{name} has {q.ncomp} components")
        pts = self._pointwise.setdefault(lname, [])
        if pts and pts[-1][0] > time:
            pts.clear()
        pts.append((float(time), _swap_vec(value)))
        self._tables_dirty = True

    def getv(self, name):
        q = self.quant(name)
        self._update(name)
        return _swap_vec(q.mult)

    def sets(self, name, value):
        self.setv(name, [value])

    def gets(self, name):
        return self.getv(name)[0]

    def _user_to_internal_array(self, arr, ncomp):
        a = np.asarray(arr, dtype=np.float64)
        if a.ndim == 3:
            a = a[None]
        if a.shape[0] != ncomp:
            raise ValueError(f"array has {a.shape[0]} components, expected {ncomp}")
        # user layout [comp][x][y][z] -> internal [comp'][z][y][x] with comp x<->z
        a = np.transpose(a, (0, 3, 2, 1))
        if ncomp == 3:
            a = a[::-1]
        n = self.size
        if a.shape[1:] != tuple(n):
            # nearest-neighbour resampling (engine/resample.go)
            idx = [np.minimum((np.arange(n[d]) * a.shape[d + 1]) // n[d], a.shape[d + 1] - 1) for d in range(3)]
            a = a[:, idx[0]][:, :, idx[1]][:, :, :, idx[2]]
        return np.ascontiguousarray(a, dtype=np.float32)

    def _internal_to_user_array(self, a, ncomp):
        a = np.asarray(a).reshape((ncomp,) + tuple(self.size))
        if ncomp == 3:
            a = a[::-1]
        return np.ascontiguousarray(np.transpose(a, (0, 3, 2, 1)))

    def setarray(self, name, arr):
        q = self.quant(name)
        a = self._user_to_internal_array(arr, q.ncomp)
        if q.name.lower() == "m":
            if self.plan is not None:
                self.plan.set_state(a.reshape(-1))
            else:
                self._m = a.reshape(-1)
            return
        if q.kind == MASK:
            if any(m != 1 for m in q.mult):  # api.go:257-262
                raise ValueError(f"{name} is not an ordinary array, but has a mask + multiplier value. "
                                 "Did you mean to set the mask or the multiplier instead of the array?")
        q.mask = a
        self._dirty_params = True

    def setmask(self, name, arr):
        q = self.quant(name)
        if q.kind != MASK:
            raise ValueError(f"{name} is not a MASK quantity")
        q.mask = self._user_to_internal_array(arr, q.ncomp)
        self._dirty_params = True

    def getarray(self, name):
        q = self.quant(name)
        lname = q.name.lower()
        if lname == "m":
            m = self._state_host()
            return self._internal_to_user_array(m, 3)
        if q.kind == MASK:
            if q.mask is None:
                return self._internal_to_user_array(
                    np.broadcast_to(np.array(q.mult)[:, None], (q.ncomp, self.ncell)), q.ncomp)
            return self._internal_to_user_array(q.mask * np.array(q.mult)[:, None, None, None], q.ncomp)
        return self._internal_to_user_array(self._field(lname), q.ncomp)

    def _field(self, lname):
        import torch
        plan = self._ensure_plan()
        m = torch.as_tensor(plan.get_state(), device=plan.device)
        st = plan.stats()
        f = plan.fields(m, noise_step=0, dt_thermal=st["dt"])
        table = {"h_eff": "eff", "h_ex": "ex", "h_anis": "anis", "h_therm": "therm", "h_dex": "demag"}
        if lname in table:
            return f[table[lname]].cpu().numpy()
        if lname == "b":
            return (f["demag"] * MU0).cpu().numpy()
        if lname == "torque":
            t, _ = plan.torque(m)
            return t.cpu().numpy()
        raise KeyError(lname)

    def _update(self, name):
        lname = name.lower()
        if self.plan is None and lname in ("t", "dt", "step"):
            return
        if lname in ("t", "dt", "step", "badsteps", "m_error", "m_peakerror"):
            if self.plan is not None:
                self._sync_stats()
            return
        if lname == "maxtorque":
            self.quant("maxtorque").mult = [self._ensure_plan().maxtorque()]
        elif lname == "<m>":
            pass
        elif lname.startswith("e") and lname in ("e", "e_zeeman", "e_ex", "e_demag", "e_anis"):
            e = self._ensure_plan().energy()
            for k in ["E", "E_zeeman", "E_ex", "E_demag", "E_anis"]:
                self.quant(k).mult = [e[k]]

    def average_m(self):
        return _swap_vec(self._ensure_plan().average())

    # ------------------------------------------------------------ autotabulate
    TAB_CAPACITY = 65536
    TAB_COLUMNS = {"t": ([0], "s"), "<m>": ([1, 2, 3], ""), "maxtorque": ([4], "/s"), "dt": ([5], "s"),
                   "step": ([6], "")}

    def autotabulate(self, quants, filename, period):
        """AutoTabulate (engine.go:609-617, notify_tabulate.go:23-28): the rows are
        recorded on the device during the run and written to `filename` after it, in the
        reference's table format (table.go:33-70).  Device columns: t, <m>, maxtorque, dt,
        step."""
        for q in quants:
            if q.lower() not in self.TAB_COLUMNS and q not in self.TAB_COLUMNS:
                raise NotImplementedError(f"device autotabulate records t, <m>, maxtorque, dt, step; not {q}")
        self._autotab = [list(quants), filename, float(period), False]
        if self.plan is not None:
            self.plan.tabulate(float(period), self.TAB_CAPACITY)

    def _drain_tab(self):
        quants, filename, _, header = self._autotab
        rows = self.plan.tabulate_read()[0]
        cols = [self.TAB_COLUMNS.get(q, self.TAB_COLUMNS.get(q.lower())) for q in quants]
        with open(filename, "a") as f:
            if not header:
                h = "#"
                for q, (idx, unit) in zip(quants, cols):
                    n = len(idx)
                    for i in range(n - 1, -1, -1):
                        comp = "_" + chr(ord("z") - i) if n > 1 else ""
                        h += f"{q}{comp} ({unit})\t"
                f.write(h + "\n")
                self._autotab[3] = True
            for r in rows:
                line = ""
                for idx, _ in cols:
                    for i in reversed(idx):   # internal ZYX -> user XYZ
                        line += go_float(r[i]) + "\t"
                f.write(line + "\n")

    # ------------------------------------------------------------ output (engine.go:555-640)
    SAVE_CAPACITY = 32
    EXT = {0: "ovf", 1: "ovf", 2: "omf", 3: "omf", 4: "dump"}

    def _next_output_id(self, t):
        """OutputID (engine.go:98-105): a new number whenever the time has changed."""
        if t != self._last_output_t:
            self._last_output_t = t
            self._output_id += 1
        return self._output_id

    def _auto_filename(self, quant, code, t):
        import os
        return os.path.join(self.outdir, f"{quant}{self._next_output_id(t):06d}.{self.EXT[code]}")

    def _field_array(self, name):
        lname = name.lower()
        q = self.quant(name)
        if lname == "m":
            return self._ensure_plan().get_state(), q
        if q.kind == MASK:
            if q.mask is None:
                return np.repeat(np.array(q.mult, dtype=np.float32), self.ncell), q
            return (q.mask * np.array(q.mult)[:, None, None, None]).reshape(-1).astype(np.float32), q
        return np.asarray(self._field(lname), dtype=np.float32), q

    def saveas(self, name, fmt, options, filename):
        from . import _native as nat
        code = nat.format_code(fmt, options)
        data, q = self._field_array(name)
        self._sync_stats() if self.plan is not None else None
        nat.write_field(filename, code, data, self.size, self.cell, self.quant("t").mult[0], q.name, q.unit)

    def save(self, name, fmt, options):
        from . import _native as nat
        code = nat.format_code(fmt, options)
        if self.plan is not None:
            self._sync_stats()
        self.saveas(name, fmt, options, self._auto_filename(name, code, self.quant("t").mult[0]))

    def autosave(self, name, fmt, options, period):
        """AutoSave (engine.go:576-582): m is copied on the device by the step that
        crosses each save time and written to the auto-numbered files after the run."""
        from . import _native as nat
        if name.lower() != "m":
            raise NotImplementedError("device autosave covers m")
        code = nat.format_code(fmt, options)
        self._autosave = (name, code, self.EXT[code], float(period))
        if self.plan is not None:
            self.plan.autosave(float(period), self.SAVE_CAPACITY)

    def _drain_save(self):
        from . import _native as nat
        name, code, _, _ = self._autosave
        times, states = self.plan.autosave_read()[0]
        q = self.quant(name)
        for t, m in zip(times, states):
            nat.write_field(self._auto_filename(name, code, t), code, m, self.size, self.cell, t, q.name, q.unit)

    def setarray_file(self, name, filename):
        """SetArray_File (api.go:267-269): read an OMF/OVF/dump file into a field."""
        from . import _native as nat
        data, n, _ = nat.read_field(filename)
        self.setarray(name, _file_to_user(data))

    def setmask_file(self, name, filename):
        from . import _native as nat
        data, n, _ = nat.read_field(filename)
        self.setmask(name, _file_to_user(data))

    def _after_run(self):
        self._sync_stats()
        if self._autotab:
            self._drain_tab()
        if self._autosave:
            self._drain_save()

    def run(self, duration):
        self._ensure_plan().run(duration)
        self._after_run()

    def steps(self, n):
        self._ensure_plan().steps(n)
        self._after_run()

    def run_until_smaller(self, name, value):
        if name.lower() != "maxtorque":
            raise NotImplementedError("run_until_smaller is supported for maxtorque (the relax idiom)")
        self._ensure_plan().run_until_maxtorque(value)
        self._after_run()


def go_float(v):
    """A float64 the way Go's fmt.Fprint writes it: shortest round-trip digits in
    strconv's 'g' form, with the exponent form when the decimal exponent is < -4 or >= 6
    (the precision strconv uses for that decision with shortest digits)."""
    import decimal
    v = float(v)
    if v != v:
        return "NaN"
    if v in (float("inf"), float("-inf")):
        return "+Inf" if v > 0 else "-Inf"
    if v == 0.0:
        return "0"
    sign, digits, exp = decimal.Decimal(repr(v)).normalize().as_tuple()
    ds = "".join(str(d) for d in digits)
    nd = len(ds)
    dp = nd + exp        # position of the decimal point
    x = dp - 1
    s = "-" if sign else ""
    if x < -4 or x >= 6:
        mant = ds[0] + ("." + ds[1:] if nd > 1 else "")
        return f"{s}{mant}e{'+' if x >= 0 else '-'}{abs(x):02d}"
    if dp <= 0:
        return s + "0." + "0" * (-dp) + ds
    if dp >= nd:
        return s + ds + "0" * (dp - nd)
    return s + ds[:dp] + "." + ds[dp:]


# ---------------------------------------------------------------- script API (src/python/mumax2.py)
_engine = None


def engine():
    global _engine
    if _engine is None:
        _engine = Engine()
    return _engine


def reset():
    global _engine
    if _engine is not None and _engine.plan is not None:
        _engine.plan.close()
    _engine = None


def setgridsize(nx, ny, nz):
    engine().set_gridsize(nx, ny, nz)


def setcellsize(cx, cy, cz):
    engine().set_cellsize(cx, cy, cz)


def setperiodic(px, py, pz):
    engine().set_periodic(px, py, pz)


def load(name):
    engine().load(name)


def setv(name, value):
    if name == "<m>":
        raise ValueError("<m> is derived")
    engine().setv(name, value)


def save(name, fmt, options=()):
    engine().save(name, fmt, options)


def saveas(name, fmt, options, filename):
    engine().saveas(name, fmt, options, filename)


def autosave(name, fmt, options, period):
    engine().autosave(name, fmt, options, period)


def setarray_file(name, filename):
    engine().setarray_file(name, filename)


def setmask_file(name, filename):
    engine().setmask_file(name, filename)


def autotabulate(quants, filename, period):
    engine().autotabulate(quants, filename, period)


def setpointwise(name, time, value):
    engine().setpointwise(name, time, value)


def getv(name):
    if name == "<m>":
        return engine().average_m()
    return engine().getv(name)


def sets(name, value):
    engine().sets(name, value)


def gets(name):
    return engine().gets(name)


def setarray(name, arr):
    engine().setarray(name, arr)


def setmask(name, arr):
    engine().setmask(name, arr)


def getarray(name):
    return engine().getarray(name)


def run(duration):
    engine().run(duration)


def steps(n):
    engine().steps(n)


def step():
    engine().steps(1)


def run_until_smaller(name, value):
    engine().run_until_smaller(name, value)
