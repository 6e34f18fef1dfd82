"""ctypes binding of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, never by the product package.

All arrays are in the reference's internal axis order (Z,Y,X), SoA
[comp][n0][n1][n2], float64.  A problem is described by a plain dict with the
keys of `DESC_FIELDS` (see `make_desc`).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

FP = C.POINTER(C.c_float)
DP = C.POINTER(C.c_double)


class OrDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int * 3), ("cell", C.c_double * 3), ("pbc", C.c_int * 3),
        ("demag", C.c_int), ("exchange", C.c_int), ("anis", C.c_int), ("zeeman", C.c_int),
        ("thermal", C.c_int), ("zhangli", C.c_int), ("slonczewski", C.c_int),
        ("demag_accuracy", C.c_int),
        ("msat", C.c_double), ("aex", C.c_double), ("alpha", C.c_double), ("gamma", C.c_double),
        ("bext", C.c_double * 3), ("ku", C.c_double), ("anisu", C.c_double * 3),
        ("temp", C.c_double), ("seed", C.c_ulonglong),
        ("j", C.c_double * 3), ("zl_pol", C.c_double), ("xi", C.c_double),
        ("p", C.c_double * 3), ("sl_pol", C.c_double), ("lambda_", C.c_double),
        ("eps_prime", C.c_double), ("t_fl", C.c_double),
        ("msat_mask", FP), ("aex_mask", FP), ("alpha_mask", FP), ("ku_mask", FP),
        ("anisu_mask", FP * 3), ("bext_mask", FP * 3), ("j_mask", FP * 3),
        ("temp_mask", FP), ("xi_mask", FP), ("zl_pol_mask", FP),
        ("p_mask", FP * 3),
        ("sl_pol_mask", FP), ("lambda_mask", FP), ("eps_prime_mask", FP), ("t_fl_mask", FP),
        ("demag_exchange", C.c_int),
        ("demag_tensor", C.c_int),
    ]


class OrState(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("mindt", C.c_double), ("maxdt", C.c_double),
        ("maxerr", C.c_double), ("err", C.c_double), ("peakerr", C.c_double),
        ("step", C.c_longlong), ("badsteps", C.c_longlong), ("evals", C.c_longlong),
        ("noise_step", C.c_longlong), ("dt_thermal", C.c_double),
    ]


SOLVERS = {"euler": 0, "heun": 1, "rk12": 2, "rk23": 3, "rk45": 4, "am12": 5}

MASK_SCALARS = ["msat", "aex", "alpha", "ku", "temp", "xi", "zl_pol", "sl_pol", "lambda",
                "eps_prime", "t_fl"]
MASK_VECTORS = ["anisu", "bext", "j", "p"]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(path)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(OrDesc)]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_kernel_arne.argtypes = [C.c_int * 3, C.c_double * 3, C.c_int * 3, C.c_int, C.c_int, DP]
        L.or_kernel_newell.argtypes = [C.c_int * 3, C.c_double * 3, C.c_int * 3, DP]
        L.or_padded_size.argtypes = [C.c_int * 3, C.c_int * 3, C.c_int * 3]
        L.or_kernel_nonzero.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.or_normalize.argtypes = [C.c_void_p, DP]
        L.or_fields.argtypes = [C.c_void_p, DP, C.c_longlong, C.c_double, DP, DP, DP, DP, DP, DP]
        L.or_torque.argtypes = [C.c_void_p, DP, C.c_longlong, C.c_double, DP, DP]
        L.or_stt.argtypes = [C.c_void_p, DP, DP, DP]
        L.or_maxtorque.restype = C.c_double
        L.or_maxtorque.argtypes = [C.c_void_p, DP]
        L.or_average.argtypes = [C.c_void_p, DP, C.c_double * 3]
        L.or_energy.argtypes = [C.c_void_p, DP, C.c_double * 5]
        L.or_step.restype = C.c_int
        L.or_step.argtypes = [C.c_void_p, C.c_int, DP, C.POINTER(OrState), DP, C.POINTER(C.c_int)]
        L.or_thermal_normals.argtypes = [C.c_ulonglong, C.c_longlong, C.c_longlong, C.c_double * 3]
        L.or_num_threads.restype = C.c_int
        L.or_set_table.restype = C.c_int
        L.or_set_table.argtypes = [C.c_void_p, C.c_int, C.c_long, DP]
        L.or_set_time.argtypes = [C.c_void_p, C.c_double]
        L.or_step_am12.restype = C.c_int
        L.or_step_am12.argtypes = [C.c_void_p, DP, C.POINTER(OrState), C.c_double, C.c_double,
                                   C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(DP) if a is not None else None


DEFAULTS = dict(
    n=(1, 8, 8), cell=(3e-9, 3e-9, 3e-9), pbc=(0, 0, 0),
    demag=1, exchange=1, anis=0, zeeman=0, thermal=0, zhangli=0, slonczewski=0,
    demag_accuracy=6, msat=8e5, aex=1.3e-11, alpha=0.02, gamma=2.211e5,
    bext=(0.0, 0.0, 0.0), ku=0.0, anisu=(0.0, 0.0, 1.0), temp=0.0, seed=0,
    j=(0.0, 0.0, 0.0), zl_pol=1.0, xi=0.05, p=(0.0, 0.0, 1.0), sl_pol=1.0, **{"lambda": 1.0},
    eps_prime=0.0, t_fl=0.0, demag_exchange=0,
)


def full_desc(**kw):
    d = dict(DEFAULTS)
    d.update(kw)
    return d


def make_desc(d):
    """Build an OrDesc from a problem dict; returns (desc, keepalive)."""
    s = OrDesc()
    keep = []
    s.n[:] = list(d["n"])
    s.cell[:] = list(d["cell"])
    s.pbc[:] = list(d["pbc"])
    for k in ["demag", "exchange", "anis", "zeeman", "thermal", "zhangli", "slonczewski",
              "demag_accuracy"]:
        setattr(s, k, int(d[k]))
    s.demag_exchange = int(d.get("demag_exchange", 0))
    s.demag_tensor = {"arne": 0, "newell": 1}.get(d.get("demag_tensor", 0), d.get("demag_tensor", 0))
    for k in ["msat", "aex", "alpha", "gamma", "ku", "temp", "zl_pol", "xi", "sl_pol",
              "eps_prime", "t_fl"]:
        setattr(s, k, float(d[k]))
    s.lambda_ = float(d["lambda"])
    s.seed = int(d["seed"])
    for k in ["bext", "anisu", "j", "p"]:
        getattr(s, k)[:] = [float(x) for x in d[k]]
    masks = d.get("masks", {}) or {}
    for k in MASK_SCALARS:
        a = masks.get(k)
        if a is not None:
            a = np.ascontiguousarray(a, dtype=np.float32).ravel()
            keep.append(a)
            setattr(s, k + "_mask", a.ctypes.data_as(FP))
    for k in MASK_VECTORS:
        a = masks.get(k)
        if a is not None:
            arr = getattr(s, k + "_mask")
            for c in range(3):
                if a[c] is None:
                    continue
                ac = np.ascontiguousarray(a[c], dtype=np.float32).ravel()
                keep.append(ac)
                arr[c] = ac.ctypes.data_as(FP)
    return s, keep


class Oracle:
    """One FP64 problem instance (geometry, parameters, demag kernel)."""

    def __init__(self, problem):
        self.d = full_desc(**problem)
        desc, keep = make_desc(self.d)
        self.h = lib().or_create(C.byref(desc))
        del keep
        n = self.d["n"]
        self.N = int(n[0]) * int(n[1]) * int(n[2])

    def __del__(self):
        try:
            lib().or_destroy(self.h)
        except Exception:
            pass

    def _m(self, m):
        return np.ascontiguousarray(m, dtype=np.float64).reshape(3 * self.N).copy()

    def normalize(self, m):
        m = self._m(m)
        lib().or_normalize(self.h, _dp(m))
        return m

    def set_table(self, which, times, values):
        """Time table of B_ext (which=0, T) or j (which=1, A/m^2): rows (t, v0, v1, v2),
        internal component order (SetPointwise, api.go:172-190)."""
        rows = np.ascontiguousarray(np.column_stack([np.asarray(times, float),
                                                     np.asarray(values, float).reshape(-1, 3)]).ravel()
                                    if len(times) else np.zeros(0))
        lib().or_set_table(self.h, int(which), len(times), _dp(rows))

    def set_time(self, t):
        lib().or_set_time(self.h, float(t))

    def fields(self, m, noise_step=0, dt_thermal=0.0):
        m = self._m(m)
        out = {k: np.zeros(3 * self.N) for k in ["demag", "ex", "anis", "zee", "therm", "eff"]}
        lib().or_fields(self.h, _dp(m), noise_step, dt_thermal, _dp(out["demag"]), _dp(out["ex"]),
                        _dp(out["anis"]), _dp(out["zee"]), _dp(out["therm"]), _dp(out["eff"]))
        return out

    def torque(self, m, noise_step=0, dt_thermal=0.0):
        """Torque array (tau/gamma incl. STT/gamma) at normalize(m); returns (torque, m_norm, H_eff)."""
        m = self._m(m)
        t = np.zeros(3 * self.N)
        h = np.zeros(3 * self.N)
        lib().or_torque(self.h, _dp(m), noise_step, dt_thermal, _dp(t), _dp(h))
        return t, m, h

    def stt(self, m):
        m = self._m(m)
        zl = np.zeros(3 * self.N)
        sl = np.zeros(3 * self.N)
        lib().or_stt(self.h, _dp(m), _dp(zl), _dp(sl))
        return zl, sl

    def maxtorque(self, torque):
        t = np.ascontiguousarray(torque, dtype=np.float64)
        return lib().or_maxtorque(self.h, _dp(t))

    def average(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = (C.c_double * 3)()
        lib().or_average(self.h, _dp(a), out)
        return np.array(out[:])

    def energy(self, m):
        m = self._m(m)
        out = (C.c_double * 5)()
        lib().or_energy(self.h, _dp(m), out)
        return dict(zip(["E_zeeman", "E_ex", "E_demag", "E_anis", "E"], out[:]))

    def nonzero_components(self):
        out = (C.c_int * 6)()
        lib().or_kernel_nonzero(self.h, out)
        return list(out[:])


class OracleRun:
    """Time integration with the oracle's solvers (reference semantics)."""

    def __init__(self, oracle, m, solver="rk12", dt=1e-15, mindt=1e-38, maxdt=1e38, maxerr=1.0 / 2000,
                 dt_thermal=0.0, abs_err=1e-4, rel_err=1e-3):
        self.abs_err, self.rel_err = abs_err, rel_err
        self.o = oracle
        self.m = oracle._m(m)
        self.solver = SOLVERS[solver]
        self.st = OrState(t=0.0, dt=dt, mindt=mindt, maxdt=maxdt, maxerr=maxerr, err=0.0, peakerr=0.0,
                          step=0, badsteps=0, evals=0, noise_step=0, dt_thermal=dt_thermal)
        self.kf = np.zeros(3 * oracle.N)
        self.fv = C.c_int(0)

    def step(self):
        if self.solver == SOLVERS["am12"]:
            if not hasattr(self, "am_alpha"):
                self.am_alpha = C.c_double(0.0)
                self.am_iterations = C.c_longlong(0)
            rc = lib().or_step_am12(self.o.h, _dp(self.m), C.byref(self.st), self.abs_err, self.rel_err,
                                    C.byref(self.am_alpha), C.byref(self.am_iterations))
            if rc == -2:
                raise RuntimeError("time outside a pointwise table")
            if rc != 0:
                raise RuntimeError("the Adams-Moulton iterator cannot converge")
            return
        rc = lib().or_step(self.o.h, self.solver, _dp(self.m), C.byref(self.st), _dp(self.kf), C.byref(self.fv))
        if rc == -2:
            raise RuntimeError("time outside a pointwise table")
        if rc != 0:
            raise RuntimeError("oracle solver failed to converge")

    def run(self, duration, record_every=None, callback=None):
        t_end = self.st.t + duration
        next_rec = self.st.t
        while self.st.t < t_end:
            if callback is not None and record_every is not None and self.st.t >= next_rec:
                callback(self)
                next_rec += record_every
            self.step()

    def invalidate_fsal(self):
        self.fv.value = 0


def kernel_arne(L, cell, pbc=(0, 0, 0), accuracy=6, round_f32=False):
    K = np.zeros(9 * L[0] * L[1] * L[2])
    lib().or_kernel_arne((C.c_int * 3)(*L), (C.c_double * 3)(*cell), (C.c_int * 3)(*pbc), accuracy,
                         int(round_f32), _dp(K))
    return K.reshape(3, 3, L[0], L[1], L[2])


def kernel_newell(L, cell, pbc=(0, 0, 0)):
    """Newell tensor K = -N, 9 components [s][d][L0][L1][L2] like kernel_arne."""
    K = np.zeros(9 * L[0] * L[1] * L[2])
    lib().or_kernel_newell((C.c_int * 3)(*L), (C.c_double * 3)(*cell), (C.c_int * 3)(*pbc), _dp(K))
    return K.reshape(3, 3, L[0], L[1], L[2])


def padded_size(n, pbc=(0, 0, 0)):
    return tuple((2 * n[i] if (n[i] > 1 and pbc[i] == 0) else n[i]) for i in range(3))


def thermal_normals(seed, cell, step):
    out = (C.c_double * 3)()
    lib().or_thermal_normals(seed, cell, step, out)
    return np.array(out[:])
