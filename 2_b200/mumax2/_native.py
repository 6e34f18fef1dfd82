"""ctypes binding of libmm_b200.so (the sm_100a CUDA library, C-ABI in include/mm_b200.h).

The library is loaded from the package directory (built in-tree by 2_b200/build.py).
There is no fallback: if the library is missing or cannot be loaded, every entry
point raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "libmm_b200.so"))
_lib = None

FP = C.POINTER(C.c_float)
DP = C.POINTER(C.c_double)

MM_OK = 0
MM_ERR_ARG = -1
MM_ERR_CUDA = -2
MM_ERR_NOT_CONVERGED = -3
MM_ERR_NAN = -4
MM_ERR_STATE = -5
MM_ERR_TIMEOUT = -6
MM_ERR_RANGE = -7
TABLES = {"bext": 0, "j": 1}
FORMATS = {"ovf": 0, "ovf_text": 1, "omf": 2, "omf_text": 3, "dump": 4}


def format_code(fmt, options=()):
    """The reference's (format, options) pair -> MM_FMT_* ("ovf"/"omf" with [] or
    ["Binary 4"] -> binary, ["Text"] -> text; "dump")."""
    fmt = fmt.lower()
    opts = [o.lower() for o in (options or [])]
    if fmt == "dump":
        if opts:
            raise ValueError("dump output format does not take options")
        return FORMATS["dump"]
    if fmt not in ("ovf", "omf"):
        raise ValueError(f"unknown output format {fmt!r}")
    if len(opts) > 1:
        raise ValueError(f"illegal {fmt.upper()} options: {options}")
    if not opts or opts[0] == "binary 4":
        return FORMATS[fmt]
    if opts[0] == "text":
        return FORMATS[fmt + "_text"]
    raise ValueError(f"illegal {fmt.upper()} data format {options[0]!r}: options are Text, Binary 4")


def write_field(path, fmt_code, data, n, cell, time, name, unit):
    """data: float32 [ncomp][n0][n1][n2] (internal order) on the host."""
    import numpy as np
    a = np.ascontiguousarray(data, dtype=np.float32)
    ncomp = a.size // (int(n[0]) * int(n[1]) * int(n[2]))
    check(lib().mm_write_field(str(path).encode(), int(fmt_code), a.ctypes.data_as(C.c_void_p), ncomp,
                               (C.c_int * 3)(*[int(x) for x in n]), (C.c_double * 3)(*[float(x) for x in cell]),
                               float(time), name.encode(), unit.encode()))


def read_field(path):
    """-> (data float32 [ncomp][n0][n1][n2] internal order, n, time)."""
    import numpy as np
    nc = C.c_int()
    n = (C.c_int * 3)()
    t = C.c_double()
    check(lib().mm_read_field(str(path).encode(), None, 0, C.byref(nc), n, C.byref(t)))
    a = np.zeros(nc.value * n[0] * n[1] * n[2], dtype=np.float32)
    check(lib().mm_read_field(str(path).encode(), a.ctypes.data_as(C.c_void_p), a.size, C.byref(nc), n, C.byref(t)))
    return a.reshape(nc.value, n[0], n[1], n[2]), tuple(n), t.value

SOLVERS = {"euler": 0, "heun": 1, "rk12": 2, "rk23": 3, "rk45": 4, "am12": 5}
TENSORS = {"arne": 0, "newell": 1}


class MMProblem(C.Structure):
    """mm_problem of include/mm_b200.h (device mask pointers)."""
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
        ("msat_mask", C.c_void_p), ("aex_mask", C.c_void_p), ("alpha_mask", C.c_void_p),
        ("ku_mask", C.c_void_p),
        ("anisu_mask", C.c_void_p * 3), ("bext_mask", C.c_void_p * 3), ("j_mask", C.c_void_p * 3),
        ("temp_mask", C.c_void_p), ("xi_mask", C.c_void_p), ("zl_pol_mask", C.c_void_p),
        ("p_mask", C.c_void_p * 3),
        ("sl_pol_mask", C.c_void_p), ("lambda_mask", C.c_void_p), ("eps_prime_mask", C.c_void_p),
        ("t_fl_mask", C.c_void_p),
        ("demag_exchange", C.c_int),
        ("demag_tensor", C.c_int),
    ]


class MMStats(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("err", C.c_double), ("peakerr", C.c_double),
        ("maxtorque", C.c_double), ("step", C.c_longlong), ("badsteps", C.c_longlong),
        ("attempts", C.c_longlong), ("evals", C.c_longlong), ("status", C.c_int), ("done", C.c_int),
        ("iterations", C.c_longlong),
    ]


class MMSim(C.Structure):
    """mm_sim of include/mm_b200.h: the scalars of one simulation of a batched plan."""
    _fields_ = [
        ("msat", C.c_double), ("aex", C.c_double), ("alpha", C.c_double), ("bext", C.c_double * 3),
        ("ku", C.c_double), ("anisu", C.c_double * 3), ("temp", C.c_double), ("seed", C.c_ulonglong),
    ]


SIM_KEYS = ["msat", "aex", "alpha", "bext", "ku", "anisu", "temp", "seed"]


def make_sims(problem, sims):
    """Array of MMSim: each entry of `sims` (dicts) overrides the problem's scalars."""
    arr = (MMSim * len(sims))()
    for b, d in enumerate(sims):
        q = dict(problem)
        q.update(d)
        s = arr[b]
        s.msat = float(q.get("msat", 8e5))
        s.aex = float(q.get("aex", 1.3e-11))
        s.alpha = float(q.get("alpha", 0.02))
        s.bext[:] = [float(x) for x in q.get("bext", (0, 0, 0))]
        s.ku = float(q.get("ku", 0.0))
        s.anisu[:] = [float(x) for x in q.get("anisu", (0, 0, 1))]
        s.temp = float(q.get("temp", 0.0))
        s.seed = int(q.get("seed", 0))
    return arr


class MMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mm_b200 error {code}: {msg}")
        self.code = code


_PROTOS = {
    "mm_last_error": (C.c_char_p, []),
    "mm_version": (C.c_char_p, []),
    "mm_plan_create": (C.c_int, [C.POINTER(MMProblem), C.POINTER(C.c_void_p)]),
    "mm_plan_destroy": (C.c_int, [C.c_void_p]),
    "mm_plan_set_problem": (C.c_int, [C.c_void_p, C.POINTER(MMProblem)]),
    "mm_plan_kernel_nonzero": (C.c_int, [C.c_void_p, C.c_int * 6]),
    "mm_plan_device_bytes": (C.c_longlong, [C.c_void_p]),
    "mm_fields": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double] + [C.c_void_p] * 6 + [C.c_void_p]),
    "mm_torque": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_void_p, C.c_void_p]),
    "mm_solver_am12_tolerances": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "mm_solver_init": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]),
    "mm_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "mm_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "mm_set_time": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "mm_set_thermal_dt": (C.c_int, [C.c_void_p, C.c_double]),
    "mm_step": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mm_run": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "mm_steps": (C.c_int, [C.c_void_p, C.c_longlong, C.c_void_p]),
    "mm_run_until_maxtorque": (C.c_int, [C.c_void_p, C.c_double, C.c_longlong, C.c_void_p]),
    "mm_queue_attempts": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "mm_get_stats": (C.c_int, [C.c_void_p, C.POINTER(MMStats), C.c_void_p]),
    "mm_maxtorque": (C.c_int, [C.c_void_p, DP, C.c_void_p]),
    "mm_average": (C.c_int, [C.c_void_p, C.c_double * 3, C.c_void_p]),
    "mm_energy": (C.c_int, [C.c_void_p, C.c_double * 5, C.c_void_p]),
    "mm_plan_launch_count": (C.c_longlong, [C.c_void_p]),
    "mm_profile_eval": (C.c_int, [C.c_void_p, C.c_int, DP, C.POINTER(C.c_int), C.c_void_p]),
    "mm_plan_geometry": (C.c_int, [C.c_void_p, C.c_int * 12]),
    "mm_average_noalloc": (C.c_int, [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]),
    "mm_set_table": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_conv3x3": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_set_wait_limit": (C.c_int, [C.c_longlong]),
    "mm_nn_conv3x3_wgrad_tc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                         C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_nn_set_conv_kernel": (C.c_int, [C.c_int]),
    "mm_nn_conv3x3_tc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_nn_conv3x3_wgrad": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_pool": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                             C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_upsample": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_relu_bwd": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_longlong,
                                 C.c_void_p]),
    "mm_nn_relu_bias_bwd": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_longlong, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_nn_bias_grad": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p]),
    "mm_nn_mse": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_void_p, C.c_int,
                            C.c_void_p, C.c_void_p]),
    "mm_nn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_float,
                             C.c_float, C.c_float, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_nn_flip": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "mm_nn_output_state": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p,
                                     C.c_void_p]),
    "mm_nn_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_nn_to_bf16": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "mm_tabulate": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "mm_autosave": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "mm_autosave_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_write_field": (C.c_int, [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_int * 3, C.c_double * 3, C.c_double,
                                 C.c_char_p, C.c_char_p]),
    "mm_read_field": (C.c_int, [C.c_char_p, C.c_void_p, C.c_longlong, C.POINTER(C.c_int), C.c_int * 3,
                                C.POINTER(C.c_double)]),
    "mm_crc64_iso": (C.c_uint64, [C.c_void_p, C.c_size_t]),
    "mm_save_async": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, C.c_void_p]),
    "mm_save_wait": (C.c_int, [C.c_void_p]),
    "mm_tabulate_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_plan_create_batch": (C.c_int, [C.POINTER(MMProblem), C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mm_plan_demag_kernel": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_demag_tensor": (C.c_int, [C.c_int * 3, C.c_double * 3, C.c_int * 3, C.c_int, C.c_int, C.c_void_p,
                                  C.c_void_p]),
    "mm_plan_tiles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_autotune_runs": (C.c_longlong, []),
    "mm_plan_set_tiles": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mm_plan_nsim": (C.c_int, [C.c_void_p]),
    "mm_batch_set_sims": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mm_batch_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_batch_cancel": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mm_batch_restart": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_longlong, C.c_void_p]),
    "mm_batch_drive": (C.c_int, [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p]),
    "mm_batch_run_until_maxtorque": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p]),
    "mm_batch_maxtorque": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_batch_average": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_batch_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "mm_ensemble_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mm_ensemble_destroy": (C.c_int, [C.c_void_p]),
    "mm_ensemble_steps": (C.c_int, [C.c_void_p, C.c_longlong, C.c_void_p]),
    "mm_ensemble_run": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "mm_ensemble_launch_count": (C.c_longlong, [C.c_void_p]),
}


def lib():
    """Load libmm_b200.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python 2_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != MM_OK:
        msg = lib().mm_last_error().decode(errors="replace")
        raise MMError(rc, msg)
    return rc


MASK_SCALARS = ["msat", "aex", "alpha", "ku", "temp", "xi", "zl_pol", "sl_pol", "lambda",
                "eps_prime", "t_fl"]
MASK_VECTORS = ["anisu", "bext", "j", "p"]


def make_problem(d, masks=None):
    """Fill an MMProblem from a dict (same keys as the oracle's problem dict);
    `masks` maps mask names to device pointers (ints) or, for vectors, 3-lists."""
    s = MMProblem()
    s.n[:] = [int(x) for x in d["n"]]
    s.cell[:] = [float(x) for x in d["cell"]]
    s.pbc[:] = [int(x) for x in d.get("pbc", (0, 0, 0))]
    for k in ["demag", "exchange", "anis", "zeeman", "thermal", "zhangli", "slonczewski"]:
        setattr(s, k, int(d.get(k, 0)))
    s.demag_accuracy = int(d.get("demag_accuracy", 6))
    s.demag_exchange = int(d.get("demag_exchange", 0))
    s.demag_tensor = TENSORS[d.get("demag_tensor", "arne")] if isinstance(d.get("demag_tensor", 0), str) \
        else int(d.get("demag_tensor", 0))
    for k, dv in [("msat", 8e5), ("aex", 1.3e-11), ("alpha", 0.02), ("gamma", 2.211e5), ("ku", 0.0),
                  ("temp", 0.0), ("zl_pol", 1.0), ("xi", 0.05), ("sl_pol", 1.0), ("eps_prime", 0.0),
                  ("t_fl", 0.0)]:
        setattr(s, k, float(d.get(k, dv)))
    s.lambda_ = float(d.get("lambda", 1.0))
    s.seed = int(d.get("seed", 0))
    s.bext[:] = [float(x) for x in d.get("bext", (0, 0, 0))]
    s.anisu[:] = [float(x) for x in d.get("anisu", (0, 0, 1))]
    s.j[:] = [float(x) for x in d.get("j", (0, 0, 0))]
    s.p[:] = [float(x) for x in d.get("p", (0, 0, 1))]
    masks = masks or {}
    for k in MASK_SCALARS:
        if masks.get(k) is not None:
            setattr(s, k + "_mask", int(masks[k]))
    for k in MASK_VECTORS:
        v = masks.get(k)
        if v is not None:
            arr = getattr(s, k + "_mask")
            for c in range(3):
                if v[c] is not None:
                    arr[c] = int(v[c])
    return s
