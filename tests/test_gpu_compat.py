"""GPU parity of the libmumax2-compatible entry points.

Each compat symbol of libmm_b200.so is called through its C-ABI with the same device
inputs as
  (a) the reference's own libmumax2 built for sm_100a from its sources (oracle/_ref,
      with the reference's --use_fast_math), when that library is present, and
  (b) the FP64 oracle, for the physics kernels.
Tolerance: 2e-6 relative (max |difference| / max |value|) against the reference
library (both FP32; the reference uses fast-math intrinsics), 1e-5 against the oracle.
"""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import rand_m, rel_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libmumax2_ref.so")
TOL_REF = 2e-6


def _libs():
    import torch
    from mumax2 import _native as nat
    ours = nat.lib()
    ours.setUsedGPUs((C.c_int * 1)(torch.cuda.current_device()), 1)
    libs = [("b200", ours)]
    if os.path.exists(REF_LIB):
        import ref_gpu
        libs.append(("ref", ref_gpu.ref_lib()))
    return libs


_LIBS = None


def libs():
    global _LIBS
    if _LIBS is None:
        _LIBS = _libs()
    return _LIBS


_KEEP = []


def dev(a):
    """Device copy of `a`, kept alive until the end of the test (the kernels run
    asynchronously: a temporary freed before the launch would hand its memory to the
    next allocation)."""
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")
    _KEEP.append(t)
    return t


@pytest.fixture(autouse=True)
def _release_buffers():
    yield
    import torch
    torch.cuda.synchronize()
    _KEEP.clear()


def pp(t):
    """float** of one device part (NULL part for None)."""
    return (C.c_void_p * 1)(t.data_ptr() if t is not None else None)


STREAM = (C.c_void_p * 1)(None)
F = C.c_float
I = C.c_int


def run_all(fn):
    """fn(lib) -> list of output tensors; returns {libname: [numpy arrays]}."""
    import torch
    out = {}
    for name, L in libs():
        res = fn(L)
        torch.cuda.synchronize()
        out[name] = [r.cpu().numpy().astype(np.float64) for r in res]
    from mumax2 import _native as nat
    assert nat.lib().mm_compat_last_status() == 0
    return out


def check_vs_ref(out, tol=TOL_REF):
    if "ref" not in out:
        pytest.skip("reference libmumax2 (oracle/_ref) not built")
    for a, b in zip(out["b200"], out["ref"]):
        err = rel_err(a, b)
        assert err < tol, err


def test_torque_compat():
    n = (2, 8, 12)
    N = 192
    m = rand_m(n, 1).reshape(3, N)
    h = np.random.default_rng(2).normal(size=(3, N)) * 1e5
    alpha = np.random.default_rng(3).uniform(0.5, 1.5, N)

    def fn(L):
        md = [dev(m[c]) for c in range(3)]
        hd = [dev(h[c]) for c in range(3)]
        t = [dev(np.zeros(N)) for _ in range(3)]
        L.torqueAsync(*[pp(x) for x in t], *[pp(x) for x in md], *[pp(x) for x in hd], pp(dev(alpha)), F(0.1),
                      STREAM, I(N))
        return t
    out = run_all(fn)
    check_vs_ref(out)


@pytest.mark.parametrize("n,pbc,masked", [((3, 5, 7), (0, 0, 0), True), ((4, 6, 8), (1, 0, 1), False),
                                          ((1, 9, 4), (0, 1, 0), True)])
def test_exchange6_compat(n, pbc, masked):
    import oracle as O
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(4)
    m = rand_m(n, 5).reshape(3, N)
    msat = rng.uniform(0.5, 1.5, N).astype(np.float32) if masked else None
    aex = rng.uniform(0.5, 1.5, N).astype(np.float32) if masked else None
    cell = (2e-9, 3e-9, 4e-9)
    pre = 2 * 1.3e-11 / (4e-7 * np.pi * 8e5)

    def fn(L):
        md = [dev(m[c]) for c in range(3)]
        hd = [dev(np.zeros(N)) for _ in range(3)]
        L.exchange6Async(*[pp(x) for x in hd], *[pp(x) for x in md], pp(dev(msat) if masked else None),
                         pp(dev(aex) if masked else None), F(pre), I(n[0]), I(n[1]), I(n[2]), I(pbc[0]), I(pbc[1]),
                         I(pbc[2]), F(cell[0]), F(cell[1]), F(cell[2]), STREAM)
        return hd
    out = run_all(fn)
    check_vs_ref(out)
    o = O.Oracle(O.full_desc(n=n, cell=cell, pbc=pbc, demag=0, exchange=1, msat=8e5, aex=1.3e-11,
                             masks=dict(msat=msat, aex=aex) if masked else {}))
    ho = o.fields(m.ravel())["ex"]
    assert rel_err(np.concatenate(out["b200"]), ho) < 1e-5


def test_uniaxial_normalize_compat():
    N = 300
    rng = np.random.default_rng(6)
    m = rng.normal(size=(3, N))
    ku = rng.uniform(0, 1, N)
    ms = rng.uniform(0, 1, N)
    ms[:10] = 0
    ux = rng.uniform(-1, 1, N)

    def fn(L):
        md = [dev(m[c]) for c in range(3)]
        hd = [dev(np.zeros(N)) for _ in range(3)]
        L.uniaxialAnisotropyAsync(*[pp(x) for x in hd], *[pp(x) for x in md], pp(dev(ku)), pp(dev(ms)), F(1.3e5),
                                  pp(dev(ux)), F(0.5), pp(None), F(0.3), pp(None), F(0.8), STREAM, I(N))
        L.normalizeAsync(*[pp(x) for x in md], pp(dev(ms)), STREAM, I(N))
        return hd + md
    check_vs_ref(run_all(fn))


def test_add_family_compat():
    N = 1000
    rng = np.random.default_rng(7)
    a, b, c = (rng.normal(size=N) for _ in range(3))

    def fn(L):
        outs = []
        A, B, Cc = dev(a), dev(b), dev(c)
        d = dev(np.zeros(N)); L.addAsync(pp(d), pp(A), pp(B), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.addMaddAsync(pp(d), pp(A), pp(B), pp(Cc), F(0.3), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.maddAsync(pp(d), pp(A), pp(B), F(-1.7), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.maddAsync(pp(d), pp(A), pp(None), F(-1.7), STREAM, I(N)); outs.append(d)
        d = dev(a); L.madd1Async(pp(d), pp(B), F(2.5), STREAM, I(N)); outs.append(d)
        d = dev(a); L.madd2Async(pp(d), pp(B), F(2.5), pp(Cc), F(-0.5), STREAM, I(N)); outs.append(d)
        d = dev(a); L.madd2Async(pp(d), pp(None), F(2.5), pp(Cc), F(-0.5), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.linearCombination2Async(pp(d), pp(A), F(0.2), pp(B), F(0.7), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.linearCombination3Async(pp(d), pp(A), F(0.2), pp(B), F(0.7), pp(Cc), F(-3.0), STREAM, I(N)); outs.append(d)
        d = dev(np.zeros(N)); L.mulAsync(pp(d), pp(A), pp(B), STREAM, I(N)); outs.append(d)
        dx, dy, dz = dev(np.zeros(N)), dev(np.zeros(N)), dev(np.zeros(N))
        L.vecMaddAsync(pp(dx), pp(dy), pp(dz), pp(A), pp(B), pp(Cc), pp(Cc), pp(A), pp(B), F(1.0), F(2.0), F(3.0),
                       STREAM, I(N))
        outs += [dx, dy, dz]
        dx, dy, dz = dev(np.zeros(N)), dev(np.zeros(N)), dev(np.zeros(N))
        L.vecMaddAsync(pp(dx), pp(dy), pp(dz), pp(A), pp(B), pp(Cc), pp(None), pp(None), pp(None), F(1.0), F(2.0),
                       F(3.0), STREAM, I(N))
        outs += [dx, dy, dz]
        d = dev(np.zeros(N)); L.zeroArrayAsync(pp(d), I(N), STREAM); outs.append(d)
        return outs
    out = run_all(fn)
    ref = [a + b, a + 0.3 * (b + c), a - 1.7 * b, a - 1.7, a + 2.5 * b, a + 2.5 * b - 0.5 * c, a + 2.5 - 0.5 * c,
           0.2 * a + 0.7 * b, 0.2 * a + 0.7 * b - 3 * c, a * b, a + c, b + 2 * a, c + 3 * b, a + 1, b + 2, c + 3,
           np.zeros(N)]
    for got, want in zip(out["b200"], ref):
        assert np.abs(got - want).max() < 1e-5
    check_vs_ref(out)


def test_cmadd_kernelmul_copypad_compat():
    rng = np.random.default_rng(8)
    NC = 500
    src = rng.normal(size=2 * NC)
    kern = rng.normal(size=NC)
    M = [rng.normal(size=2 * NC) for _ in range(3)]
    K = [rng.normal(size=NC) for _ in range(6)]
    S = (3, 4, 5)
    D = (6, 8, 10)
    arr = rng.normal(size=2 * 60)

    def fn(L):
        d = dev(rng.normal(size=2 * NC) * 0 + 1.0)
        L.cmaddAsync(pp(d), F(0.5), F(-2.0), pp(dev(kern)), pp(dev(src)), STREAM, I(NC))
        md = [dev(x) for x in M]
        L.kernelMulMicromag3DAsync(*[pp(x) for x in md], *[pp(dev(x)) for x in K], STREAM, I(2 * NC))
        padded = dev(np.zeros(2 * 480))
        L.copyPad3DAsync(pp(padded), I(D[0]), I(D[1]), I(D[2]), pp(dev(arr)), I(S[0]), I(S[1]), I(S[2]), I(2), STREAM)
        back = dev(np.zeros(2 * 60))
        L.copyUnPad3DAsync(pp(back), I(S[0]), I(S[1]), I(S[2]), pp(padded), I(D[0]), I(D[1]), I(D[2]), I(2), STREAM)
        return [d] + md + [padded, back]
    out = run_all(fn)
    assert np.abs(out["b200"][-1] - arr.astype(np.float32)).max() == 0.0
    check_vs_ref(out)


@pytest.mark.parametrize("N", [1000, 4096 * 3, 100003])
def test_partial_reductions_compat(N):
    from mumax2 import _native as nat
    rng = np.random.default_rng(9)
    a, b, c, d, e, f = (rng.normal(size=N).astype(np.float32) for _ in range(6))
    threads = 512
    while N <= threads:
        threads //= 2
    blocks = (N + 2 * threads - 1) // (2 * threads)
    L = nat.lib()
    A, B, Cc, Dd, E, Fd = (dev(x) for x in (a, b, c, d, e, f))
    out = dev(np.zeros(blocks))

    def red(call, how):
        call()
        import torch
        torch.cuda.synchronize()
        return how(out.cpu().numpy().astype(np.float64))
    got = {
        "sum": red(lambda: L.partialSumAsync(pp(A), pp(out), I(blocks), I(threads), I(N), STREAM), np.sum),
        "sdot": red(lambda: L.partialSDotAsync(pp(A), pp(B), pp(out), I(blocks), I(threads), I(N), STREAM), np.sum),
        "max": red(lambda: L.partialMaxAsync(pp(A), pp(out), I(blocks), I(threads), I(N), STREAM), np.max),
        "min": red(lambda: L.partialMinAsync(pp(A), pp(out), I(blocks), I(threads), I(N), STREAM), np.min),
        "maxabs": red(lambda: L.partialMaxAbsAsync(pp(A), pp(out), I(blocks), I(threads), I(N), STREAM), np.max),
        "maxdiff": red(lambda: L.partialMaxDiffAsync(pp(A), pp(B), pp(out), I(blocks), I(threads), I(N), STREAM), np.max),
        "maxsum": red(lambda: L.partialMaxSumAsync(pp(A), pp(B), pp(out), I(blocks), I(threads), I(N), STREAM), np.max),
        "maxn3": red(lambda: L.partialMaxNorm3SqAsync(pp(A), pp(B), pp(Cc), pp(out), I(blocks), I(threads), I(N),
                                                      STREAM), np.max),
        "maxn3d": red(lambda: L.partialMaxNorm3SqDiffAsync(pp(A), pp(B), pp(Cc), pp(Dd), pp(E), pp(Fd), pp(out),
                                                           I(blocks), I(threads), I(N), STREAM), np.max),
    }
    a64, b64, c64, d64, e64, f64 = (x.astype(np.float64) for x in (a, b, c, d, e, f))
    want = {"sum": a64.sum(), "sdot": (a64 * b64).sum(), "max": a64.max(), "min": a64.min(),
            "maxabs": np.abs(a64).max(), "maxdiff": np.abs(a64 - b64).max(), "maxsum": np.abs(a64 + b64).max(),
            "maxn3": (a64 ** 2 + b64 ** 2 + c64 ** 2).max(),
            "maxn3d": ((a64 - d64) ** 2 + (b64 - e64) ** 2 + (c64 - f64) ** 2).max()}
    for k in want:
        scale = np.abs(a64).sum() if k in ("sum", "sdot") else abs(want[k])
        assert abs(got[k] - want[k]) <= 1e-6 * scale + 1e-30, (k, got[k], want[k])


def test_temperature_scale_compat():
    N = 777
    rng = np.random.default_rng(10)
    noise = rng.normal(size=N)
    al, tm, ms = rng.uniform(0.5, 1, N), rng.uniform(0.5, 1, N), rng.uniform(0, 1, N)
    ms[:5] = 0

    def fn(L):
        nd = dev(noise)
        L.temperature_scaleNoise(pp(nd), pp(dev(al)), pp(dev(tm)), F(1e-21), pp(dev(ms)), F(1e-30), STREAM, I(N))
        return [nd]
    check_vs_ref(run_all(fn))


# The reference kernel touches the arrays before its bounds check (zhang-li_torque.cu:145-156),
# so sizes are multiples of its 16x16 thread blocks: every thread it launches is in range.
@pytest.mark.parametrize("n,pbc,j", [((1, 16, 32), (0, 0, 0), (0, 0, 1e12)), ((3, 16, 16), (1, 0, 1), (3e11, 0, -1e12)),
                                     ((2, 16, 32), (0, 1, 0), (0, 1e12, 2e11))])
def test_zhangli_compat(n, pbc, j):
    import oracle as O
    N = n[0] * n[1] * n[2]
    m = rand_m(n, 11).reshape(3, N)
    rng = np.random.default_rng(12)
    msat = (rng.random(N) > 0.1).astype(np.float32)
    cell = (2e-9, 2e-9, 3e-9)
    pred = 0.5 * 9.2740091523e-24 / (1.60217646e-19 * 8.6e5)

    def fn(L):
        md = [dev(m[c]) for c in range(3)]
        s = [dev(np.zeros(N)) for _ in range(3)]
        L.zhangli_async(*[pp(x) for x in s], *[pp(x) for x in md], pp(None), pp(None), pp(None), pp(dev(msat)),
                        pp(None), pp(None), pp(None), F(j[0]), F(j[1]), F(j[2]), F(pred), F(0.05), F(0.02), I(n[0]),
                        I(n[1]), I(n[2]), F(cell[0]), F(cell[1]), F(cell[2]), I(pbc[0]), I(pbc[1]), I(pbc[2]), STREAM)
        return s
    out = run_all(fn)
    check_vs_ref(out, tol=1e-5)
    o = O.Oracle(O.full_desc(n=n, cell=cell, pbc=pbc, demag=0, exchange=0, zhangli=1, j=j, zl_pol=0.5, xi=0.05,
                             alpha=0.02, msat=8.6e5, masks=dict(msat=msat)))
    zl, _ = o.stt(m.ravel())
    assert rel_err(np.concatenate(out["b200"]), zl) < 1e-5


def test_slonczewski_compat():
    # the reference kernel reads and writes before its bounds check
    # (slonczewski_torque.cu:35-51): N is a multiple of its 512-thread blocks
    import oracle as O
    n = (1, 16, 32)
    N = 512
    m = rand_m(n, 13).reshape(3, N)
    rng = np.random.default_rng(14)
    msat = (rng.random(N) > 0.2).astype(np.float32)
    beta = 1.054571726e-34 * 2.211e5 / (4e-7 * np.pi * 1.60217646e-19 * 8e5)

    def fn(L):
        md = [dev(m[c]) for c in range(3)]
        s = [dev(np.zeros(N)) for _ in range(3)]
        L.slonczewski_async(*[pp(x) for x in s], *[pp(x) for x in md], pp(dev(msat)), pp(None), pp(None), pp(None),
                            pp(None), pp(None), pp(None), pp(None), pp(None), pp(None), pp(None), pp(None),
                            F(0.0), F(0.0), F(1.0), F(1e11), F(0.0), F(0.0), F(0.5669 * beta), F(0.1 * beta),
                            F(1.0), F(1.0), F(1.0), F(0.02), F(3e-9), F(2.0), I(N), STREAM)
        return s
    out = run_all(fn)
    check_vs_ref(out, tol=1e-5)
    o = O.Oracle(O.full_desc(n=n, cell=(3e-9, 2e-9, 2e-9), demag=0, exchange=0, slonczewski=1, j=(1e11, 0, 0),
                             p=(0, 0, 1), sl_pol=0.5669, eps_prime=0.1, t_fl=3e-9, alpha=0.02, msat=8e5,
                             masks=dict(msat=msat), **{"lambda": 2.0}))
    _, sl = o.stt(m.ravel())
    assert rel_err(np.concatenate(out["b200"]), sl) < 1e-5
