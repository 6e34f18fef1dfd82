"""The allocation-free <m> entry point (mm_average_noalloc) against the plan-based one
and against an FP64 numpy mean of the same float32 state.

mm_average_noalloc exists for callers that cannot allocate device memory (code running
inside a CUDA stream capture, engines whose GPU memory is owned by another allocator):
it keeps its block partials in a fixed file-scope device array instead of a plan
workspace.  This file is collected last so that a run stopping at the first failure has
run every other test first; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-6   # both are compensated FP32 sums of unit-vector components, folded in double


def _plan_and_state(n, seed):
    from mumax2 import Plan
    prob = dict(n=n, cell=(2e-9, 3e-9, 3e-9), demag=0, exchange=1, msat=8e5, aex=1.3e-11)
    p = Plan(prob)
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(3, n[0] * n[1] * n[2]))
    m[0] += 0.3   # a non-zero mean
    p.solver("rk23")
    p.set_state(m.ravel())
    return p


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 37, 53), (4, 128, 128)])
def test_noalloc_average_matches_plan_average_twice(n):
    import torch
    from mumax2 import _native as nat
    lib = nat.lib()
    p = _plan_and_state(n, seed=sum(n))
    want = p.average()                          # existing entry point (plan workspace)
    state = p.get_state()
    md = torch.as_tensor(state, device="cuda")   # the same float32 state
    N = n[0] * n[1] * n[2]
    exact = np.asarray(state, dtype=np.float32).astype(np.float64).reshape(3, N).mean(axis=1)
    for call in range(2):                       # two calls in a row share the scratch array
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.mm_average_noalloc(C.c_void_p(md.data_ptr()), N, C.c_void_p(out.data_ptr()), None)
        assert rc == nat.MM_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.abs(got - want).max() <= TOL, (call, got, want)
        assert np.abs(got - exact).max() <= TOL, (call, got, exact)   # FP64 mean of the same floats
    p.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from mumax2 import _native as nat
    lib = nat.lib()
    md = torch.zeros(3, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    big = 2048 * 8192 + 1
    assert lib.mm_average_noalloc(C.c_void_p(md.data_ptr()), big, C.c_void_p(out.data_ptr()), None) == nat.MM_ERR_ARG
    assert b"16777216" in lib.mm_last_error()
    assert lib.mm_average_noalloc(C.c_void_p(md.data_ptr()), 0, C.c_void_p(out.data_ptr()), None) == nat.MM_ERR_ARG
    assert lib.mm_average_noalloc(None, 1, C.c_void_p(out.data_ptr()), None) == nat.MM_ERR_ARG
