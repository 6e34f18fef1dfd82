"""The reference-GPU baseline (oracle/ref_gpu.py: the reference's own libmumax2 kernels
driven by a restatement of its Go RK12 loop, cuFFT for the transforms) against this
repository's fused path on the same problem.  This pins the baseline that bench.py times:
its demag field and torque agree with the fused path to 1e-5 relative (FP32 both; the
reference library uses fast-math intrinsics), and ten RK12 steps from the same state give
the same accepted/rejected step counts and states within 1e-4."""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu

N = (4, 16, 32)
CELL = (2e-9, 4e-9, 4e-9)
PAR = dict(msat=8e5, aex=1.3e-11, alpha=0.1, gamma=2.211e5, ku=5e5, anisu=(1.0, 0.0, 0.0))


def _pair(dt=1e-13, maxerr=1e-5):
    import oracle as O
    import ref_gpu as R
    from mumax2 import Plan
    if not R.available():
        pytest.skip("reference library not built (oracle/build_ref.sh)")
    prob = O.full_desc(n=N, cell=CELL, demag=1, exchange=1, anis=1, zeeman=0, **PAR)
    ours = Plan(prob)
    ref = R.RefPath(N, CELL, PAR["msat"], PAR["aex"], PAR["alpha"], PAR["gamma"], PAR["ku"], PAR["anisu"],
                    ours.demag_kernel(), dt=dt, maxerr=maxerr)
    return ours, ref


def test_reference_path_fields_match():
    import ref_gpu as R
    ours, ref = _pair()
    m = rand_m(N, seed=5)
    ref.set_state(m)
    ref.evaluate()
    f = ours.fields(m)
    hd = to_np(ref.B).ravel() / R.MU0
    assert rel_err(hd, to_np(f["demag"])) < 1e-5
    assert rel_err(to_np(ref.Hex).ravel(), to_np(f["ex"])) < 1e-5
    assert rel_err(to_np(ref.H).ravel(), to_np(f["eff"])) < 1e-5
    t, _ = ours.torque(m)
    assert rel_err(to_np(ref.tau).ravel(), to_np(t)) < 1e-5
    ours.close()


def test_reference_path_rk12_trajectory_matches():
    ours, ref = _pair()
    m = rand_m(N, seed=6)
    ours.solver("rk12", dt=1e-13, maxerr=1e-5)
    ours.set_state(m)
    ref.set_state(m)
    ours.steps(10)
    for _ in range(10):
        ref.step()
    st = ours.stats()
    assert st["step"] == ref.step_count and st["badsteps"] == ref.bad_steps
    assert np.abs(ours.get_state() - ref.state()).max() < 1e-4
    ours.close()
