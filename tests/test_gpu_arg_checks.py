"""The Python plan refuses state, threshold and scalar arrays of the wrong size before
anything reaches the library (which reads exactly 3N floats per simulation from the
pointers it is given), and the library refuses slots out of range."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batched(nsim=4):
    from mumax2 import Plan
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(nsim, seed=2)
    p = Plan(problem, masks={"msat": np.concatenate(masks)}, sims=sims, masks_per_sim=True)
    p.solver("rk23", dt=1e-14, maxerr=1e-6)
    return p, problem, sims


def test_state_sizes_are_checked():
    import torch
    from mumax2 import workloads as W
    p, problem, sims = _batched()
    n = problem["n"]
    good = W.cold_state(n, p.nsim)
    p.set_state(good)
    for bad in (good[:-1], np.concatenate([good, good[:3]]), good[:3 * p.N]):
        with pytest.raises(ValueError):
            p.set_state(bad)
        with pytest.raises(ValueError):
            p.torque(bad)
        with pytest.raises(ValueError):
            p.fields(bad)
    with pytest.raises(ValueError):
        p.set_state(torch.as_tensor(good[:-5], device="cuda"))
    p.close()


def test_batch_restart_sizes_are_checked():
    import torch
    from mumax2 import _native as nat
    from mumax2 import workloads as W
    p, problem, sims = _batched()
    cold = W.cold_state(problem["n"], 1)
    thr = np.full(2, 1.0)
    with pytest.raises(ValueError):           # one scalar per slot instead of a state
        p.batch_restart([0, 1], np.array([cold[0], cold[0]]), thr)
    with pytest.raises(ValueError):           # a device tensor one state short
        p.batch_restart([0, 1], torch.as_tensor(cold, device="cuda"), thr)
    with pytest.raises(ValueError):           # thresholds do not match the slots
        p.batch_restart([0, 1], np.stack([cold, cold]), np.full(3, 1.0))
    with pytest.raises(ValueError):
        p.batch_restart([0, 1], np.stack([cold, cold]), thr, sims=sims[:1])
    with pytest.raises(nat.MMError):          # the library checks the slot range
        p.batch_restart([0, p.nsim], np.stack([cold, cold]), thr)
    with pytest.raises(ValueError):
        p.set_sims(sims[:2])
    with pytest.raises(ValueError):
        p.batch_run_until_maxtorque(np.ones(p.nsim + 1))
    p.batch_restart([0, 1], np.stack([cold, cold]), thr)   # the right sizes still work
    p.close()


def test_transform_sizes_with_large_prime_factors_are_refused():
    """Padded sizes whose prime factors are at most 31 are transformed (mixed radix);
    others (here L1 = 2 x 37) are refused with a message naming the size."""
    from mumax2 import Plan
    from mumax2 import _native as nat
    with pytest.raises(nat.MMError) as ei:
        Plan(dict(n=(1, 37, 8), cell=(3e-9, 3e-9, 3e-9), demag=1, msat=8e5))
    assert "74" in str(ei.value)
    Plan(dict(n=(1, 31, 8), cell=(3e-9, 3e-9, 3e-9), demag=1, msat=8e5)).close()   # 62 = 2 x 31 is served
