"""The epilogue that forms the next stage state also writes its R2C rows, so that the next
evaluation of the attempt starts at its column pass (RK23 / RK45 stages, Heun's
corrector), and the combine that forms an attempt's first stage state (RK23 / RK45; the
Euler predictor of RK12) writes them too.  It packs, transforms and post-processes the rows exactly as the separate row
pass does, so the stepped trajectory must be bit-identical to the one of a plan created
with MM_EPI_R2C=0 (every evaluation with its own row pass), and each fused attempt must
launch fewer kernels."""
import numpy as np
import pytest

from helpers import rand_m

pytestmark = pytest.mark.gpu


def _run(monkeypatch, fused, prob, m0, solver, steps, masks=None, sims=None, masks_per_sim=False, thermal_dt=None,
         **solver_kw):
    from mumax2 import Plan
    if fused:
        monkeypatch.delenv("MM_EPI_R2C", raising=False)
    else:
        monkeypatch.setenv("MM_EPI_R2C", "0")
    monkeypatch.setenv("MM_AUTOTUNE", "0")
    p = Plan(prob, masks=masks, sims=sims, masks_per_sim=masks_per_sim)
    p.solver(solver, **solver_kw)
    if thermal_dt:
        p.set_thermal_dt(thermal_dt)
    p.set_state(m0)
    l0 = p.launch_count()
    p.steps(steps)
    out = (p.get_state(), p.stats() if sims is None else None, p.launch_count() - l0)
    p.close()
    return out


def _compare(monkeypatch, *args, **kw):
    a = _run(monkeypatch, False, *args, **kw)
    b = _run(monkeypatch, True, *args, **kw)
    assert np.array_equal(a[0], b[0])
    if a[1] is not None:
        for k in ("step", "badsteps", "attempts", "evals", "t", "dt"):
            assert a[1][k] == b[1][k], k
    assert b[2] < a[2], (a[2], b[2])
    return a, b


@pytest.mark.parametrize("solver", ["rk23", "rk45", "rk12"])
def test_film3d_masked(monkeypatch, solver):
    """3-D film with a non-binary Msat mask, anisotropy and Zeeman; row pass, y, z and
    inverse passes; adaptive steps with rejections allowed."""
    import oracle as O
    n = (8, 32, 64)
    rng = np.random.default_rng(5)
    mask = rng.uniform(0.3, 1.0, size=n[0] * n[1] * n[2]).astype(np.float32)
    mask[rng.random(mask.size) < 0.1] = 0.0
    prob = O.full_desc(n=n, cell=(2e-9, 4e-9, 4e-9), demag=1, exchange=1, anis=1, zeeman=1, msat=9e5, aex=1.3e-11,
                       ku=3e5, anisu=(0.6, 0.0, 0.8), bext=(0.01, 0.0, 0.02), alpha=0.05, masks={"msat": mask})
    m0 = rand_m(n, seed=11)
    a, b = _compare(monkeypatch, prob, m0, solver, 25, masks={"msat": mask}, dt=1e-13, maxerr=1e-5)
    assert a[1]["attempts"] >= 25


def test_single_layer_rk45(monkeypatch):
    """Single-layer film (row pass, y transform with the kernel multiply, C2R + epilogue)."""
    import oracle as O
    n = (1, 64, 128)
    prob = O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, zeeman=1, msat=8e5, aex=1.3e-11,
                       bext=(0.0, 0.02, 0.01), alpha=0.02)
    _compare(monkeypatch, prob, rand_m(n, seed=2, kind="near_x"), "rk45", 30, dt=1e-13, maxerr=1e-5)


def test_periodic_axes(monkeypatch):
    """A periodic x axis (no padding: every float of the row is input) and a periodic y
    axis (the rows keep their zero half)."""
    import oracle as O
    for n, pbc in (((4, 16, 32), (0, 0, 1)), ((1, 16, 32), (0, 1, 0))):
        prob = O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), pbc=pbc, demag=1, exchange=1, msat=8e5, aex=1.3e-11,
                           alpha=0.1)
        _compare(monkeypatch, prob, rand_m(n, seed=7), "rk23", 15, dt=1e-13, maxerr=1e-5)


def test_demag_exchange_kernel(monkeypatch):
    """demagexch convolves m itself (no Msat mask on the convolution input)."""
    import oracle as O
    n = (2, 32, 32)
    mask = np.ones(n[0] * n[1] * n[2], np.float32)
    mask[: mask.size // 3] = 0.5
    prob = O.full_desc(n=n, cell=(3e-9, 3e-9, 3e-9), demag=1, exchange=0, msat=8e5, aex=1.3e-11, alpha=0.1,
                       demag_exchange=1, demag_accuracy=8, masks={"msat": mask})
    _compare(monkeypatch, prob, rand_m(n, seed=8), "rk23", 15, masks={"msat": mask}, dt=1e-14, maxerr=1e-5)


def test_heun_thermal(monkeypatch):
    """Heun (fixed step) with thermal noise: the corrector starts at its column pass."""
    import oracle as O
    n = (1, 32, 32)
    prob = O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, zeeman=1, thermal=1, temp=300.0, seed=17,
                       msat=7e5, aex=1.2e-11, alpha=0.05, bext=(0.0, 0.02, 0.01))
    a, b = _compare(monkeypatch, prob, rand_m(n, seed=4, kind="near_x"), "heun", 40, dt=5e-14,
                    thermal_dt=5e-14)
    assert a[1]["step"] == 40


def test_batched_relax_plan(monkeypatch):
    """Batched plan of single-layer films with per-simulation Msat masks and scalars
    (the relaxation pools), RK23."""
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(8, seed=3)
    m0 = np.concatenate([rand_m(problem["n"], seed=s) for s in range(8)])
    _compare(monkeypatch, problem, m0, "rk23", 20, masks={"msat": np.concatenate(masks)}, sims=sims,
             masks_per_sim=True, dt=1e-14, maxerr=1e-6)
