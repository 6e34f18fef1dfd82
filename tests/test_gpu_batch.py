"""Batched plans (many simulations of one geometry per launch) and ensembles (several
batched plans stepped from one CUDA graph).

Every simulation of a batch must reproduce the single-simulation plan with the same
scalars: the batch runs the same kernels on the same numbers, so fields agree to 1e-6
relative and trajectories to 1e-6 absolute in m (TOL_SAME).  One simulation per batch
is also checked against the FP64 oracle at the field tolerance (1e-5).
"""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-6
TOL_FIELD = 1e-5

SIMS = [
    dict(msat=8.0e5, aex=1.3e-11, alpha=0.02, bext=(0.0, 0.01, 0.02), ku=0.0, anisu=(1, 0, 0), seed=11),
    dict(msat=4.5e5, aex=6.0e-12, alpha=0.08, bext=(0.03, 0.0, -0.01), ku=2e5, anisu=(0, 0.6, 0.8), seed=12),
    dict(msat=1.1e6, aex=1.9e-11, alpha=0.05, bext=(0.0, -0.02, 0.0), ku=4e5, anisu=(0, 0, 1), seed=13),
]


def _base(n, **kw):
    import oracle as O
    d = dict(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, zeeman=1, anis=1, gamma=2.211e5)
    d.update(kw)
    return O.full_desc(**d)


def _single(base, sim, masks=None):
    from mumax2 import Plan
    q = dict(base)
    q.update(sim)
    return Plan(q, masks=masks or {})


def _batch_m(n, nsim, seed):
    return np.concatenate([rand_m(n, seed + b) for b in range(nsim)])


@pytest.mark.parametrize("n", [(1, 32, 64), (2, 16, 32), (4, 16, 16), (1, 8, 8)])
def test_batch_fields_match_single_and_oracle(n):
    import oracle as O
    from mumax2 import Plan
    base = _base(n)
    g = Plan(base, sims=SIMS)
    assert g.nsim == 3 and g.geometry()["nsim"] == 3
    N = n[0] * n[1] * n[2]
    m = _batch_m(n, 3, 100)
    fb = g.fields(m)
    for b, sim in enumerate(SIMS):
        s = _single(base, sim)
        fs = s.fields(m[3 * N * b:3 * N * (b + 1)])
        for k in ["demag", "ex", "anis", "zee", "eff"]:
            err = rel_err(to_np(fb[k])[3 * N * b:3 * N * (b + 1)], to_np(fs[k]))
            assert err < TOL_SAME, (b, k, err)
    q = dict(base)
    q.update(SIMS[1])
    fo = O.Oracle(q).fields(m[3 * N:6 * N])
    for k in ["demag", "ex", "anis", "zee"]:
        assert rel_err(to_np(fb[k])[3 * N:6 * N], fo[k]) < TOL_FIELD, k


def test_batch_without_demag_matches_single():
    from mumax2 import Plan
    n = (2, 8, 16)
    base = _base(n, demag=0)
    g = Plan(base, sims=SIMS)
    N = n[0] * n[1] * n[2]
    m = _batch_m(n, 3, 7)
    tb, _ = g.torque(m)
    for b, sim in enumerate(SIMS):
        ts, _ = _single(base, sim).torque(m[3 * N * b:3 * N * (b + 1)])
        assert rel_err(to_np(tb)[3 * N * b:3 * N * (b + 1)], to_np(ts)) < TOL_SAME


def test_batch_thermal_heun_fixed_dt_matches_single():
    """Stochastic Heun at fixed dt with per-simulation seeds and temperatures."""
    from mumax2 import Plan
    n = (1, 16, 32)
    base = _base(n, thermal=1, temp=300.0)
    sims = [dict(s, temp=t) for s, t in zip(SIMS, [300.0, 50.0, 600.0])]
    g = Plan(base, sims=sims)
    g.solver("heun", dt=5e-14)
    N = n[0] * n[1] * n[2]
    m = _batch_m(n, 3, 200)
    g.set_state(m)
    g.steps(20)
    mb = g.get_state()
    st = g.batch_stats()
    for b, sim in enumerate(sims):
        s = _single(base, sim)
        s.solver("heun", dt=5e-14)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.steps(20)
        assert np.abs(mb[3 * N * b:3 * N * (b + 1)] - s.get_state()).max() < TOL_SAME, b
        assert st[b]["step"] == 20 and st[b]["t"] == pytest.approx(20 * 5e-14)
    # different seeds and temperatures give different noise
    assert np.abs(mb[:3 * N] - mb[3 * N:6 * N]).max() > 1e-3


@pytest.mark.parametrize("solver", ["rk12", "rk23", "rk45"])
def test_batch_adaptive_per_simulation_control(solver):
    """Each simulation keeps its own dt, error and accept/reject decisions."""
    from mumax2 import Plan
    n = (1, 16, 32)
    base = _base(n)
    g = Plan(base, sims=SIMS)
    g.solver(solver, dt=1e-15, maxerr=1e-4)
    N = n[0] * n[1] * n[2]
    m = _batch_m(n, 3, 300)
    g.set_state(m)
    g.run(5e-12)
    mb = g.get_state()
    st = g.batch_stats()
    assert len({s["step"] for s in st}) > 1  # the simulations took different numbers of steps
    for b, sim in enumerate(SIMS):
        s = _single(base, sim)
        s.solver(solver, dt=1e-15, maxerr=1e-4)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.run(5e-12)
        ss = s.stats()
        assert st[b]["step"] == ss["step"] and st[b]["badsteps"] == ss["badsteps"], (b, st[b], ss)
        assert st[b]["t"] == pytest.approx(ss["t"], rel=1e-12)
        assert np.abs(mb[3 * N * b:3 * N * (b + 1)] - s.get_state()).max() < TOL_SAME, b


def test_batch_relax_until_maxtorque_and_reductions():
    """run_until_maxtorque stops each simulation on its own; finished ones stay frozen."""
    from mumax2 import Plan
    n = (1, 16, 16)
    base = _base(n)
    sims = [dict(s, alpha=1.0) for s in SIMS]
    g = Plan(base, sims=sims)
    # an explicit solver relaxes only down to a torque floor set by its error tolerance:
    # 1e-6 takes these films below the threshold in a few hundred to a few thousand steps
    g.solver("rk23", dt=1e-14, maxerr=1e-6)
    N = n[0] * n[1] * n[2]
    m = np.concatenate([rand_m(n, 400 + b, kind="near_x") for b in range(3)])
    g.set_state(m)
    thr = 1e-4 * 2.211e5 * np.array([s["msat"] for s in sims])
    # one threshold for all: the smallest, so that every simulation must reach it
    g.run_until_maxtorque(float(thr.min()), max_steps=20000)
    mb = g.get_state()
    st = g.batch_stats()
    mt = g.batch_maxtorque()
    av = g.batch_average()
    en = g.batch_energy()
    for b, sim in enumerate(sims):
        assert st[b]["maxtorque"] < thr.min(), (b, st[b])
        s = _single(base, sim)
        s.solver("rk23", dt=1e-14, maxerr=1e-6)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.run_until_maxtorque(float(thr.min()), max_steps=20000)
        assert st[b]["step"] == s.stats()["step"], b
        assert np.abs(mb[3 * N * b:3 * N * (b + 1)] - s.get_state()).max() < TOL_SAME
        assert mt[b] == pytest.approx(s.maxtorque(), rel=1e-5)
        assert np.allclose(av[b], s.average(), atol=1e-6)
        es = s.energy()
        assert en[b][4] == pytest.approx(es["E"], rel=1e-5)
    with pytest.raises(Exception):
        g.stats()  # single-simulation query on a batched plan


def test_batch_masks_per_simulation():
    from mumax2 import Plan
    n = (1, 16, 16)
    base = _base(n)
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(5)
    masks = [(rng.uniform(size=N) > 0.3).astype(np.float32) for _ in range(3)]
    g = Plan(base, masks={"msat": np.concatenate(masks)}, sims=SIMS, masks_per_sim=True)
    m = _batch_m(n, 3, 500)
    tb, mn = g.torque(m)
    for b, sim in enumerate(SIMS):
        ts, ms = _single(base, sim, masks={"msat": masks[b]}).torque(m[3 * N * b:3 * N * (b + 1)])
        assert rel_err(to_np(tb)[3 * N * b:3 * N * (b + 1)], to_np(ts)) < TOL_SAME
        assert np.abs(to_np(mn)[3 * N * b:3 * N * (b + 1)] - to_np(ms)).max() < TOL_SAME


def test_ensemble_of_grid_classes_matches_plans_alone():
    """Two batched plans of different grids stepped from one graph = each stepped alone."""
    from mumax2 import Ensemble, Plan
    grids = [(1, 16, 16), (2, 16, 32)]
    states, plans = [], []
    for i, n in enumerate(grids):
        base = _base(n, thermal=1, temp=300.0)
        sims = [dict(s, temp=300.0, seed=50 + 10 * i + b) for b, s in enumerate(SIMS)]
        p = Plan(base, sims=sims)
        p.solver("heun", dt=5e-14)
        m = _batch_m(n, 3, 600 + i)
        p.set_state(m)
        plans.append((p, base, sims, m))
    ens = Ensemble([p for p, *_ in plans], attempts=8)
    ens.steps(30)
    assert ens.launch_count() > 0
    for p, base, sims, m in plans:
        got = p.get_state()
        assert all(s["step"] == 30 for s in p.batch_stats())
        alone = Plan(base, sims=sims)
        alone.solver("heun", dt=5e-14)
        alone.set_state(m)
        alone.steps(30)
        assert np.abs(got - alone.get_state()).max() < TOL_SAME


def test_batch_per_simulation_thresholds():
    """mm_batch_run_until_maxtorque: each simulation stops at its own threshold."""
    from mumax2 import Plan
    n = (1, 16, 16)
    base = _base(n)
    sims = [dict(s, alpha=1.0) for s in SIMS]
    g = Plan(base, sims=sims)
    g.solver("rk23", dt=1e-14, maxerr=1e-6)
    N = n[0] * n[1] * n[2]
    m = np.concatenate([rand_m(n, 700 + b, kind="near_x") for b in range(3)])
    g.set_state(m)
    thr = np.array([1e-4 * 2.211e5 * s["msat"] for s in sims])
    g.batch_run_until_maxtorque(thr, max_steps=50000)
    st = g.batch_stats()
    mb = g.get_state()
    for b, sim in enumerate(sims):
        assert st[b]["maxtorque"] < thr[b], (b, st[b])
        s = _single(base, sim)
        s.solver("rk23", dt=1e-14, maxerr=1e-6)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.run_until_maxtorque(float(thr[b]), max_steps=50000)
        assert st[b]["step"] == s.stats()["step"], b
        assert np.abs(mb[3 * N * b:3 * N * (b + 1)] - s.get_state()).max() < TOL_SAME


def test_continuous_batching_slots_restart_independently():
    """mm_batch_restart / mm_batch_drive: a finished slot takes a new problem while the
    other slots keep running; every problem ends exactly as it does alone."""
    from mumax2 import Plan
    n = (1, 16, 16)
    base = _base(n)
    N = n[0] * n[1] * n[2]
    probs = [dict(s, alpha=1.0) for s in SIMS] + [dict(SIMS[0], alpha=1.0, msat=6e5)]
    ms = [rand_m(n, 800 + q, kind="near_x") for q in range(4)]
    thr = [1e-4 * 2.211e5 * p["msat"] * 3 for p in probs]
    g = Plan(base, sims=probs[:2])
    g.solver("rk23", dt=1e-14, maxerr=1e-6)
    g.batch_restart([0, 1], np.stack(ms[:2]), thr[:2], sims=probs[:2])
    slot_job, nxt, results = [0, 1], 2, {}
    while len(results) < 4:
        g.batch_drive(target_active=1 if nxt < 4 else 0)
        st = g.batch_stats()
        state = g.get_state()
        for b in range(2):
            q = slot_job[b]
            if q >= 0 and st[b]["done"]:
                results[q] = (st[b]["step"], state[3 * N * b:3 * N * (b + 1)].copy())
                slot_job[b] = -1
                if nxt < 4:
                    g.batch_restart([b], ms[nxt][None, :], [thr[nxt]], sims=[probs[nxt]])
                    slot_job[b] = nxt
                    nxt += 1
    for q in range(4):
        s = _single(base, probs[q])
        s.solver("rk23", dt=1e-14, maxerr=1e-6)
        s.set_state(ms[q])
        s.run_until_maxtorque(thr[q], max_steps=50000)
        assert results[q][0] == s.stats()["step"], q
        assert np.abs(results[q][1] - s.get_state()).max() < TOL_SAME, q
