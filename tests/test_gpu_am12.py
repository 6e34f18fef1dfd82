"""solver/am12 (solve_am01.go:46-301) on the device against the FP64 oracle's restatement.

The fixed-point iterations and the step-size decisions take the same branches in FP32 as
in FP64 on these runs, so step and bad-step counts agree exactly and m to 1e-4.
"""
import numpy as np
import pytest

from helpers import rand_m

pytestmark = pytest.mark.gpu

FILM = dict(n=(1, 16, 32), cell=(3e-9, 3.90625e-9, 3.90625e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
            aex=1.3e-11, alpha=0.05, bext=(0.0, 4.3e-3, -24.6e-3))


@pytest.mark.parametrize("n,kind,dur", [((1, 16, 32), "near_x", 5e-12), ((2, 8, 16), "sphere", 2e-12)])
def test_am12_trajectory(n, kind, dur):
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(**dict(FILM, n=n))
    o = O.Oracle(prob)
    m0 = rand_m(n, seed=8, kind=kind)
    r = O.OracleRun(o, m0.copy(), solver="am12", dt=1e-15)
    g = Plan(prob)
    g.solver("am12", dt=1e-15)
    g.set_state(m0)
    r.run(dur)
    g.run(dur)
    st = g.stats()
    mo = o.normalize(r.m.copy())
    err = np.abs(g.get_state() - mo).max()
    print("am12", n, st["step"], r.st.step, st["t"], r.st.t, err)
    assert abs(st["step"] - r.st.step) <= max(1, 0.01 * r.st.step)
    assert st["t"] == pytest.approx(r.st.t, rel=1e-3)
    assert err < 1e-4
    assert st["iterations"] >= 3


def test_am12_batched_matches_single():
    import oracle as O
    from mumax2 import Plan
    base = O.full_desc(**FILM)
    sims = [dict(msat=8e5, alpha=0.05), dict(msat=5e5, alpha=0.2)]
    N = 512
    m = np.concatenate([rand_m(FILM["n"], seed=20 + b, kind="near_x") for b in range(2)])
    g = Plan(base, sims=sims)
    g.solver("am12", dt=1e-15)
    g.set_state(m)
    g.run(3e-12)
    st = g.batch_stats()
    mb = g.get_state()
    for b, sim in enumerate(sims):
        q = dict(base)
        q.update(sim)
        s = Plan(q)
        s.solver("am12", dt=1e-15)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.run(3e-12)
        assert st[b]["step"] == s.stats()["step"]
        assert np.abs(mb[3 * N * b:3 * N * (b + 1)] - s.get_state()).max() < 1e-6


def test_am12_script_module():
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(32, 16, 1)
    mm.setcellsize(3.90625e-9, 3.90625e-9, 3e-9)
    mm.load("micromagnetism")
    mm.load("solver/am12") if False else None
    mm.reset()
    mm.setgridsize(32, 16, 1)
    mm.setcellsize(3.90625e-9, 3.90625e-9, 3e-9)
    for mod in ["demag", "exchange6", "llg", "zeeman", "solver/am12", "maxtorque"]:
        mm.load(mod)
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 1.0)
    mm.setv("dt", 1e-15)
    mm.setarray("m", [[[[1]]], [[[0.1]]], [[[0]]]])
    mm.run_until_smaller("maxtorque", 1e-3 * mm.gets("gamma") * 8e5)
    assert mm.gets("maxtorque") < 1e-3 * mm.gets("gamma") * 8e5
    assert mm.gets("bdf_iterations") >= 3
    mm.reset()
