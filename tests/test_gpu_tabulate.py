"""Autotabulate recorded on the device (AutoTabulate, notify_tabulate.go:23-28): rows are
written by the step's own kernels with no host synchronisation.  Checked against the
oracle stepping the same solver and applying the reference's record rule after every
accepted step; <m> within the trajectory tolerance (2e-4), times to 1e-9 relative."""
import numpy as np
import pytest

from helpers import rand_m

pytestmark = pytest.mark.gpu

FILM = dict(n=(1, 16, 32), cell=(3e-9, 3.90625e-9, 3.90625e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
            aex=1.3e-11, alpha=0.05, bext=(0.0, 4.3e-3, -24.6e-3))


def _oracle_rows(problem, m0, solver, dt, maxerr, period, duration):
    import oracle as O
    o = O.Oracle(O.full_desc(**problem))
    r = O.OracleRun(o, m0, solver=solver, dt=dt, maxerr=maxerr)
    rows, count = [], 0
    while r.st.t < duration:
        r.step()
        if r.st.t - count * period >= period:
            rows.append((r.st.t, *o.average(o.normalize(r.m.copy()))))
            count += 1
    return np.array(rows)


@pytest.mark.parametrize("solver,dt,maxerr", [("rk12", 1e-15, 1e-4), ("rk23", 1e-15, 1e-5), ("heun", 5e-14, 1e-3)])
def test_device_rows_match_oracle(solver, dt, maxerr):
    import oracle as O
    from mumax2 import Plan
    g = Plan(O.full_desc(**FILM))
    m0 = rand_m(FILM["n"], seed=4, kind="near_x")
    g.solver(solver, dt=dt, maxerr=maxerr)
    g.set_state(m0)
    period = 1e-12
    g.tabulate(period, capacity=256)
    g.run(2e-11)
    rows = g.tabulate_read()[0]
    ref = _oracle_rows(FILM, m0, solver, dt, maxerr, period, 2e-11)
    assert len(rows) == len(ref) and len(rows) >= 15
    assert np.allclose(rows[:, 0], ref[:, 0], rtol=1e-9)
    assert np.abs(rows[:, 1:4] - ref[:, 1:4]).max() < 2e-4
    assert (np.diff(rows[:, 6]) > 0).all()
    # reading empties the table
    assert len(g.tabulate_read()[0]) == 0
    g.run(2e-12)
    assert len(g.tabulate_read()[0]) >= 1


def test_batched_rows_match_single_plans():
    import oracle as O
    from mumax2 import Plan
    base = O.full_desc(**FILM)
    sims = [dict(msat=8e5, alpha=0.05, seed=1), dict(msat=5e5, alpha=0.1, seed=2)]
    g = Plan(base, sims=sims)
    N = 512
    m = np.concatenate([rand_m(FILM["n"], seed=10 + b, kind="near_x") for b in range(2)])
    g.solver("rk23", dt=1e-15, maxerr=1e-5)
    g.set_state(m)
    g.tabulate(2e-12, capacity=64)
    g.run(1e-11)
    rows = g.tabulate_read()
    for b, sim in enumerate(sims):
        q = dict(base)
        q.update(sim)
        s = Plan(q)
        s.solver("rk23", dt=1e-15, maxerr=1e-5)
        s.set_state(m[3 * N * b:3 * N * (b + 1)])
        s.tabulate(2e-12, capacity=64)
        s.run(1e-11)
        r1 = s.tabulate_read()[0]
        assert rows[b].shape == r1.shape
        assert np.abs(rows[b] - r1).max() <= 1e-12 * np.abs(r1).max()


def test_full_table_counts_lost_rows():
    import oracle as O
    from mumax2 import Plan
    g = Plan(O.full_desc(**FILM))
    g.solver("rk23", dt=1e-15, maxerr=1e-5)
    g.set_state(rand_m(FILM["n"], seed=4, kind="near_x"))
    g.tabulate(1e-13, capacity=4)
    g.run(2e-12)
    rows = g.tabulate_read()[0]
    assert len(rows) == 4 and g.tab_lost[0] > 0


def test_script_autotabulate_file(tmp_path):
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(32, 16, 1)
    mm.setcellsize(3.90625e-9, 3.90625e-9, 3e-9)
    mm.load("micromagnetism")
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 0.05)
    mm.setv("m_maxerror", 1e-4)
    mm.setarray("m", [[[[1]]], [[[0.1]]], [[[0]]]])
    fn = str(tmp_path / "m.txt")
    mm.autotabulate(["t", "<m>"], fn, 2e-12)
    mm.run(1e-11)
    lines = open(fn).read().splitlines()
    assert lines[0] == "#t (s)\t<m>_x ()\t<m>_y ()\t<m>_z ()\t"
    vals = np.array([[float(x) for x in ln.split("\t") if x] for ln in lines[1:]])
    assert len(vals) == 5 and np.all(np.diff(vals[:, 0]) > 0)
    assert np.allclose(vals[-1, 1:], mm.getv("<m>"), atol=1e-3)
    mm.reset()
