"""Time-dependent inputs (SetPointwise, api.go:172-190 / update_pointwise.go:30-88)
evaluated on the device at every stage time, against the FP64 oracle's tables.

Fields at a given time agree to the field tolerance (1e-5 relative); trajectories driven
by a field pulse agree to 2e-4 in m with identical step counts, as in the solver tests.
"""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu

FILM = dict(n=(1, 16, 32), cell=(3e-9, 3.90625e-9, 3.90625e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
            aex=1.3e-11, alpha=0.05, bext=(0.0, 0.0, 0.0))
# a 50 ps field pulse along internal y and a ramp along internal z (T)
TIMES = [0.0, 5e-12, 2e-11, 4e-11, 1e-9]
VALUES = [(0.0, 0.0, 0.0), (0.0, 0.05, -0.01), (0.01, 0.05, -0.02), (0.0, 0.0, 0.01), (0.0, 0.0, 0.0)]


def _pair(problem):
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(**problem)
    return O.Oracle(prob), Plan(prob)


@pytest.mark.parametrize("t", [0.0, 1e-12, 5e-12, 1.3e-11, 3.9e-11])
def test_bext_table_fields(t):
    o, g = _pair(FILM)
    o.set_table(0, TIMES, VALUES)
    g.set_table("bext", TIMES, VALUES)
    o.set_time(t)
    g.set_time(t)
    m = rand_m(FILM["n"], seed=3)
    fo, fg = o.fields(m), g.fields(m)
    if t == 0.0:
        # at (and before) the first point the reference's updater gives 0
        assert np.abs(to_np(fg["zee"])).max() == 0.0
        return
    assert rel_err(to_np(fg["zee"]), fo["zee"]) < 1e-5
    assert rel_err(to_np(fg["eff"]), fo["eff"]) < 1e-5


@pytest.mark.parametrize("solver,dt,maxerr", [("heun", 2e-14, 1e-3), ("rk12", 1e-15, 1e-4), ("rk23", 1e-15, 1e-5),
                                              ("rk45", 1e-15, 1e-5)])
def test_field_pulse_trajectory(solver, dt, maxerr):
    import oracle as O
    o, g = _pair(FILM)
    o.set_table(0, TIMES, VALUES)
    g.set_table("bext", TIMES, VALUES)
    m0 = rand_m(FILM["n"], seed=5, kind="near_x")
    r = O.OracleRun(o, m0, solver=solver, dt=dt, maxerr=maxerr)
    g.solver(solver, dt=dt, maxerr=maxerr)
    g.set_state(m0)
    dur = 3e-11
    r.run(dur)
    g.run(dur)
    st = g.stats()
    mo = o.normalize(r.m)
    err = np.abs(g.get_state() - mo).max()
    print(solver, st["step"], r.st.step, err)
    assert err < 2e-4
    if solver != "heun":
        assert abs(st["step"] - r.st.step) <= max(2, 0.02 * r.st.step)
    # the pulse moved the magnetisation
    assert np.abs(mo - o.normalize(m0.copy())).max() > 1e-3


def test_current_table_zhang_li():
    o, g = _pair(dict(n=(1, 8, 64), cell=(2e-9, 2e-9, 2e-9), demag=1, exchange=1, zhangli=1, msat=8.6e5,
                      aex=1.3e-11, alpha=0.02, zl_pol=0.5, xi=0.05, j=(0.0, 0.0, 0.0)))
    times = [0.0, 1e-10, 2e-10]
    vals = [(0.0, 0.0, 0.0), (0.0, 0.0, 1e12), (0.0, 0.0, 5e11)]
    o.set_table(1, times, vals)
    g.set_table("j", times, vals)
    m = rand_m((1, 8, 64), seed=9)
    for t in [5e-11, 1.5e-10]:
        o.set_time(t)
        g.set_time(t)
        to, _, _ = o.torque(m)
        tg, _ = g.torque(m)
        assert rel_err(to_np(tg), to) < 1e-5


def test_stepping_past_the_table_is_an_error():
    from mumax2 import _native as nat
    _, g = _pair(FILM)
    g.set_table("bext", [0.0, 1e-12], [(0, 0, 0), (0, 0.01, 0)])
    g.solver("rk23", dt=1e-13, maxerr=1e-4)
    g.set_state(rand_m(FILM["n"], seed=1, kind="near_x"))
    with pytest.raises(nat.MMError) as e:
        g.run(5e-12)
    assert e.value.code == nat.MM_ERR_RANGE
    g.set_table("bext", [], [])  # removing the table makes the plan usable again
    g.solver("rk23", dt=1e-13, maxerr=1e-4)
    g.run(1e-12)


def test_script_setpointwise():
    """setpointwise through the script API (user axes) against the oracle."""
    import oracle as O
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
    for t, v in zip(TIMES, VALUES):
        mm.setpointwise("B_ext", t, list(v[::-1]))  # user order is the reverse of internal
    mm.run(2e-11)
    m_user = mm.getv("<m>")
    o = O.Oracle(O.full_desc(**FILM))
    o.set_table(0, TIMES, VALUES)
    N = 512
    m = np.zeros(3 * N)
    m[2 * N:] = 1.0
    m[N:2 * N] = 0.1
    r = O.OracleRun(o, m, solver="rk12", dt=1e-15, mindt=1e-15, maxerr=1e-4)
    r.run(2e-11)
    mo = o.average(o.normalize(r.m))[::-1]
    assert np.abs(np.array(m_user) - mo).max() < 1e-4
    mm.reset()


def test_bext_table_on_mixed_radix_batched_plan():
    """A B_ext time table on a batched plan whose padded sizes are not powers of two (the
    mixed-radix C2R epilogue with staged per-simulation scalars): each simulation's
    fields at a table time equal its own single plan's and the oracle's."""
    import oracle as O
    from mumax2 import Plan
    n = (1, 12, 20)
    prob = dict(FILM, n=n)
    sims = [dict(msat=8e5, aex=1.3e-11, alpha=0.05, bext=(0.0, 0.0, 0.0)),
            dict(msat=6e5, aex=1.0e-11, alpha=0.1, bext=(0.0, 0.01, 0.0))]
    g = Plan(O.full_desc(**prob), sims=sims)
    g.set_table("bext", TIMES, VALUES)
    g.set_time(1.3e-11)
    N = n[1] * n[2]
    m = np.concatenate([rand_m(n, seed=8), rand_m(n, seed=9)])
    fg = to_np(g.fields(m)["eff"])
    for b, sm in enumerate(sims):
        q = O.full_desc(**dict(prob, **sm))
        o = O.Oracle(q)
        o.set_table(0, TIMES, VALUES)
        o.set_time(1.3e-11)
        err = rel_err(fg[3 * N * b:3 * N * (b + 1)], o.fields(m[3 * N * b:3 * N * (b + 1)])["eff"])
        print("mixed-radix batched table", b, err)
        assert err < 1e-5
