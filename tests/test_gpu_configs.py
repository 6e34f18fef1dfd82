"""The single-simulation configurations against the FP64 oracle: the 128x32x1 film with
RK45 (<m> trajectory within 1e-4) and a Neel wall moved by Zhang-Li current (wall
position from <m_x> within 0.05 nm), on runs short enough for the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sp4_film_rk45_trajectory():
    import oracle as O
    from mumax2 import Plan
    from mumax2 import workloads as W
    prob, m0 = W.sp4_film(seed=3)
    d = O.full_desc(**prob)
    o = O.Oracle(d)
    g = Plan(d)
    g.solver("rk45", dt=1e-15, maxerr=1e-5)
    g.set_state(m0)
    g.tabulate(1e-11, capacity=16)
    r = O.OracleRun(o, m0.astype(np.float64), solver="rk45", dt=1e-15, maxerr=1e-5)
    ref = []
    while r.st.t < 5e-11:
        r.step()
        if r.st.t - len(ref) * 1e-11 >= 1e-11:
            ref.append(o.average(o.normalize(r.m.copy())))
    g.run(5e-11)
    rows = g.tabulate_read()[0]
    assert len(rows) == len(ref) == 5
    assert np.abs(rows[:, 1:4] - np.array(ref)).max() < 1e-4
    assert abs(g.stats()["step"] - r.st.step) <= 2


def test_neel_wall_zhang_li_position():
    import oracle as O
    from mumax2 import Plan
    from mumax2 import workloads as W
    prob, m0, x0 = W.neel_wall_strip(seed=1)
    # a quarter-size strip (256 x 64) keeps the oracle run short
    nx, ny = 256, 64
    m = m0.reshape(3, 1, 128, 512)[:, :, :ny, 128:128 + nx].copy().ravel()
    prob = dict(prob, n=(1, ny, nx))
    d = O.full_desc(**prob)
    o = O.Oracle(d)
    g = Plan(d)
    g.solver("rk45", dt=1e-15, maxerr=1e-5)
    g.set_state(m)
    r = O.OracleRun(o, m.astype(np.float64), solver="rk45", dt=1e-15, maxerr=1e-5)
    dur = 1e-11
    r.run(dur)
    g.run(dur)
    L = nx * 2e-9
    xo = W.wall_position(o.average(o.normalize(r.m.copy()))[2], L)
    xg = W.wall_position(g.average()[2], L)
    x_start = W.wall_position(m.reshape(3, -1)[2].mean(), L)
    print("wall", x_start, xo, xg)
    assert abs(xg - xo) < 5e-11
    assert abs(xo - x_start) > 1e-11   # the current moved the wall
