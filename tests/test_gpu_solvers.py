"""GPU time stepping against the FP64 oracle and the reference's golden SP4 trace.

The GPU integrates in FP32 with the same solver logic as the oracle (FP64).  Short
trajectories must agree to 2e-4 in m (accumulated FP32 rounding); step counts of the
adaptive solvers must agree to within a few percent.
"""
import os

import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _pair(problem, masks=None):
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(**problem)
    if masks:
        prob["masks"] = masks
    return O.Oracle(prob), Plan(prob, masks=masks or {})


FILM = dict(n=(1, 16, 32), cell=(3e-9, 3.90625e-9, 3.90625e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
            aex=1.3e-11, alpha=0.05, bext=(0.0, 4.3e-3, -24.6e-3))


@pytest.mark.parametrize("solver,dt,maxerr,dur", [
    ("euler", 5e-15, 1e-3, 2e-12),
    ("heun", 2e-14, 1e-3, 1e-11),
    ("rk12", 1e-15, 1e-4, 1e-11),
    ("rk23", 1e-15, 1e-5, 2e-11),
    ("rk45", 1e-15, 1e-5, 2e-11),
])
def test_solver_trajectory(solver, dt, maxerr, dur):
    import oracle as O
    o, g = _pair(FILM)
    m0 = rand_m(FILM["n"], seed=11, kind="near_x")
    r = O.OracleRun(o, m0, solver=solver, dt=dt, mindt=1e-18, maxerr=maxerr)
    r.run(dur)
    g.solver(solver, dt=dt, mindt=1e-18, maxerr=maxerr)
    g.set_state(m0)
    g.run(dur)
    st = g.stats()
    mg = g.get_state().astype(np.float64)
    err = np.abs(mg - r.m).max()
    print(solver, "steps oracle", r.st.step, "gpu", st["step"], "t", r.st.t, st["t"], "max|dm|", err)
    assert st["status"] == 0
    assert err < 2e-4
    assert abs(st["step"] - r.st.step) <= max(2, 0.05 * r.st.step)
    assert st["t"] >= r.st.t - 1e-9 * dur or abs(st["t"] - r.st.t) < 0.05 * dur


def test_rk12_counts_match_reference_semantics():
    # bad steps are re-done from the saved state (solve_rk12.go:117-210)
    import oracle as O
    o, g = _pair(FILM)
    m0 = rand_m(FILM["n"], seed=12)  # random state: large torque, many rejections from dt=1e-13
    r = O.OracleRun(o, m0, solver="rk12", dt=1e-13, mindt=1e-18, maxerr=1e-4)
    for _ in range(20):
        r.step()
    g.solver("rk12", dt=1e-13, mindt=1e-18, maxerr=1e-4)
    g.set_state(m0)
    g.steps(20)
    st = g.stats()
    print("badsteps oracle", r.st.badsteps, "gpu", st["badsteps"], "t", r.st.t, st["t"])
    assert st["step"] == 20
    assert st["badsteps"] == r.st.badsteps
    assert abs(st["t"] - r.st.t) / r.st.t < 1e-3


def test_reductions_match_oracle():
    prob = dict(FILM)
    prob.update(anis=1, ku=2e5, anisu=(0.0, 0.6, 0.8))
    o, g = _pair(prob)
    m = rand_m(prob["n"], seed=13)
    g.solver("rk45")
    g.set_state(m)
    mn = o.normalize(m)
    t, _, _ = o.torque(m)
    mt_o = o.maxtorque(t)
    mt_g = g.maxtorque()
    print("maxtorque", mt_o, mt_g)
    assert abs(mt_g - mt_o) / mt_o < 1e-5
    av_o = o.average(mn)
    av_g = g.average()
    print("avg", av_o, av_g)
    assert np.abs(av_g - av_o).max() < 1e-6
    eo = o.energy(m)
    eg = g.energy()
    for k in eo:
        print(k, eo[k], eg[k])
        assert abs(eg[k] - eo[k]) <= 1e-5 * max(abs(eo[k]), 1e-30) + 1e-6 * abs(eo["E_demag"])


def test_relax_run_until_maxtorque():
    import oracle as O
    prob = dict(FILM)
    prob.update(alpha=1.0, bext=(0, 0, 0))
    o, g = _pair(prob)
    m0 = rand_m(prob["n"], seed=14, kind="near_x")
    thr = 1e-2 * 2.211e5 * prob["msat"]
    g.solver("rk23", dt=1e-15, maxerr=1e-5)
    g.set_state(m0)
    g.run_until_maxtorque(thr)
    st = g.stats()
    mt = g.maxtorque()
    print("relax steps", st["step"], "maxtorque", mt, thr)
    assert st["status"] == 0 and mt < thr * 1.001
    r = O.OracleRun(o, m0, solver="rk23", dt=1e-15, maxerr=1e-5)
    while True:
        t, _, _ = o.torque(r.m)
        if o.maxtorque(t) < thr:
            break
        r.step()
    print("oracle relax steps", r.st.step)
    assert abs(st["step"] - r.st.step) <= max(3, 0.05 * r.st.step)


def test_sp4_against_golden_trace():
    """muMAG standard problem 4 (tests/stdproblem4.py of the reference) on the GPU: relax
    2 ns at alpha=1 from (1,1,0), then 1 ns in B=(-24.6, 4.3, 0) mT at alpha=0.02 with
    RK12, m_maxerror 1/3000; <m>(t) compared with the reference's golden trace."""
    gold = np.loadtxt(os.path.join(GOLDEN, "sp4_stdsolution4.txt"))
    n = (1, 32, 128)
    prob = dict(n=n, cell=(3e-9, 125e-9 / 32, 500e-9 / 128), demag=1, exchange=1, zeeman=1, msat=800e3,
                aex=1.3e-11, alpha=1.0)
    o, g = _pair(prob)
    N = 32 * 128
    m = np.zeros(3 * N)
    m[N:2 * N] = 1
    m[2 * N:] = 1
    g.solver("rk12", dt=1e-15, mindt=1e-15, maxerr=1.0 / 3000)
    g.set_state(m)
    g.run(2e-9)
    prob2 = dict(prob, alpha=0.02, bext=(0.0, 4.3e-3, -24.6e-3))
    g.set_problem(prob2)
    g.solver("rk12", dt=1e-15, mindt=1e-15, maxerr=1.0 / 3000)
    g.set_time(0.0, 1e-15)
    rec = []
    for k in range(101):
        rec.append((g.stats()["t"] * 1e9, *g.average()[::-1]))
        if k < 100:
            g.run(10e-12)
    rec = np.array(rec)
    rec = rec[rec[:, 0] <= gold[-1, 0]]   # compare inside the golden trace's time window only
    errs = []
    for c in range(3):
        gi = np.interp(rec[:, 0], gold[:, 0], gold[:, c + 1])
        errs.append((np.abs(gi - rec[:, c + 1]).max(), np.sqrt(((gi - rec[:, c + 1]) ** 2).mean())))
    print("sp4 max/rms per component", errs)
    for mx, rms in errs:
        assert mx < 0.05 and rms < 0.025


def test_rk23_trajectory_on_mixed_radix_grid():
    """RK23 on a film whose padded sizes are not powers of two (24 x 40 cells, padded
    48 x 80): the same accepted and rejected steps as the oracle, m within 2e-4."""
    import oracle as O
    prob = dict(FILM)
    prob["n"] = (1, 24, 40)
    o, g = _pair(prob)
    m0 = rand_m(prob["n"], seed=14, kind="near_x")
    r = O.OracleRun(o, m0, solver="rk23", dt=1e-15, mindt=1e-18, maxerr=1e-5)
    for _ in range(20):
        r.step()
    g.solver("rk23", dt=1e-15, mindt=1e-18, maxerr=1e-5)
    g.set_state(m0)
    g.steps(20)
    st = g.stats()
    err = np.abs(g.get_state().astype(np.float64) - o.normalize(r.m.copy())).max()
    print("mixed-radix rk23: gpu", st["step"], st["badsteps"], "oracle", r.st.step, r.st.badsteps, "max|dm|", err)
    assert st["status"] == 0 and st["step"] == r.st.step and st["badsteps"] == r.st.badsteps
    assert err < 2e-4
