"""Error of the GPU path against the FP64 oracle, one figure per configuration (each test
prints it): the single-layer film over the full simulated nanosecond, the field of a
3-D film, the benchmarked 256x256x16 film at full size (fields, energy, five RK23
steps), one member of the thermal ensemble stepped with the same Philox noise, and a
relaxation of the warm-start problem set.  Targets: 1e-5 relative on H_eff, 1e-4 on the
averaged magnetisation, 1e-4 relative on the relaxed energy."""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu


def test_film_rk45_one_nanosecond():
    """128x32x1 film (SP4 geometry), RK45 at max error 1e-5, 1 ns: <m> every 100 ps."""
    import oracle as O
    from mumax2 import Plan
    from mumax2 import workloads as W
    prob, m0 = W.sp4_film(seed=3)
    d = O.full_desc(**prob)
    o = O.Oracle(d)
    g = Plan(d)
    g.solver("rk45", dt=1e-15, maxerr=1e-5)
    g.set_state(m0)
    g.tabulate(1e-10, capacity=16)
    r = O.OracleRun(o, m0.astype(np.float64), solver="rk45", dt=1e-15, maxerr=1e-5)
    ref = []
    while r.st.t < 1e-9:
        r.step()
        if r.st.t - len(ref) * 1e-10 >= 1e-10:
            ref.append(o.average(o.normalize(r.m.copy())))
    g.run(1e-9)
    rows = g.tabulate_read()[0]
    n = min(len(rows), len(ref))
    err = np.abs(rows[:n, 1:4] - np.array(ref[:n])).max()
    print("config film 128x32x1 RK45: max |<m> - oracle| over 1 ns =", err, "steps", g.stats()["step"], r.st.step)
    assert n >= 9
    assert err < 1e-4


def test_film3d_field_64x64x16():
    """3-D film with the headline's material (Ms 1.1e6, Aex 1.5e-11, Ku1 5e5 along z) on a
    64x64x16 grid: H_eff and torque."""
    import oracle as O
    from mumax2 import Plan
    n = (16, 64, 64)
    d = O.full_desc(n=n, cell=(2e-9, 4e-9, 4e-9), demag=1, exchange=1, anis=1, msat=1.1e6, aex=1.5e-11, ku=5e5,
                    anisu=(1.0, 0.0, 0.0), alpha=0.1)
    o = O.Oracle(d)
    g = Plan(d)
    m = rand_m(n, seed=9)
    err = rel_err(to_np(g.fields(m)["eff"]), o.fields(m)["eff"])
    t_err = rel_err(to_np(g.torque(m)[0]), o.torque(m)[0])
    print("config film3d 64x64x16: H_eff rel err", err, "torque rel err", t_err)
    assert err < 1e-5 and t_err < 1e-5


def test_headline_film3d_256x256x16_full_size():
    """The benchmarked workload itself (bench.py WORKLOAD: 256x256x16 cells of 4x4x2 nm,
    Ms 1.1e6, Aex 1.5e-11, Ku1 5e5 along z, alpha 0.1, RK23 at max error 1e-5, the
    seeded random initial state of the bench) at full size against the FP64 oracle:
    every field term, H_eff per component, the torque and the energy of that state
    (1e-5 relative), then 5 RK23 steps with the same accepted and rejected step counts,
    the same time reached and max |dm| < 2e-4."""
    import bench
    import oracle as O
    from mumax2 import Plan
    w = bench.WORKLOAD
    d = O.full_desc(**bench.problem())
    o = O.Oracle(d)
    g = Plan(d)
    m0 = bench.initial_m(0).astype(np.float64)
    N = int(np.prod(w["n"]))
    fg, fo = g.fields(m0), o.fields(m0)
    for term in ["demag", "ex", "anis", "eff"]:
        e = rel_err(to_np(fg[term]), fo[term])
        print(f"headline 256x256x16: {term} rel err {e:.3e}")
        assert e < 1e-5, term
    heg, heo = to_np(fg["eff"]).reshape(3, N), fo["eff"].reshape(3, N)
    per_comp = [float(np.abs(heg[c] - heo[c]).max() / np.abs(heo[c]).max()) for c in range(3)]
    print("headline 256x256x16: H_eff rel err per component (z, y, x internal)", per_comp)
    assert max(per_comp) < 1e-5
    t_err = rel_err(to_np(g.torque(m0)[0]), o.torque(m0)[0])
    print("headline 256x256x16: torque rel err", t_err)
    assert t_err < 1e-5
    g.solver(w["solver"], dt=w["dt0"], maxerr=w["maxerr"])
    g.set_state(m0)
    eg, eo = g.energy(), o.energy(m0)
    for k in ["E_ex", "E_demag", "E_anis", "E"]:
        e = abs(eg[k] - eo[k]) / abs(eo[k])
        print(f"headline 256x256x16: {k} rel err {e:.3e}")
        assert e < 1e-5, k
    r = O.OracleRun(o, m0, solver=w["solver"], dt=w["dt0"], maxerr=w["maxerr"])
    for _ in range(5):
        r.step()
    g.steps(5)
    st = g.stats()
    mg = g.get_state().astype(np.float64)
    dm = np.abs(mg - o.normalize(r.m.copy())).max()
    print("headline 256x256x16, 5 RK23 steps: gpu", st["step"], st["badsteps"], st["t"], "oracle", r.st.step,
          r.st.badsteps, r.st.t, "max|dm|", dm)
    assert st["status"] == 0
    assert st["step"] == r.st.step and st["badsteps"] == r.st.badsteps
    assert abs(st["t"] - r.st.t) <= 1e-6 * r.st.t
    assert dm < 2e-4


def test_thermal_ensemble_member():
    """One ensemble member (32x32x1, 4x4x3 nm, T = 300 K, stochastic Heun at 50 fs, 200
    steps = 10 ps): the same Philox noise on both sides, <m> compared."""
    import oracle as O
    from mumax2 import Plan
    n = (1, 32, 32)
    d = O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, zeeman=1, thermal=1, temp=300.0, seed=17,
                    msat=7e5, aex=1.2e-11, alpha=0.05, bext=(0.0, 0.02, 0.01))
    o = O.Oracle(d)
    g = Plan(d)
    m0 = rand_m(n, seed=4, kind="near_x")
    g.solver("heun", dt=5e-14)
    g.set_thermal_dt(5e-14)
    g.set_state(m0)
    g.steps(200)
    r = O.OracleRun(o, m0, solver="heun", dt=5e-14, dt_thermal=5e-14)
    for _ in range(200):
        r.step()
    mg = g.get_state().astype(np.float64)
    err = np.abs(o.average(mg) - o.average(o.normalize(r.m.copy()))).max()
    cell_err = np.abs(mg - o.normalize(r.m.copy())).max()
    print("config thermal member 32x32x1, 200 Heun steps: max |<m> - oracle|", err, "max cell", cell_err)
    assert err < 1e-4


def test_relaxation_energy():
    """A warm-start problem (64x64x1, seeded mask and parameters, alpha 1, RK23 at 1e-6)
    relaxed to maxtorque/(gamma Ms) < 1e-4 on both sides from the cold start: relaxed
    energy and <m>."""
    import oracle as O
    from mumax2 import Plan
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(1, seed=31)
    s = sims[0]
    d = O.full_desc(n=problem["n"], cell=problem["cell"], demag=1, exchange=1, anis=1, zeeman=1, msat=s["msat"],
                    aex=s["aex"], ku=s["ku"], anisu=s["anisu"], bext=s["bext"], alpha=1.0,
                    masks={"msat": masks[0]})
    o = O.Oracle(d)
    g = Plan(d, masks={"msat": masks[0]})
    m0 = W.cold_state(problem["n"], 1)
    thr = WS.thresholds(sims)[0]
    g.solver("rk23", dt=1e-14, maxerr=1e-6)
    g.set_state(m0)
    g.run_until_maxtorque(thr)
    r = O.OracleRun(o, m0.astype(np.float64), solver="rk23", dt=1e-14, maxerr=1e-6)
    while True:
        t, _, _ = o.torque(r.m)
        if o.maxtorque(t) < thr:
            break
        r.step()
    eg = g.energy()["E"]
    eo = o.energy(o.normalize(r.m.copy()))["E"]
    mg = g.get_state().astype(np.float64)
    m_err = np.abs(o.average(mg) - o.average(o.normalize(r.m.copy()))).max()
    print("config relax 64x64x1: energy rel err", abs(eg - eo) / abs(eo), "<m> err", m_err,
          "steps", g.stats()["step"], r.st.step)
    assert abs(eg - eo) / abs(eo) < 1e-4
