"""The script API (mirror of the reference's mumax2.py / api.go) on the GPU path,
against the FP64 oracle driven directly in internal axes.  Checks the user<->internal
axis swap (api.go:13,44,152), module wiring and the lazy derived quantities."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_script_api_matches_oracle():
    import oracle as O
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(32, 16, 1)                       # user x, y, z
    mm.setcellsize(4e-9, 3.9e-9, 3e-9)
    mm.load("micromagnetism")
    mm.load("micromag/energy")
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 0.05)
    mm.setarray("m", [[[[1]]], [[[1]]], [[[0]]]])  # user (1, 1, 0), resampled to the grid
    mm.setv("B_ext", [-24.6e-3, 4.3e-3, 0.0])
    mm.setv("m_maxerror", 1e-4)
    mm.run(5e-12)
    m_user = mm.getv("<m>")
    t = mm.gets("t")
    E = mm.gets("E")
    mt = mm.gets("maxtorque")

    n = (1, 16, 32)
    o = O.Oracle(O.full_desc(n=n, cell=(3e-9, 3.9e-9, 4e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
                             aex=1.3e-11, alpha=0.05, bext=(0.0, 4.3e-3, -24.6e-3)))
    N = 512
    m = np.zeros(3 * N)
    m[N:2 * N] = 1
    m[2 * N:] = 1
    r = O.OracleRun(o, m, solver="rk12", dt=1e-15, mindt=1e-15, maxerr=1e-4)
    r.run(5e-12)
    mo = o.average(o.normalize(r.m))[::-1]
    print("gpu", m_user, t, "oracle", mo, r.st.t)
    assert abs(t - r.st.t) < 1e-3 * t
    assert np.abs(np.array(m_user) - mo).max() < 1e-4
    eo = o.energy(r.m)["E"]
    assert abs(E - eo) < 1e-4 * abs(eo)
    to, _, _ = o.torque(r.m)
    assert abs(mt - o.maxtorque(to)) < 1e-4 * mt
    # arrays come back in user layout [comp][x][y][z]
    a = mm.getarray("m")
    assert a.shape == (3, 32, 16, 1)
    assert np.allclose(a.mean(axis=(1, 2, 3)), m_user, atol=1e-6)
    mm.reset()


def test_relax_idiom_run_until_smaller():
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(32, 32, 1)
    mm.setcellsize(4e-9, 4e-9, 3e-9)
    mm.load("micromagnetism")
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 1.0)
    rng = np.random.default_rng(0)
    mm.setarray("m", rng.normal(size=(3, 32, 32, 1)))
    thr = 1e-2 * 2.211e5 * 8e5
    mm.run_until_smaller("maxtorque", thr)     # api.go:122-131, relax idiom of stdproblem5.py:55
    assert mm.gets("maxtorque") < thr
    mm.reset()


def test_demagexch_module_script():
    """load("demagexch") + llg + solver: the combined convolution drives the dynamics."""
    import oracle as O
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(16, 8, 2)
    mm.setcellsize(4e-9, 4e-9, 3e-9)
    mm.load("demagexch")
    mm.load("llg")
    mm.load("solver/rk23")
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 0.1)
    mm.setv("m_maxerror", 1e-5)
    mm.setarray("m", [[[[1]]], [[[0.2]]], [[[0.1]]]])
    mm.run(2e-12)
    m_user = mm.getv("<m>")
    n = (2, 8, 16)
    o = O.Oracle(O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, msat=8e5, aex=1.3e-11,
                             alpha=0.1, demag_exchange=1, demag_accuracy=8))
    N = 2 * 8 * 16
    m = np.zeros(3 * N)
    m[:N], m[N:2 * N], m[2 * N:] = 0.1, 0.2, 1.0
    r = O.OracleRun(o, m, solver="rk23", dt=1e-15, maxerr=1e-5)
    r.run(2e-12)
    mo = o.average(o.normalize(r.m))[::-1]
    assert np.abs(np.array(m_user) - mo).max() < 1e-4
    h = mm.getarray("H_dex")
    assert h.shape == (3, 16, 8, 2) and np.abs(h).max() > 0
    mm.reset()
