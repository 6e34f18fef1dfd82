"""Output fed from the GPU: asynchronous snapshots (D2H on a side stream, file written by a
host thread) and device autosave (the state copied by the step that crosses each save
time, notify_autosave.go:25-31), checked against synchronous reads of the same states."""
import numpy as np
import pytest

from helpers import rand_m

pytestmark = pytest.mark.gpu

FILM = dict(n=(1, 16, 32), cell=(3e-9, 3.90625e-9, 3.90625e-9), demag=1, exchange=1, zeeman=1, msat=8e5,
            aex=1.3e-11, alpha=0.05, bext=(0.0, 4.3e-3, -24.6e-3))


def _plan():
    import oracle as O
    from mumax2 import Plan
    g = Plan(O.full_desc(**FILM))
    g.solver("rk23", dt=1e-15, maxerr=1e-5)
    g.set_state(rand_m(FILM["n"], seed=2, kind="near_x"))
    return g


@pytest.mark.parametrize("fmt", ["ovf", "omf", "dump"])
def test_save_async_matches_state(tmp_path, fmt):
    from mumax2 import _native as nat
    g = _plan()
    g.run(2e-12)
    ref = g.get_state().reshape(3, *FILM["n"])
    t = g.stats()["t"]
    p = tmp_path / f"m.{fmt}"
    g.save_async(p, fmt)
    g.run(2e-12)          # the GPU keeps stepping while the file is written
    g.save_wait()
    data, n, tf = nat.read_field(p)
    assert n == FILM["n"] and np.array_equal(data, ref)
    if fmt != "omf":
        assert tf == pytest.approx(t, rel=1e-15)


def test_device_autosave_times_and_states():
    import oracle as O
    g = _plan()
    period = 1e-12
    g.autosave(period, capacity=16)
    g.run(5e-12)
    times, states = g.autosave_read()[0]
    assert len(times) == 5 and (np.diff(times) > 0).all()
    # each save is the first accepted step past k * period
    assert all(t >= (k + 1) * period for k, t in enumerate(times))
    # the last saved state is a state of the trajectory: re-run to that time and compare
    g2 = _plan()
    g2.run(float(times[-1]))
    st = g2.stats()
    assert st["t"] == pytest.approx(times[-1], rel=1e-12)
    assert np.array_equal(g2.get_state(), states[-1])


def test_script_save_autosave_and_setarray_file(tmp_path):
    from mumax2 import _native as nat
    from mumax2 import engine as mm
    mm.reset()
    mm.setgridsize(32, 16, 1)
    mm.setcellsize(3.90625e-9, 3.90625e-9, 3e-9)
    mm.load("micromagnetism")
    mm.setv("Msat", 8e5)
    mm.setv("Aex", 1.3e-11)
    mm.setv("alpha", 0.05)
    mm.setarray("m", [[[[1]]], [[[0.1]]], [[[0]]]])
    mm.engine().outdir = str(tmp_path)
    mm.autosave("m", "ovf", [], 2e-12)
    mm.run(6e-12)
    files = sorted(p.name for p in tmp_path.glob("m*.ovf"))
    assert files == ["m000001.ovf", "m000002.ovf", "m000003.ovf"]
    mm.saveas("m", "omf", ["Text"], str(tmp_path / "final.omf"))
    a = mm.getarray("m")
    mm.setarray("m", [[[[0]]], [[[1]]], [[[0]]]])
    mm.setarray_file("m", str(tmp_path / "final.omf"))
    assert np.allclose(mm.getarray("m"), a, atol=1e-7)
    data, n, _ = nat.read_field(tmp_path / "m000003.ovf")
    assert n == (1, 16, 32)
    mm.reset()
