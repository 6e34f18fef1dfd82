"""The learned warm start end to end at a small scale: relaxed states from the plain
relaxer train the U-Net, whose predictions then start relaxations of unseen problems.
The warm relaxations must take fewer solver steps on average than the cold ones, and
most must end in a state the cold relax confirms (max torque and energy)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_warm_start_saves_steps():
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    problem, sims, masks, res = WS.generate(4096, seed=11)
    assert (res["maxtorque"] < WS.thresholds(sims)).all()
    data = WS.Dataset(problem, sims, masks, res["state"])
    net, losses = WS.train(data, epochs=40, batch=256, lr=2e-3)
    assert losses[-1] < 0.5 * losses[0]
    _, hs, hm = W.relax_set(256, seed=77)
    ev = WS.evaluate(net, problem, hs, hm, max_steps=WS.step_budget(res["steps"]))
    print(ev)
    assert ev["warm_ok_frac"] > 0.9
    assert ev["warm_steps_mean"] < ev["cold_steps_mean"]


def test_pool_drain_on_small_plan_matches():
    """A pool that moves its last relaxations to a 16-slot plan reaches the same relaxed
    states (energy within 1e-4 relative, every threshold met) as one that finishes them
    in place; the moved relaxations pay at most a few steps for the restarted step
    control."""
    import numpy as np
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(96, seed=21)
    thr = WS.thresholds(sims)
    cold = W.cold_state(problem["n"], 1)
    a = WS.relax_pool(problem, sims, masks, [cold] * 96, thr, slots=64, tail_slots=16)
    b = WS.relax_pool(problem, sims, masks, [cold] * 96, thr, slots=64, tail_slots=64)
    assert (a["maxtorque"] < thr).all() and (b["maxtorque"] < thr).all()
    erel = np.abs(a["energy"] - b["energy"]) / np.abs(b["energy"])
    assert erel.max() < 1e-4
    assert (a["steps"] <= b["steps"] + 40).all()


def test_speculative_redo_gives_the_same_results():
    """Redos started speculatively beside long first attempts (here from the first step
    on, so that most are started and cancelled) give the results of the queued redos: every
    run is the same computation in whichever slot it lands, so without the drain phase the
    arrays agree exactly; with it, within the drain test's bounds."""
    import numpy as np
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(96, seed=21)
    thr = WS.thresholds(sims)
    n = problem["n"]
    cold = W.cold_state(n, 1)
    fallback = W.uniform_state(n, (0.0, 1.0, 0.0), 1)

    def accept(q, steps, mt, e):
        return q % 5 != 0

    runs = {}
    for spec, tail in ((0, 64), (1, 64), (0, 16), (1, 16)):
        runs[spec, tail] = WS.relax_pool(problem, sims, masks, [cold] * 96, thr, slots=64, tail_slots=tail,
                                         accept=accept, fallback=fallback, spec_steps=spec)
    a, b = runs[0, 64], runs[1, 64]
    assert b["spec_started"] > 0 and b["spec_cancelled"] > 0 and a["spec_started"] == 0
    for k in ("steps", "maxtorque", "energy", "first_steps", "first_maxtorque", "first_energy", "fell_back"):
        assert np.array_equal(a[k], b[k]), k
    assert a["fell_back"].sum() == len(range(0, 96, 5))
    c, d = runs[0, 16], runs[1, 16]
    assert (d["maxtorque"] < thr).all() and np.array_equal(c["fell_back"], d["fell_back"])
    erel = np.abs(d["energy"] - a["energy"]) / np.abs(a["energy"])
    assert erel.max() < 1e-4


def test_mirror_x_is_a_symmetry_of_the_plain_relax():
    """The training set's mirror augmentation: reflecting a problem along x (mask and
    fields, B_y -> -B_y, u_y -> -u_y) and relaxing it from the same cold start (+x) gives
    the mirror image of the original relaxed state with m -> (m_x, -m_y, -m_z), the
    energy unchanged."""
    from mumax2 import warmstart as WS
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(16, seed=5)
    n = problem["n"]
    ny, nx = n[1], n[2]
    N = ny * nx
    msims = []
    for s in sims:
        q = dict(s)
        q["anisu"] = (s["anisu"][0], -s["anisu"][1], s["anisu"][2])   # internal (z, y, x)
        q["bext"] = (s["bext"][0], -s["bext"][1], s["bext"][2])
        msims.append(q)
    mmasks = [np.asarray(m).reshape(ny, nx)[:, ::-1].ravel().copy() for m in masks]
    thr = WS.thresholds(sims)
    cold = W.cold_state(n, 1)
    a = WS.relax_pool(problem, sims, masks, [cold] * 16, thr, slots=16, keep_states=True)
    b = WS.relax_pool(problem, msims, mmasks, [cold] * 16, thr, slots=16, keep_states=True)
    assert (a["maxtorque"] < thr).all() and (b["maxtorque"] < thr).all()
    sa = a["state"].reshape(16, 3, ny, nx)
    sb = b["state"].reshape(16, 3, ny, nx)
    want = sa[:, :, :, ::-1] * np.array([-1.0, -1.0, 1.0])[None, :, None, None]   # internal (z, y, x) comps
    dm = np.abs(sb - want).max(axis=(1, 2, 3))
    erel = np.abs(a["energy"] - b["energy"]) / np.abs(a["energy"])
    print("mirror: max |dm| per problem", dm, "energy", erel.max(), "steps", a["steps"], b["steps"])
    assert erel.max() < 1e-4
    assert np.median(dm) < 1e-2
