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
    problem, sims, masks, res = WS.generate(1024, seed=11)
    assert (res["maxtorque"] < WS.thresholds(sims)).all()
    data = WS.Dataset(problem, sims, masks, res["state"])
    net, losses = WS.train(data, epochs=40, batch=256, lr=1e-3)
    assert losses[-1] < 0.5 * losses[0]
    _, hs, hm = W.relax_set(256, seed=77)
    ev = WS.evaluate(net, problem, hs, hm, max_steps=WS.step_budget(res["steps"]))
    print(ev)
    assert ev["warm_ok_frac"] > 0.9
    assert ev["warm_steps_mean"] < ev["cold_steps_mean"]
