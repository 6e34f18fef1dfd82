"""Host-side generator of the thermal-ensemble workload (no GPU)."""
import numpy as np

from mumax2 import workloads as W


def test_ensemble_draws_are_seeded_and_in_range():
    a = W.ensemble(nsim=2048, seed=0)
    b = W.ensemble(nsim=2048, seed=0)
    c = W.ensemble(nsim=2048, seed=1)
    assert [x["ids"].tolist() for x in a] == [x["ids"].tolist() for x in b]
    assert [x["ids"].tolist() for x in a] != [x["ids"].tolist() for x in c]
    assert sum(len(x["sims"]) for x in a) == 2048
    ids = np.sort(np.concatenate([x["ids"] for x in a]))
    assert (ids == np.arange(2048)).all()
    grids = {tuple(x["n"]) for x in a}
    assert grids == {(1, 32, 32), (1, 32, 64), (1, 64, 64), (2, 64, 128), (4, 128, 128)}
    seeds = set()
    for cls in a:
        assert cls["cell"] == (3e-9, 4e-9, 4e-9)
        for s, m0 in zip(cls["sims"], cls["m0"]):
            assert 4e5 <= s["msat"] <= 1.2e6
            assert 5e-12 <= s["aex"] <= 2e-11
            assert 0.01 <= s["alpha"] <= 0.1
            assert np.linalg.norm(s["bext"]) <= 0.05 + 1e-12
            assert s["temp"] == 300.0
            assert abs(np.linalg.norm(m0) - 1.0) < 1e-12
            seeds.add(s["seed"])
    assert len(seeds) == 2048
    # mean cells per simulation of the five sizes is about 17.8 k
    assert 30e6 < W.cells_of(a) < 45e6


def test_uniform_state_layout():
    st = W.uniform_state((1, 2, 3), [(1, 0, 0), (0, 0.6, 0.8)], 2)
    assert st.shape == (2 * 3 * 6,)
    s1 = st[18:].reshape(3, 6)
    assert np.allclose(s1[1], 0.6) and np.allclose(s1[2], 0.8) and np.allclose(s1[0], 0.0)
