"""The tile autotuner: every tile variant of the row, column and epilogue passes gives
bit-identical fields and torques (only the block decomposition changes), the tuned choice
is a valid variant with a measured evaluation time, and a stepped trajectory does not
depend on the tiles."""
import itertools

import numpy as np
import pytest

from helpers import rand_m, to_np

pytestmark = pytest.mark.gpu

VARIANTS = [list(t) for t in itertools.product((-1, 0, 1), (-1, 0, 1), (-1, 0))]


def _plan(n, cell, nsim=1, **terms):
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(n=n, cell=cell, msat=8e5, aex=1.3e-11, **terms)
    if nsim == 1:
        return Plan(prob)
    from mumax2 import workloads as W
    _, sims, _ = W.relax_set(nsim, seed=4)
    return Plan(prob, sims=sims)


@pytest.mark.parametrize("n,cell,nsim", [
    ((16, 64, 64), (2e-9, 4e-9, 4e-9), 1),     # 3-D: row, column and epilogue passes
    ((4, 32, 256), (2e-9, 4e-9, 4e-9), 1),     # long rows
    ((1, 64, 64), (3e-9, 4e-9, 4e-9), 8),      # batched single-layer films
])
def test_tile_variants_are_bit_identical(n, cell, nsim):
    p = _plan(n, cell, nsim, demag=1, exchange=1, anis=1, ku=3e5, anisu=(0.0, 0.6, 0.8), zeeman=1,
              bext=(0.0, 0.01, 0.02))
    tiles, us = p.tiles()
    assert tiles in VARIANTS and us > 0.0
    m = np.concatenate([rand_m(n, seed=s) for s in range(nsim)])
    p.set_tiles([0, 0, 0])
    ref_t, _ = p.torque(m)
    ref_f = p.fields(m)["eff"]
    ref_t, ref_f = to_np(ref_t), to_np(ref_f)
    for v in VARIANTS:
        p.set_tiles(v)
        t, _ = p.torque(m)
        f = p.fields(m)["eff"]
        assert np.array_equal(to_np(t), ref_t), v
        assert np.array_equal(to_np(f), ref_f), v
    p.close()


def test_trajectory_independent_of_tiles():
    n, cell = (8, 32, 32), (3e-9, 4e-9, 4e-9)
    m0 = rand_m(n, seed=3)
    out = []
    for v in ([0, 0, 0], [1, -1, -1], [-1, 1, 0]):
        p = _plan(n, cell, demag=1, exchange=1)
        p.set_tiles(v)
        p.solver("rk23", dt=1e-13, maxerr=1e-5)
        p.set_state(m0)
        p.steps(20)
        out.append((p.get_state(), p.stats()))
        p.close()
    for s, st in out[1:]:
        assert np.array_equal(s, out[0][0])
        assert st["step"] == out[0][1]["step"] and st["badsteps"] == out[0][1]["badsteps"]


def test_set_tiles_rejects_out_of_range():
    from mumax2 import _native as nat
    p = _plan((2, 8, 8), (3e-9, 3e-9, 3e-9), demag=1, exchange=1)
    with pytest.raises(nat.MMError):
        p.set_tiles([0, 0, 1])
    with pytest.raises(nat.MMError):
        p.set_tiles([2, 0, 0])
    p.close()
