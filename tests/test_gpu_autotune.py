"""The tile autotuner: every tile variant of the row, column and epilogue passes, and the
fused single-layer evaluation (one launch, spectrum in shared memory), gives bit-identical
fields and torques (the same arithmetic in another block decomposition), the tuned choice
is a valid variant with a measured evaluation time, and a stepped trajectory does not
depend on the tiles."""
import itertools

import numpy as np
import pytest

from helpers import rand_m, to_np

pytestmark = pytest.mark.gpu

VARIANTS = [list(t) + [0] for t in itertools.product((-1, 0, 1), (-1, 0, 1), (-1, 0))]


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
    assert tiles[:3] + [0] in VARIANTS and tiles[3] in (0, 1) and us > 0.0
    if tiles[3]:
        assert n[0] == 1
    m = np.concatenate([rand_m(n, seed=s) for s in range(nsim)])
    p.set_tiles([0, 0, 0])
    ref_t, _ = p.torque(m)
    ref_f = p.fields(m)["eff"]
    ref_t, ref_f = to_np(ref_t), to_np(ref_f)
    variants = VARIANTS + ([[0, 0, 0, 1], [0, -1, -1, 1]] if n[0] == 1 else [])
    for v in variants:
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


@pytest.mark.parametrize("n", [(1, 32, 32), (1, 32, 64), (1, 64, 32), (1, 64, 64), (1, 32, 128), (1, 16, 32),
                               (1, 128, 64)])
def test_fused_single_layer_matches_passes(n):
    """The fused evaluation against the separate passes on every single-layer size it
    serves (and a size it does not, which must be refused), for a batched plan with
    per-simulation masks and for a single plan; then a batched relaxation stepped both
    ways gives the same states and step counts."""
    import oracle as O
    from mumax2 import Plan, _native as nat
    from mumax2 import workloads as W
    _, sims, _ = W.relax_set(6, seed=8)
    rng = np.random.default_rng(3)
    N = n[1] * n[2]
    masks = (rng.uniform(size=6 * N) > 0.15).astype(np.float32)
    prob = O.full_desc(n=n, cell=(3e-9, 4e-9, 4e-9), msat=8e5, aex=1.3e-11, demag=1, exchange=1, anis=1, ku=2e5,
                       anisu=(0.0, 0.6, 0.8), zeeman=1, bext=(0.0, 0.01, 0.02))
    p = Plan(prob, masks={"msat": masks}, sims=sims, masks_per_sim=True)
    m = np.concatenate([rand_m(n, seed=s) for s in range(6)])
    if n[1] > 64 or n[2] < 32:
        with pytest.raises(nat.MMError):
            p.set_tiles([0, 0, 0, 1])
        p.close()
        return
    p.set_tiles([0, 0, 0, 0])
    ref = to_np(p.torque(m)[0])
    p.set_tiles([0, 0, 0, 1])
    got = to_np(p.torque(m)[0])
    assert np.array_equal(got, ref)
    # stepping
    out = []
    for fused in (0, 1):
        p.set_tiles([0, 0, 0, fused])
        p.solver("rk23", dt=1e-14, maxerr=1e-6)
        p.set_state(m)
        before = [s["step"] for s in p.batch_stats()]
        p.steps(15)
        out.append((p.get_state(), [s["step"] - b for s, b in zip(p.batch_stats(), before)]))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    p.close()
    single = Plan(prob)
    single.set_tiles([0, 0, 0, 0])
    r1 = to_np(single.torque(m[:3 * N])[0])
    single.set_tiles([0, 0, 0, 1])
    r2 = to_np(single.torque(m[:3 * N])[0])
    assert np.array_equal(r1, r2)
    single.close()


def test_tuning_is_reused_for_plans_of_the_same_shape():
    """The autotuner times a plan shape once per process and device: a second plan of the
    same shape takes the first one's tiles without a tuning run, a new shape runs it."""
    import os
    from mumax2 import Plan
    from mumax2 import _native as nat
    if os.environ.get("MM_AUTOTUNE", "1").startswith("0"):
        return
    L = nat.lib()
    prob = dict(n=(1, 8, 512), cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, msat=8e5, aex=1.3e-11)
    r0 = L.mm_autotune_runs()
    a = Plan(prob)
    r1 = L.mm_autotune_runs()
    b = Plan(prob)
    r2 = L.mm_autotune_runs()
    assert r1 == r0 + 1 and r2 == r1
    assert a.tiles() == b.tiles()
    c = Plan(dict(prob, n=(1, 8, 256)))
    assert L.mm_autotune_runs() == r2 + 1
    for p in (a, b, c):
        p.close()
