"""The specialised C2R epilogues against the general one on the same problem.

A single-simulation plan with no per-cell mask and no thermal or spin-transfer term runs
the LEAN instantiation of the C2R + epilogue kernels, four-step or mixed-radix (those terms
compiled out, 32-bit exchange offsets).  An all-ones Msat mask changes no result: every mask factor is
1.0, the exchange weight 2ab/(a+b) of two unit ratios is 1.0 and the normalisation keeps
its norm map of 1.0.  But it sends the same plan through the general kernels.  Torques and
RK23 trajectories of the two plans must therefore agree bit for bit, and the LEAN torque
must match the FP64 oracle within the field tolerance (1e-5 relative).
"""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu

TOL_TORQUE = 1e-5

CASES = [
    # 3-D films whose padded rows are powers of two (the four-step passes)
    dict(n=(4, 32, 64), cell=(2e-9, 4e-9, 4e-9)),
    dict(n=(16, 64, 64), cell=(2e-9, 4e-9, 4e-9)),
    # periodic in-plane exchange and demag images
    dict(n=(2, 32, 32), cell=(3e-9, 4e-9, 4e-9), pbc=(0, 1, 1)),
    # padded sizes that are not powers of two (L = 6 x 40 x 56): the mixed-radix C2R pass
    dict(n=(3, 20, 28), cell=(2e-9, 4e-9, 4e-9)),
]


def _problem(case):
    import oracle as O
    return O.full_desc(demag=1, exchange=1, anis=1, zeeman=1, msat=8e5, aex=1.3e-11, ku=5e5,
                       anisu=(0.0, 0.6, 0.8), alpha=0.1, bext=(0.01, -0.02, 0.03), **case)


@pytest.mark.parametrize("case", CASES)
def test_lean_torque_bit_identical_and_oracle(case):
    import oracle as O
    from mumax2 import Plan
    prob = _problem(case)
    N = int(np.prod(prob["n"]))
    lean = Plan(prob)
    gen = Plan(prob, masks={"msat": np.ones(N, np.float32)})
    m = rand_m(prob["n"], seed=5)
    tl, _ = lean.torque(m)
    tg, _ = gen.torque(m)
    a, b = to_np(tl), to_np(tg)
    assert np.array_equal(a, b), np.abs(a - b).max()
    ref, _, _ = O.Oracle(prob).torque(m)
    assert rel_err(a, ref) < TOL_TORQUE
    lean.close()
    gen.close()


@pytest.mark.parametrize("case", CASES[:2] + CASES[3:])
def test_lean_rk23_steps_bit_identical(case):
    from mumax2 import Plan
    prob = _problem(case)
    N = int(np.prod(prob["n"]))
    lean = Plan(prob)
    gen = Plan(prob, masks={"msat": np.ones(N, np.float32)})
    m = rand_m(prob["n"], seed=9)
    for g in (lean, gen):
        g.solver("rk23", dt=1e-14, maxerr=1e-5)
        g.set_state(m)
        g.steps(12)
    sl, sg = lean.stats(), gen.stats()
    assert (sl["step"], sl["badsteps"], sl["evals"]) == (sg["step"], sg["badsteps"], sg["evals"])
    assert sl["t"] == sg["t"] and sl["dt"] == sg["dt"]
    assert np.array_equal(lean.get_state(), gen.get_state())
    assert lean.maxtorque() == gen.maxtorque()
    lean.close()
    gen.close()


def _steps_equal(pa, pb, m, solver="rk23", n=12):
    for g in (pa, pb):
        g.solver(solver, dt=1e-14, maxerr=1e-5)
        g.set_state(m)
        g.steps(n)
    sa, sb = pa.stats(), pb.stats()
    assert (sa["step"], sa["badsteps"], sa["evals"]) == (sb["step"], sb["badsteps"], sb["evals"])
    assert sa["t"] == sb["t"] and sa["dt"] == sb["dt"]
    assert np.array_equal(pa.get_state(), pb.get_state())


def test_unmasked_zhang_li_film_matches_general():
    """A Zhang-Li film without masks or thermal term runs the kernel with masks and thermal
    compiled out (spin-transfer kept); an all-ones Msat mask sends it through the general
    kernel.  Torques and RK23 steps agree bit for bit, the torque with the oracle to 1e-5."""
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(n=(4, 32, 64), cell=(2e-9, 4e-9, 4e-9), demag=1, exchange=1, zhangli=1, msat=8.6e5,
                       aex=1.3e-11, alpha=0.02, zl_pol=0.5, xi=0.05, j=(0.0, 2e11, 1e12))
    N = int(np.prod(prob["n"]))
    spec = Plan(prob)
    gen = Plan(prob, masks={"msat": np.ones(N, np.float32)})
    m = rand_m(prob["n"], seed=13)
    a, b = to_np(spec.torque(m)[0]), to_np(gen.torque(m)[0])
    assert np.array_equal(a, b), np.abs(a - b).max()
    ref, _, _ = O.Oracle(prob).torque(m)
    assert rel_err(a, ref) < TOL_TORQUE
    _steps_equal(spec, gen, m)
    spec.close()
    gen.close()


def test_masked_film_without_thermal_matches_general():
    """A masked film without thermal and spin-transfer terms runs the kernel with those two
    compiled out (masks kept); the same film with a thermal term at T = 0 (zero noise) runs
    the general kernel.  Torques and RK23 steps agree bit for bit."""
    import oracle as O
    from mumax2 import Plan
    base = dict(n=(4, 32, 64), cell=(2e-9, 4e-9, 4e-9), demag=1, exchange=1, anis=1, zeeman=1, msat=8e5,
                aex=1.3e-11, ku=5e5, anisu=(0.0, 0.6, 0.8), alpha=0.1, bext=(0.01, -0.02, 0.03))
    N = int(np.prod(base["n"]))
    rng = np.random.default_rng(3)
    msat = rng.uniform(0.5, 1.5, N).astype(np.float32)
    msat[rng.random(N) < 0.1] = 0.0
    masks = {"msat": msat}
    spec = Plan(O.full_desc(**base), masks=masks)
    gen = Plan(O.full_desc(thermal=1, temp=0.0, **base), masks=masks)
    m = rand_m(base["n"], seed=17)
    # a thermal time step > 0 keeps the zero-temperature noise scale finite (0 / dt)
    a, b = to_np(spec.torque(m, dt_thermal=1e-13)[0]), to_np(gen.torque(m, dt_thermal=1e-13)[0])
    assert np.array_equal(a, b), np.abs(a - b).max()
    _steps_equal(spec, gen, m)
    spec.close()
    gen.close()

