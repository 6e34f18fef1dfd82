"""GPU parity of the effective-field terms and the torque against the FP64 oracle.

Tolerance: FP32 arithmetic on the GPU against FP64 on the CPU; every field term must
agree to 1e-5 relative (max |difference| / max |oracle|), the bound stated for H_eff.
"""
import numpy as np
import pytest

from helpers import rand_m, rel_err, to_np

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-5
TOL_TORQUE = 1e-5


def _pair(problem, masks_host=None):
    import oracle as O
    from mumax2 import Plan
    prob = O.full_desc(**problem)
    if masks_host:
        prob["masks"] = masks_host
    o = O.Oracle(prob)
    g = Plan(prob, masks=masks_host or {})
    return o, g


@pytest.mark.parametrize("n,cell", [
    ((1, 16, 32), (3e-9, 4e-9, 5e-9)),       # 2-D film, 4 kernel components
    ((1, 32, 128), (3e-9, 3.90625e-9, 3.90625e-9)),  # SP4 geometry
    ((4, 8, 16), (2e-9, 4e-9, 4e-9)),        # 3-D, 6 components
    ((2, 4, 4), (4e-9, 4e-9, 3e-9)),         # tiny 3-D
    ((8, 16, 8), (3e-9, 3e-9, 3e-9)),
    # padded sizes that are not powers of two (mixed-radix passes): 2^n * {3, 5, 7}
    ((1, 24, 40), (3e-9, 4e-9, 5e-9)),       # L = 1 x 48 x 80
    ((3, 20, 28), (2e-9, 4e-9, 4e-9)),       # L = 6 x 40 x 56: every axis mixed
    ((1, 15, 21), (3e-9, 4e-9, 4e-9)),       # L = 1 x 30 x 42, odd row length 21
    ((5, 16, 32), (2e-9, 4e-9, 4e-9)),       # mixed z (L0 = 10) with power-of-two y, x
    ((2, 12, 64), (2e-9, 4e-9, 4e-9)),       # mixed y (L1 = 24) only
    ((1, 11, 26), (3e-9, 4e-9, 4e-9)),       # prime factors 11 and 13 (direct-DFT stages)
])
def test_demag_field(n, cell):
    o, g = _pair(dict(n=n, cell=cell, demag=1, exchange=0, msat=8e5))
    assert g.kernel_nonzero() == o.nonzero_components()
    m = rand_m(n, seed=1)
    ho = o.fields(m)["demag"]
    hg = to_np(g.fields(m)["demag"])
    err = rel_err(hg, ho)
    print("demag", n, err)
    assert err < TOL_FIELD


def test_demag_uniform_film_known_answer():
    # uniform out-of-plane magnetisation of a wide thin film: H_z ~ -Ms in the centre
    n = (1, 64, 64)
    o, g = _pair(dict(n=n, cell=(2e-9, 5e-9, 5e-9), demag=1, exchange=0, msat=1e6))
    N = 64 * 64
    m = np.zeros(3 * N)
    m[:N] = 1.0
    hg = to_np(g.fields(m)["demag"]).reshape(3, 64, 64)
    assert -1.0 < hg[0, 32, 32] / 1e6 < -0.95
    assert abs(hg[1, 32, 32]) < 1e-3 * 1e6


@pytest.mark.parametrize("n,pbc", [((3, 5, 7), (0, 0, 0)), ((1, 6, 9), (0, 1, 1)), ((4, 4, 4), (1, 0, 1)),
                                   ((1, 1, 16), (0, 0, 0))])
def test_exchange_with_masks(n, pbc):
    rng = np.random.default_rng(3)
    N = n[0] * n[1] * n[2]
    msat_mask = rng.uniform(0.5, 1.5, N).astype(np.float32)
    msat_mask[rng.random(N) < 0.1] = 0.0
    aex_mask = rng.uniform(0.5, 2.0, N).astype(np.float32)
    masks = dict(msat=msat_mask, aex=aex_mask)
    o, g = _pair(dict(n=n, cell=(2e-9, 3e-9, 4e-9), pbc=pbc, demag=0, exchange=1, msat=7e5, aex=1.1e-11), masks)
    m = o.normalize(rand_m(n, seed=2))
    ho = o.fields(m)["ex"]
    hg = to_np(g.fields(m)["ex"])
    err = rel_err(hg, ho)
    print("exchange", n, pbc, err)
    assert err < TOL_FIELD


def test_anisotropy_zeeman_masks():
    n = (2, 6, 10)
    rng = np.random.default_rng(4)
    N = 120
    masks = dict(msat=rng.uniform(0, 1, N).astype(np.float32), ku=rng.uniform(0, 2, N).astype(np.float32),
                 anisu=[rng.uniform(-1, 1, N), None, rng.uniform(-1, 1, N)],
                 bext=[None, rng.uniform(-1, 1, N), rng.uniform(0, 1, N)])
    masks["msat"][:7] = 0
    o, g = _pair(dict(n=n, cell=(3e-9, 3e-9, 3e-9), demag=0, exchange=0, anis=1, zeeman=1, ku=5e5,
                      anisu=(0.3, 0.5, 0.8), bext=(0.01, -0.02, 0.03), msat=1.1e6), masks)
    m = rand_m(n, seed=5)
    fo, fg = o.fields(m), g.fields(m)
    for k in ["anis", "zee"]:
        err = rel_err(to_np(fg[k]), fo[k])
        print(k, err)
        assert err < TOL_FIELD


def test_thermal_field_matches_oracle_noise():
    n = (1, 8, 12)
    o, g = _pair(dict(n=n, cell=(3e-9, 4e-9, 4e-9), demag=0, exchange=0, thermal=1, temp=300.0, alpha=0.05,
                      seed=1234))
    m = rand_m(n, seed=6)
    for step in [0, 1, 77, 2**33 + 5]:
        ho = o.fields(m, noise_step=step, dt_thermal=5e-14)["therm"]
        hg = to_np(g.fields(m, noise_step=step, dt_thermal=5e-14)["therm"])
        err = rel_err(hg, ho)
        print("thermal", step, err)
        assert err < 1e-5


def test_thermal_statistics():
    # the noise is standard normal per component and uncorrelated between steps
    n = (1, 64, 64)
    o, g = _pair(dict(n=n, cell=(3e-9, 4e-9, 4e-9), demag=0, exchange=0, thermal=1, temp=300.0, alpha=0.1,
                      seed=99))
    m = rand_m(n, seed=7)
    a = to_np(g.fields(m, noise_step=0, dt_thermal=1e-13)["therm"])
    b = to_np(g.fields(m, noise_step=1, dt_thermal=1e-13)["therm"])
    V = 3e-9 * 4e-9 * 4e-9
    sigma = np.sqrt(2 * 0.1 * 1.380650424e-23 * 300.0 / (4e-7 * np.pi * V * 2.211e5 * 1e-13 * 8e5))
    z = a / sigma
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.02
    assert abs(np.corrcoef(a, b)[0, 1]) < 0.03


@pytest.mark.parametrize("terms", [
    dict(demag=1, exchange=1, zeeman=1, bext=(0.0, 4.3e-3, -24.6e-3)),
    dict(demag=1, exchange=1, anis=1, ku=5e5, anisu=(1, 0, 0), alpha=0.1),
    dict(demag=0, exchange=1, zhangli=1, j=(0, 0, 1e12), zl_pol=0.5, xi=0.05),
    dict(demag=0, exchange=1, zhangli=1, j=(2e11, -1e12, 5e11), zl_pol=0.7, xi=0.1, pbc=(0, 1, 0)),
    dict(demag=1, exchange=1, slonczewski=1, j=(1e11, 0, 0), p=(1, 0, 0), sl_pol=0.5669, **{"lambda": 2.0},
         eps_prime=0.1, t_fl=3e-9),
])
def test_torque_parity(terms):
    n = (2, 8, 16)
    prob = dict(n=n, cell=(3e-9, 4e-9, 4e-9), msat=8.6e5, aex=1.3e-11, alpha=0.02)
    prob.update(terms)
    o, g = _pair(prob)
    m = rand_m(n, seed=8)
    to, _, _ = o.torque(m)
    tg, _ = g.torque(m)
    err = rel_err(to_np(tg), to)
    print("torque", terms, err)
    assert err < TOL_TORQUE


def test_stt_with_masks():
    n = (1, 12, 20)
    N = 240
    rng = np.random.default_rng(9)
    masks = dict(msat=(rng.random(N) > 0.2).astype(np.float32), j=[None, None, rng.uniform(0.5, 1.5, N)],
                 xi=rng.uniform(0.5, 1.5, N), zl_pol=rng.uniform(0.5, 1, N), alpha=rng.uniform(0.5, 2, N),
                 p=[rng.uniform(-1, 1, N), rng.uniform(-1, 1, N), rng.uniform(0.1, 1, N)],
                 t_fl=rng.uniform(0.5, 1.5, N), lambda_=None)
    masks.pop("lambda_")
    for kind in [dict(zhangli=1), dict(slonczewski=1, eps_prime=0.2, t_fl=2e-9, **{"lambda": 1.5})]:
        prob = dict(n=n, cell=(2e-9, 2e-9, 2e-9), demag=0, exchange=1, msat=8.6e5, j=(0.0, 0.0, 1e12), zl_pol=0.5,
                    xi=0.05, p=(0, 0, 1))
        prob.update(kind)
        o, g = _pair(prob, masks)
        m = o.normalize(rand_m(n, seed=10))
        to, _, _ = o.torque(m)
        tg, _ = g.torque(m)
        err = rel_err(to_np(tg), to)
        print("stt masks", kind, err)
        assert err < TOL_TORQUE


@pytest.mark.parametrize("n,pbc", [((1, 16, 32), (0, 0, 1)), ((1, 16, 32), (0, 1, 0)), ((1, 8, 16), (0, 1, 1)),
                                   ((4, 8, 16), (1, 0, 0)), ((2, 8, 8), (0, 1, 1)),
                                   ((1, 12, 36), (0, 1, 1)), ((6, 10, 24), (1, 0, 0)), ((1, 20, 24), (0, 0, 1))])
def test_demag_periodic(n, pbc):
    """Periodic dimensions are not padded (zeropad.go:12-22) and the tensor sums the
    periodic images (kernel_magnetostatic.go:55-65)."""
    o, g = _pair(dict(n=n, cell=(3e-9, 4e-9, 4e-9), pbc=pbc, demag=1, exchange=1, msat=8e5))
    assert g.kernel_nonzero() == o.nonzero_components()
    m = rand_m(n, seed=21)
    fo, fg = o.fields(m), g.fields(m)
    for k in ["demag", "ex"]:
        err = rel_err(to_np(fg[k]), fo[k])
        print("pbc", n, pbc, k, err)
        assert err < TOL_FIELD


@pytest.mark.parametrize("n,pbc,tensor", [((1, 16, 32), (0, 0, 0), "arne"), ((4, 8, 16), (0, 0, 0), "arne"),
                                          ((2, 8, 8), (0, 1, 1), "arne"), ((1, 8, 16), (0, 0, 1), "arne"),
                                          ((3, 12, 20), (0, 0, 0), "arne"), ((1, 16, 32), (0, 0, 0), "newell"),
                                          ((3, 10, 12), (0, 1, 0), "newell")])
def test_demagexch_field_and_torque(n, pbc, tensor):
    """Module demagexch: exchange folded into the demag kernel (mod_demagexchange.go), on
    power-of-two and mixed-radix grids, with either demag tensor."""
    prob = dict(n=n, cell=(3e-9, 4e-9, 4e-9), pbc=pbc, demag=1, exchange=1, msat=8e5, aex=1.3e-11,
                demag_exchange=1, demag_accuracy=8, demag_tensor=tensor)
    o, g = _pair(prob)
    assert g.kernel_nonzero()[:3] == [1, 1, 1]
    m = rand_m(n, seed=31)
    fo, fg = o.fields(m), g.fields(m)
    assert np.abs(to_np(fg["ex"])).max() == 0.0        # no separate stencil term
    err = rel_err(to_np(fg["demag"]), fo["demag"])
    print("dex", n, pbc, err)
    assert err < TOL_FIELD
    to, _, _ = o.torque(m)
    tg, _ = g.torque(m)
    assert rel_err(to_np(tg), to) < TOL_TORQUE
    # Aex and Ms enter the combined kernel: changing them rebuilds it
    import oracle as O
    prob2 = O.full_desc(**dict(prob, aex=2.0e-11, msat=6e5))
    g.set_problem(prob2)
    fo2 = O.Oracle(prob2).fields(m)
    assert rel_err(to_np(g.fields(m)["demag"]), fo2["demag"]) < TOL_FIELD


@pytest.mark.parametrize("kind", ["arne", "newell"])
@pytest.mark.parametrize("L,cell,pbc", [
    ((1, 32, 64), (3e-9, 3.90625e-9, 3.90625e-9), (0, 0, 0)),   # single-layer film
    ((8, 32, 32), (2e-9, 4e-9, 4e-9), (0, 0, 0)),               # 3-D, anisotropic cells
    ((1, 16, 32), (3e-9, 4e-9, 4e-9), (0, 1, 0)),               # periodic y images
    ((6, 20, 24), (2e-9, 3e-9, 5e-9), (1, 0, 0)),               # periodic z, even non-2^n sizes
])
def test_demag_tensor_fp64_matches_oracle(kind, L, cell, pbc):
    """The real-space FP64 tensor from the GPU (mm_demag_tensor) against the oracle's
    FP64 restatement of the same method, before any FP32 rounding: 1e-12 of the largest
    element."""
    import ctypes as C

    import oracle as O
    import torch
    from mumax2 import _native as nat
    NL = L[0] * L[1] * L[2]
    out = torch.full((6 * NL,), float("nan"), dtype=torch.float64, device="cuda")
    nat.check(nat.lib().mm_demag_tensor((C.c_int * 3)(*L), (C.c_double * 3)(*cell), (C.c_int * 3)(*pbc),
                                        nat.TENSORS[kind], 6, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    g = out.cpu().numpy().reshape(6, *L)
    K = O.kernel_newell(L, cell, pbc) if kind == "newell" else O.kernel_arne(L, cell, pbc, 6)
    o = np.stack([K[0, 0], K[1, 1], K[2, 2], K[1, 2], K[0, 2], K[0, 1]])
    err = np.abs(g - o).max() / np.abs(o).max()
    print(kind, L, pbc, "FP64 tensor GPU vs oracle, max |diff| / max |K|:", err)
    assert np.isfinite(g).all()
    assert err < 1e-12


@pytest.mark.parametrize("n,cell,pbc", [((1, 16, 32), (3e-9, 4e-9, 5e-9), (0, 0, 0)),
                                        ((4, 8, 16), (2e-9, 4e-9, 4e-9), (0, 0, 0)),
                                        ((1, 16, 16), (3e-9, 3e-9, 3e-9), (0, 1, 1))])
def test_demag_field_newell(n, cell, pbc):
    """The demag field of a plan built on the Newell tensor against the oracle's."""
    o, g = _pair(dict(n=n, cell=cell, pbc=pbc, demag=1, exchange=0, msat=8e5, demag_tensor="newell"))
    m = rand_m(n, seed=3)
    err = rel_err(to_np(g.fields(m)["demag"]), o.fields(m)["demag"])
    print("demag (Newell)", n, pbc, err)
    assert err < TOL_FIELD


def test_newell_minus_arne_per_configuration():
    """H_demag of the Newell tensor against the reference's Kernel_Arne, both on the GPU,
    for the grids and cells of every configuration (the seeded states of each), reported
    as max |H_newell - H_arne| / max |H_arne|.  The two integrate the same physics; Arne
    uses a finite number of face-charge points, so they differ at the 1e-3 level."""
    from mumax2 import Plan
    from mumax2 import workloads as W
    import bench
    cases = []
    prob, m0 = W.sp4_film(seed=0)
    cases.append(("film 128x32x1 (SP4 geometry)", prob, m0))
    cases.append(("film3d 256x256x16", bench.problem(), bench.initial_m(0)))
    prob, m0, _ = W.neel_wall_strip(seed=0)
    cases.append(("Neel wall 512x128x1", prob, m0))
    for nm, n in [("ensemble 128x128x4", (4, 128, 128)), ("relax 64x64x1", (1, 64, 64))]:
        cell = (3e-9, 4e-9, 4e-9)
        cases.append((nm, dict(n=n, cell=cell, demag=1, exchange=0, msat=8e5), rand_m(n, seed=5)))
    for nm, prob, m0 in cases:
        base = {k: v for k, v in prob.items() if k in ("n", "cell", "pbc", "msat")}
        base.update(demag=1, exchange=0, anis=0, zeeman=0, zhangli=0, slonczewski=0)
        ha = to_np(Plan(dict(base)).fields(m0)["demag"])
        hn = to_np(Plan(dict(base, demag_tensor="newell")).fields(m0)["demag"])
        d = rel_err(hn, ha)
        print(f"Newell - Kernel_Arne, {nm}: max |dH| / max |H| = {d:.3e}")
        assert d < 5e-3


def test_mixed_radix_batch_equals_single_plans():
    """A batched plan of two simulations on a grid with non-power-of-two padded sizes
    (3-D, 3 x 20 x 28 cells) gives each simulation the torque its own plan gives."""
    from mumax2 import Plan
    n = (3, 20, 28)
    prob = dict(n=n, cell=(2e-9, 4e-9, 4e-9), demag=1, exchange=1, anis=1, zeeman=1, msat=8e5, aex=1.3e-11,
                ku=2e5, anisu=(0.0, 0.6, 0.8), alpha=0.05, bext=(0.0, 0.01, 0.02))
    sims = [dict(msat=8e5, aex=1.3e-11, alpha=0.05, bext=(0.0, 0.01, 0.02), ku=2e5, anisu=(0.0, 0.6, 0.8)),
            dict(msat=6e5, aex=1.0e-11, alpha=0.1, bext=(0.02, 0.0, 0.0), ku=1e5, anisu=(1.0, 0.0, 0.0))]
    N = n[0] * n[1] * n[2]
    m = np.concatenate([rand_m(n, seed=40), rand_m(n, seed=41)])
    gb = Plan(prob, sims=sims)
    tb = to_np(gb.torque(m)[0])
    for b, sm in enumerate(sims):
        q = dict(prob)
        q.update(sm)
        ts = to_np(Plan(q).torque(m[3 * N * b:3 * N * (b + 1)])[0])
        err = rel_err(tb[3 * N * b:3 * N * (b + 1)], ts)
        print("mixed-radix batch vs single", b, err)
        assert err < 1e-6
