"""CPU tests that pin the FP64 oracle (no GPU).

- the reference's golden muMAG standard problem 4 trace (tests/stdsolution4.txt of
  mumax/2, subsampled into tests/golden by tests/golden/make_golden.py);
- known answers: thin-film demag, tensor symmetry, uniform exchange, precession sense
  and the analytic damped single-spin trajectory;
- Philox4x32-10 known-answer vectors of the published algorithm;
- Runge-Kutta tableau consistency and convergence order of the fixed-step solvers.
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import rand_m

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MU0 = 4e-7 * np.pi


def test_sp4_golden_trace():
    """Oracle RK12 run of the reference's tests/stdproblem4.py protocol against its
    golden <m>(t): relax 2 ns at alpha=1 from (1,1,0), then 1 ns at alpha=0.02 in
    B=(-24.6, 4.3, 0) mT, m_maxerror 1/3000, mindt 1e-15."""
    gold = np.loadtxt(os.path.join(GOLDEN, "sp4_stdsolution4.txt"))
    n = (1, 32, 128)
    N = 32 * 128
    base = dict(n=n, cell=(3e-9, 125e-9 / 32, 500e-9 / 128), demag=1, exchange=1, zeeman=1, msat=800e3,
                aex=1.3e-11)
    o = O.Oracle(dict(base, alpha=1.0))
    m = np.zeros(3 * N)
    m[N:2 * N] = 1
    m[2 * N:] = 1
    r = O.OracleRun(o, m, solver="rk12", dt=1e-15, mindt=1e-15, maxerr=1 / 3000)
    r.run(2e-9)
    o2 = O.Oracle(dict(base, alpha=0.02, bext=(0.0, 4.3e-3, -24.6e-3)))
    r2 = O.OracleRun(o2, r.m, solver="rk12", dt=1e-15, mindt=1e-15, maxerr=1 / 3000)
    rec = []
    r2.run(1e-9, record_every=10e-12, callback=lambda rr: rec.append((rr.st.t * 1e9, *o2.average(rr.m)[::-1])))
    rec = np.array(rec)
    assert abs(rec[0, 1] - gold[0, 1]) < 5e-3 and abs(rec[0, 2] - gold[0, 2]) < 5e-3  # relaxed S-state
    for c in range(3):
        gi = np.interp(rec[:, 0], gold[:, 0], gold[:, c + 1])
        d = np.abs(gi - rec[:, c + 1])
        print("component", c, "max", d.max(), "rms", np.sqrt((d ** 2).mean()))
        assert d.max() < 0.05 and np.sqrt((d ** 2).mean()) < 0.025


def test_kernel_symmetry_and_thin_film_limit():
    L = (1, 16, 16)
    K = O.kernel_arne(L, (2e-9, 3e-9, 3e-9))
    # upper and lower triangle agree to the integration accuracy (~2e-5 of the largest
    # element here); the reference keeps only the upper one (LoadKernel)
    for s in range(3):
        for d in range(3):
            assert np.abs(K[s, d] - K[d, s]).max() < 1e-4 * np.abs(K).max()
    # self term of a flat cell: N_zz (internal 0) dominates, trace of the self term = -1
    self_trace = K[0, 0, 0, 0, 0] + K[1, 1, 0, 0, 0] + K[2, 2, 0, 0, 0]
    assert abs(self_trace + 1.0) < 2e-3
    assert K[0, 0, 0, 0, 0] < K[1, 1, 0, 0, 0]


def test_uniform_film_demag_and_zero_exchange():
    n = (1, 64, 64)
    o = O.Oracle(dict(n=n, cell=(2e-9, 5e-9, 5e-9), demag=1, exchange=1, msat=1e6))
    N = 64 * 64
    m = np.zeros(3 * N)
    m[:N] = 1
    f = o.fields(m)
    hd = f["demag"].reshape(3, 64, 64)
    assert -1.0 < hd[0, 32, 32] / 1e6 < -0.95
    assert np.abs(f["ex"]).max() == 0.0


def test_precession_sense_and_damped_single_spin():
    # B along user +z (internal 0), m along user +x: dm/dt = -gamma m x H -> +y (user)
    B = 0.1
    o = O.Oracle(dict(n=(1, 1, 1), cell=(3e-9,) * 3, demag=0, exchange=0, zeeman=1, bext=(B, 0, 0), alpha=0.0))
    t, _, _ = o.torque(np.array([0.0, 0.0, 1.0]))
    assert t[1] > 0 and abs(t[0]) < 1e-9 and abs(t[2]) < 1e-9
    # damped: tan(theta/2) = tan(theta0/2) exp(-alpha gamma H t / (1+alpha^2))
    alpha, gam = 0.1, 2.211e5
    o = O.Oracle(dict(n=(1, 1, 1), cell=(3e-9,) * 3, demag=0, exchange=0, zeeman=1, bext=(B, 0, 0), alpha=alpha))
    th0 = 1.0
    m0 = np.array([np.cos(th0), 0.0, np.sin(th0)])
    r = O.OracleRun(o, m0, solver="rk45", dt=1e-14, maxerr=1e-8)
    T = 50e-12
    r.run(T)
    th = np.arccos(np.clip(r.m[0], -1, 1))
    H = B / MU0
    want = 2 * np.arctan(np.tan(th0 / 2) * np.exp(-alpha * gam * H * r.st.t / (1 + alpha ** 2)))
    assert abs(th - want) < 1e-6


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors (Salmon et al., SC'11, published with the
    algorithm) reproduced through the normal generator's raw 32-bit words."""
    import ctypes as C
    lib = O.lib()
    # expose the raw generator through a tiny restatement check: the normals of
    # (seed, cell, step) are a pure function of the Philox output, so instead the
    # reference vectors are checked by a local restatement bound to the same constants
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85

    def philox(c, k):
        c = list(c)
        k = list(k)
        for _ in range(10):
            p0 = M0 * c[0]
            p1 = M1 * c[2]
            c = [((p1 >> 32) ^ c[1] ^ k[0]) & 0xffffffff, p1 & 0xffffffff,
                 ((p0 >> 32) ^ c[3] ^ k[1]) & 0xffffffff, p0 & 0xffffffff]
            k = [(k[0] + W0) & 0xffffffff, (k[1] + W1) & 0xffffffff]
        return c
    assert philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
    # the oracle's normals follow from the same words
    seed, cell, step = 0x299f31d0a4093822, 17, 5
    w = philox([cell, step, 0, 0x7e57], [seed & 0xffffffff, seed >> 32])
    u = [((x >> 8) + 0.5) * 2.0 ** -24 for x in w]
    want = [np.sqrt(-2 * np.log(u[0])) * np.cos(2 * np.pi * u[1]),
            np.sqrt(-2 * np.log(u[0])) * np.sin(2 * np.pi * u[1]),
            np.sqrt(-2 * np.log(u[2])) * np.cos(2 * np.pi * u[3])]
    got = O.thermal_normals(seed, cell, step)
    assert np.allclose(got, want, rtol=0, atol=1e-14)
    del lib, C


def test_thermal_normals_statistics():
    x = np.array([O.thermal_normals(7, c, 3) for c in range(20000)]).ravel()
    assert abs(x.mean()) < 0.02 and abs(x.std() - 1) < 0.02


@pytest.mark.parametrize("solver,order", [("euler", 1), ("heun", 2)])
def test_fixed_step_convergence_order(solver, order):
    # single damped spin against the analytic solution, halving dt
    alpha, gam, B = 0.1, 2.211e5, 0.05
    o = O.Oracle(dict(n=(1, 1, 1), cell=(3e-9,) * 3, demag=0, exchange=0, zeeman=1, bext=(B, 0, 0), alpha=alpha))
    th0 = 1.2
    errs = []
    T = 20e-12
    for dt in [2e-14, 1e-14, 5e-15]:
        r = O.OracleRun(o, np.array([np.cos(th0), 0.0, np.sin(th0)]), solver=solver, dt=dt)
        while r.st.t < T - 1e-20:
            r.step()
        th = np.arccos(np.clip(r.m[0], -1, 1))
        want = 2 * np.arctan(np.tan(th0 / 2) * np.exp(-alpha * gam * (B / MU0) * r.st.t / (1 + alpha ** 2)))
        errs.append(abs(th - want))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    print(solver, errs, rates)
    assert all(abs(rt - order) < 0.3 for rt in rates)


def test_tableaux_consistency():
    import ctypes as C  # noqa: F401
    # row sums of the Dormand-Prince and Bogacki-Shampine stages give the nodes c
    DP_A = [[1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9],
            [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
            [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
            [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
    assert np.allclose([sum(r) for r in DP_A], [1 / 5, 3 / 10, 4 / 5, 8 / 9, 1, 1])
    bstar = [5179 / 57600, 0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]
    assert abs(sum(bstar) - 1) < 1e-15 and abs(sum(DP_A[-1]) - 1) < 1e-15


def test_energy_conservation_without_damping():
    n = (1, 8, 16)
    o = O.Oracle(dict(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, zeeman=1, bext=(0.01, 0.0, 0.02),
                      alpha=0.0))
    m = rand_m(n, 3, kind="near_x")
    e0 = o.energy(m)["E"]
    r = O.OracleRun(o, m, solver="rk45", dt=1e-15, maxerr=1e-7)
    r.run(5e-12)
    e1 = o.energy(r.m)["E"]
    assert abs(e1 - e0) < 1e-4 * abs(e0)


def test_relax_lowers_energy():
    n = (1, 8, 16)
    o = O.Oracle(dict(n=n, cell=(3e-9, 4e-9, 4e-9), demag=1, exchange=1, alpha=1.0))
    m = rand_m(n, 4)
    e0 = o.energy(m)["E"]
    r = O.OracleRun(o, m, solver="rk23", dt=1e-15, maxerr=1e-5)
    r.run(20e-12)
    assert o.energy(r.m)["E"] < e0


def test_demagexch_equals_demag_plus_exchange_in_the_interior():
    """Module demagexch (mod_demagexchange.go): away from the boundaries the combined
    convolution is the demag field plus the 6-neighbour exchange field; on a film the
    reference's kernel quirk (the size-1 dimension's neighbour writes replace the centre)
    only adds a field parallel to m, so the torque is unchanged."""
    import oracle as O
    from helpers import rand_m
    for n in [(1, 8, 16), (4, 8, 8)]:
        m = rand_m(n, 3)
        kw = dict(n=n, cell=(3e-9, 4e-9, 5e-9), demag=1, exchange=1, msat=8e5, aex=1.3e-11)
        a = O.Oracle(O.full_desc(**kw))
        b = O.Oracle(O.full_desc(demag_exchange=1, **kw))
        sl = (slice(None),) + tuple(slice(1, -1) if k > 2 else slice(None) for k in n)
        ta, _, _ = a.torque(m)
        tb, _, _ = b.torque(m)
        assert np.abs((ta - tb).reshape(3, *n)[sl]).max() < 1e-6 * np.abs(ta).max()
        if n[0] > 1:
            fa, fb = a.fields(m), b.fields(m)
            hs = (fa["demag"] + fa["ex"]).reshape(3, *n)
            assert np.abs(hs[sl] - fb["demag"].reshape(3, *n)[sl]).max() < 1e-6 * np.abs(hs).max()
