"""The Newell demag tensor of the oracle (test infrastructure) against known answers.

The tensor is N_ab = 1/(4 pi V) times the 27-point difference of Newell, Williams &
Dunlop's f (diagonal) and g (off-diagonal) within 8 largest-cell-edges, and the
cell-averaged dipole tensor by Gauss quadrature beyond; the plans use K = -N.  Pinned
here by: the self term of a cube (-1/3), the unit trace of any cell's self term, the
symmetry K_ab = K_ba, the thin-film limit (sum of K_zz over a wide film -> -1), the
far-field quadrature against the closed form evaluated in 80-bit long double, and the
reference's own tensor (Kernel_Arne), which integrates the same physics with a finite
number of points (agreement to about 1e-3 of the largest element).
"""
import math

import numpy as np

import oracle as O

LD = np.longdouble


def _f(x, y, z):
    x2, y2, z2 = x * x, y * y, z * z
    R = np.sqrt(x2 + y2 + z2)
    r = (2 * x2 - y2 - z2) * R / 6
    if x2 + z2 > 0:
        r += y / 2 * (z2 - x2) * np.arcsinh(y / np.sqrt(x2 + z2))
    if x2 + y2 > 0:
        r += z / 2 * (y2 - x2) * np.arcsinh(z / np.sqrt(x2 + y2))
    if x != 0:
        r -= x * y * z * np.arctan(y * z / (x * R))
    return r


def _g(x, y, z):
    x2, y2, z2 = x * x, y * y, z * z
    R = np.sqrt(x2 + y2 + z2)
    r = -x * y * R / 3
    if x2 + y2 > 0:
        r += x * y * z * np.arcsinh(z / np.sqrt(x2 + y2))
    if y2 + z2 > 0:
        r += y / 6 * (3 * z2 - y2) * np.arcsinh(x / np.sqrt(y2 + z2))
    if x2 + z2 > 0:
        r += x / 6 * (3 * z2 - x2) * np.arcsinh(y / np.sqrt(x2 + z2))
    if z != 0:
        r -= z * z2 / 6 * np.arctan(x * y / (z * R))
    if y != 0:
        r -= z * y2 / 2 * np.arctan(x * z / (y * R))
    if x != 0:
        r -= z * x2 / 2 * np.arctan(y * z / (x * R))
    return r


def _newell_ld(F, X, d):
    """Closed-form N at offset X (units of cells scaled to the largest edge), long double."""
    X = [LD(v) for v in X]
    d = [LD(v) for v in d]
    s = LD(0)
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            for k in (-1, 0, 1):
                w = LD((2 if i == 0 else -1) * (2 if j == 0 else -1) * (2 if k == 0 else -1))
                s += w * F(X[0] + i * d[0], X[1] + j * d[1], X[2] + k * d[2])
    return s / (4 * LD(math.pi) * d[0] * d[1] * d[2])


def test_self_terms():
    K = O.kernel_newell((1, 2, 2), (1e-9, 1e-9, 1e-9))[:, :, 0, 0, 0]
    assert np.abs(K - (-np.eye(3) / 3)).max() < 1e-15
    K = O.kernel_newell((1, 2, 2), (2e-9, 4e-9, 5e-9))[:, :, 0, 0, 0]
    assert abs(np.trace(K) + 1) < 1e-14
    assert np.abs(K - np.diag(np.diag(K))).max() < 1e-15
    assert K[0, 0] < K[1, 1] < K[2, 2] < 0   # the thinnest axis demagnetises most


def test_symmetry_and_thin_film_limit():
    K = O.kernel_newell((4, 16, 32), (2e-9, 3e-9, 5e-9))
    for a in range(3):
        for b in range(3):
            assert np.array_equal(K[a, b], K[b, a])
    film = O.kernel_newell((1, 512, 512), (3e-9, 3e-9, 3e-9))
    assert abs(film[0, 0].sum() + 1) < 2e-3          # perpendicular: -1
    assert abs(film[1, 1].sum()) < 2e-3 and abs(film[2, 2].sum()) < 2e-3


def test_far_field_quadrature_against_long_double_closed_form():
    # the oracle switches to the dipole quadrature at 8 edges; compare there and beyond
    L = (32, 64, 64)
    cell = (2e-9, 4e-9, 4e-9)
    K = O.kernel_newell(L, cell)
    d = [c / max(cell) for c in cell]
    kmax = np.abs(K).max()
    worst = 0.0
    for (x, y, z) in [(0, 8, 1), (3, 6, 5), (5, 7, 4), (9, 12, 3), (15, 20, 20), (1, 31, 0)]:
        X = (x * d[0], y * d[1], z * d[2])
        want = [-_newell_ld(_f, X, d), -_newell_ld(_f, (X[1], X[0], X[2]), (d[1], d[0], d[2])),
                -_newell_ld(_g, X, d)]
        got = [K[0, 0, x, y, z], K[1, 1, x, y, z], K[0, 1, x, y, z]]
        for gv, wv in zip(got, want):
            worst = max(worst, abs(float(gv - wv)) / kmax)
    print("far-field quadrature vs long-double closed form, max |diff| / max |K|:", worst)
    assert worst < 1e-12


def test_newell_against_kernel_arne():
    L = (8, 64, 64)
    cell = (2e-9, 4e-9, 4e-9)
    Kn = O.kernel_newell(L, cell)
    Ka = O.kernel_arne(L, cell, (0, 0, 0), 6)
    diff = np.abs(Kn - Ka).max() / np.abs(Kn).max()
    print("Newell vs Kernel_Arne (accuracy 6), max |diff| / max |K|:", diff)
    assert diff < 3e-3


def test_periodic_images_accumulate():
    # a periodic axis sums the images: the tensor along that axis repeats with period L
    Kp = O.kernel_newell((1, 16, 8), (3e-9, 3e-9, 3e-9), (0, 1, 0))
    Ko = O.kernel_newell((1, 16, 8), (3e-9, 3e-9, 3e-9), (0, 0, 0))
    assert not np.allclose(Kp, Ko)
    assert np.abs(Kp[0, 0, 0, 1] - Kp[0, 0, 0, -1]).max() < 1e-15   # even in y
