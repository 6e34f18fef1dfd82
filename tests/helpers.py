"""Shared helpers of the test-suite: seeded inputs and error measures."""
import numpy as np


def rand_m(n, seed, kind="sphere"):
    """Seeded magnetisation, internal order SoA (3*N,) float64."""
    rng = np.random.default_rng(seed)
    N = int(n[0]) * int(n[1]) * int(n[2])
    if kind == "sphere":
        v = rng.normal(size=(3, N))
    elif kind == "near_x":   # user x = internal component 2
        v = np.zeros((3, N))
        v[2] = 1.0
        v[1] = 0.1
        v += 0.01 * rng.uniform(-1, 1, size=(3, N))
    else:
        raise ValueError(kind)
    v /= np.linalg.norm(v, axis=0, keepdims=True)
    return v.ravel()


def rel_err(a, b):
    """max |a - b| / max |b| over all entries."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max()
    if den == 0:
        return float(np.abs(a).max())
    return float(np.abs(a - b).max() / den)


def to_np(t):
    try:
        return t.detach().cpu().numpy().astype(np.float64)
    except AttributeError:
        return np.asarray(t, dtype=np.float64)
