"""Seeded synthetic workloads of the batched path (host-side generators, no GPU).

Thermal ensemble: `nsim` independent simulations whose grid is drawn by seed from five
sizes (user x*y*z: 32x32x1, 64x32x1, 64x64x1, 128x64x2, 128x128x4) with 4x4x3 nm cells;
per simulation Ms ~ U[4e5, 1.2e6] A/m, Aex ~ U[5e-12, 2e-11] J/m, alpha ~ U[0.01, 0.1],
an applied field of magnitude U[0, 50] mT along a direction uniform on the sphere,
T = 300 K and its own thermal seed; stochastic Heun at a fixed 50 fs.  The initial state
of each simulation is uniform along a seeded direction.

Everything is in the engine's internal axis order (Z,Y,X): user (x, y, z) sizes become
n = (z, y, x) and vectors are stored as (z, y, x) components.
"""
import numpy as np

ENSEMBLE_GRIDS_USER = [(32, 32, 1), (64, 32, 1), (64, 64, 1), (128, 64, 2), (128, 128, 4)]
ENSEMBLE_CELL_USER = (4e-9, 4e-9, 3e-9)
ENSEMBLE_DT = 50e-15
ENSEMBLE_TEMP = 300.0


def _internal(v):
    return (v[2], v[1], v[0])


def ensemble(nsim=2048, seed=0):
    """Returns a list of grid classes, each a dict with
    n (internal), cell (internal), problem (base problem dict), sims (list of per-sim
    scalar dicts), ids (the simulations' indices in 0..nsim-1) and m0 (list of initial
    directions, internal order)."""
    rng = np.random.default_rng(seed)
    cls = rng.integers(0, len(ENSEMBLE_GRIDS_USER), size=nsim)
    ms = rng.uniform(4e5, 1.2e6, size=nsim)
    aex = rng.uniform(5e-12, 2e-11, size=nsim)
    alpha = rng.uniform(0.01, 0.1, size=nsim)
    bmag = rng.uniform(0.0, 0.05, size=nsim)
    bdir = rng.normal(size=(nsim, 3))
    bdir /= np.linalg.norm(bdir, axis=1, keepdims=True)
    mdir = rng.normal(size=(nsim, 3))
    mdir /= np.linalg.norm(mdir, axis=1, keepdims=True)
    out = []
    for c, grid in enumerate(ENSEMBLE_GRIDS_USER):
        ids = np.nonzero(cls == c)[0]
        if len(ids) == 0:
            continue
        n = _internal(grid)
        cell = _internal(ENSEMBLE_CELL_USER)
        problem = dict(n=n, cell=cell, pbc=(0, 0, 0), demag=1, exchange=1, zeeman=1, anis=0, thermal=1,
                       demag_accuracy=6, msat=float(ms[ids[0]]), aex=float(aex[ids[0]]),
                       alpha=float(alpha[ids[0]]), gamma=2.211e5, temp=ENSEMBLE_TEMP)
        sims, m0 = [], []
        for i in ids:
            b = bmag[i] * bdir[i]
            sims.append(dict(msat=float(ms[i]), aex=float(aex[i]), alpha=float(alpha[i]),
                             bext=tuple(float(x) for x in _internal(b)), ku=0.0, anisu=(0.0, 0.0, 1.0),
                             temp=ENSEMBLE_TEMP, seed=int(seed) * 1_000_003 + int(i)))
            m0.append(tuple(float(x) for x in _internal(mdir[i])))
        out.append(dict(n=n, cell=cell, problem=problem, sims=sims, ids=ids, m0=m0))
    return out


def uniform_state(n, direction, count=1):
    """SoA state of `count` simulations, each uniform along its direction."""
    N = int(n[0]) * int(n[1]) * int(n[2])
    dirs = np.atleast_2d(np.asarray(direction, dtype=np.float32))
    if dirs.shape[0] == 1 and count > 1:
        dirs = np.repeat(dirs, count, axis=0)
    return np.concatenate([np.repeat(d[:, None], N, axis=1).ravel() for d in dirs]).astype(np.float32)


def cells_of(classes):
    return sum(int(np.prod(c["n"])) * len(c["sims"]) for c in classes)
