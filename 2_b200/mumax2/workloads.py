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


def partition(weights, world):
    """Contiguous blocks of items, one per rank, balanced by weight: rank r takes the items
    whose weight prefix (the sum up to and including the item's midpoint) falls in the r-th
    of `world` equal parts.  Returns [(start, end)] per rank (end exclusive)."""
    w = np.asarray(weights, dtype=np.float64)
    if world <= 1 or len(w) == 0:
        return [(0, len(w))] + [(len(w), len(w))] * max(0, world - 1)
    mid = np.cumsum(w) - 0.5 * w
    owner = np.minimum((mid / w.sum() * world).astype(int), world - 1)
    out = []
    for r in range(world):
        idx = np.nonzero(owner == r)[0]
        if len(idx):
            out.append((int(idx[0]), int(idx[-1]) + 1))
        else:
            prev = out[-1][1] if out else 0
            out.append((prev, prev))
    return out


def ensemble_shard(nsim, seed, rank, world):
    """This rank's share of the ensemble of `nsim` simulations (ensemble(nsim, seed), drawn
    identically on every rank): a contiguous block of simulation indices balanced by cells
    per simulation (the byte model of a Heun step is proportional to the cells), the grid
    classes restricted to it.  Returns (classes, (start, end))."""
    full = ensemble(nsim, seed=seed)
    cells = np.zeros(nsim)
    for c in full:
        cells[c["ids"]] = float(np.prod(c["n"]))
    lo, hi = partition(cells, world)[rank]
    out = []
    for c in full:
        keep = [k for k, i in enumerate(c["ids"]) if lo <= i < hi]
        if not keep:
            continue
        d = dict(c)
        d["ids"] = c["ids"][keep]
        d["sims"] = [c["sims"][k] for k in keep]
        d["m0"] = [c["m0"][k] for k in keep]
        out.append(d)
    return out, (lo, hi)


def gather_per_sim(dist, ids, rows, nsim):
    """Per-simulation result rows of every rank, gathered to rank 0 in simulation order
    (one all-gather of a few KB over the process group; None on the other ranks)."""
    payload = (np.asarray(ids, dtype=np.int64), np.asarray(rows, dtype=np.float64))
    world = dist.get_world_size()
    parts = [None] * world
    dist.all_gather_object(parts, payload)
    if dist.get_rank() != 0:
        return None
    width = payload[1].shape[1] if payload[1].ndim > 1 else 1
    out = np.full((nsim, width), np.nan)
    for pid, prow in parts:
        out[pid] = np.asarray(prow).reshape(len(pid), width)
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


# ---------------------------------------------------------------- relaxation set
RELAX_GRID_USER = (64, 64, 1)
RELAX_CELL_USER = (4e-9, 4e-9, 3e-9)


def geometry_mask(rng, nx, ny):
    """1-3 ellipses or rectangles (union) filling 40-100 % of the nx x ny film; returns a
    float32 [ny][nx] 0/1 mask.  Shapes are redrawn until the fill is in range."""
    yy, xx = np.mgrid[0:ny, 0:nx]
    xx = (xx + 0.5) / nx
    yy = (yy + 0.5) / ny
    for _ in range(1000):
        m = np.zeros((ny, nx), dtype=bool)
        for _ in range(int(rng.integers(1, 4))):
            cx, cy = rng.uniform(0.2, 0.8, size=2)
            ax, ay = rng.uniform(0.25, 0.75, size=2)
            if rng.uniform() < 0.5:
                m |= ((xx - cx) / ax) ** 2 + ((yy - cy) / ay) ** 2 <= 1.0
            else:
                m |= (np.abs(xx - cx) <= ax / 2) & (np.abs(yy - cy) <= ay / 2)
        fill = m.mean()
        if 0.4 <= fill <= 1.0:
            return m.astype(np.float32)
    raise RuntimeError("no mask with 40-100 % fill")


def relax_set(nsim, seed=0):
    """Seeded relaxation problems on 64x64x1 films of 4x4x3 nm cells: a geometry mask,
    Ms ~ U[4e5, 1.2e6], Aex ~ U[5e-12, 2e-11], Ku1 ~ U[0, 5e5] along an in-plane axis,
    |B| ~ U[0, 100] mT at an in-plane angle.  Returns (problem, sims, masks [nsim][N]) with
    the relax damping alpha = 1."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = RELAX_GRID_USER
    n = (nz, ny, nx)
    problem = dict(n=n, cell=_internal(RELAX_CELL_USER), pbc=(0, 0, 0), demag=1, exchange=1, zeeman=1, anis=1,
                   thermal=0, demag_accuracy=6, msat=8e5, aex=1.3e-11, alpha=1.0, gamma=2.211e5)
    sims, masks = [], []
    for i in range(nsim):
        masks.append(geometry_mask(rng, nx, ny).ravel())
        ms = rng.uniform(4e5, 1.2e6)
        aex = rng.uniform(5e-12, 2e-11)
        ku = rng.uniform(0.0, 5e5)
        phi_u = rng.uniform(0, 2 * np.pi)
        bmag = rng.uniform(0.0, 0.1)
        phi_b = rng.uniform(0, 2 * np.pi)
        u = (np.cos(phi_u), np.sin(phi_u), 0.0)            # user (x, y, z)
        b = (bmag * np.cos(phi_b), bmag * np.sin(phi_b), 0.0)
        sims.append(dict(msat=float(ms), aex=float(aex), alpha=1.0, ku=float(ku),
                         anisu=tuple(float(x) for x in _internal(u)),
                         bext=tuple(float(x) for x in _internal(b)), temp=0.0, seed=int(seed) * 1_000_003 + i))
    return problem, sims, masks


def cold_state(n, count):
    """The uninformed start of a plain relax: uniform along user +x (internal component 2)."""
    return uniform_state(n, (0.0, 0.0, 1.0), count)


# ---------------------------------------------------------------- single-simulation configs
def sp4_film(seed=0):
    """128x32x1 film of 3.90625x3.90625x3 nm (the SP4 geometry): Ms 8e5, Aex 1.3e-11,
    alpha 0.02; m = (1, 0.1, 0) + seeded uniform noise of amplitude 0.01, renormalised;
    an in-plane field of seeded magnitude U[10, 30] mT at a seeded angle.  Returns
    (problem, m0) in internal order."""
    rng = np.random.default_rng(seed)
    n = (1, 32, 128)
    N = 32 * 128
    bmag = rng.uniform(0.01, 0.03)
    phi = rng.uniform(0, 2 * np.pi)
    b_user = (bmag * np.cos(phi), bmag * np.sin(phi), 0.0)
    problem = dict(n=n, cell=(3e-9, 3.90625e-9, 3.90625e-9), pbc=(0, 0, 0), demag=1, exchange=1, zeeman=1,
                   msat=8e5, aex=1.3e-11, alpha=0.02, gamma=2.211e5, bext=_internal(b_user))
    m = np.zeros((3, N))
    m[2] = 1.0   # user x
    m[1] = 0.1   # user y
    m += 0.01 * rng.uniform(-1, 1, size=(3, N))
    m /= np.linalg.norm(m, axis=0, keepdims=True)
    return problem, m.astype(np.float32).ravel()


def neel_wall_strip(seed=0, current=1e12):
    """512x128x1 strip of 2 nm cells: Ms 8.6e5, Aex 1.3e-11, alpha 0.02, a Neel wall
    m_x = -tanh((x - x0)/20 nm), m_y = sech((x - x0)/20 nm) with x0 ~ U[300, 700] nm, and
    Zhang-Li torque with j along x (P 0.5, xi 0.05).  Returns (problem, m0, x0)."""
    rng = np.random.default_rng(seed)
    nx, ny = 512, 128
    x0 = rng.uniform(300e-9, 700e-9)
    x = (np.arange(nx) + 0.5) * 2e-9
    u = (x - x0) / 20e-9
    mx, my = -np.tanh(u), 1.0 / np.cosh(u)
    m = np.zeros((3, 1, ny, nx))
    m[2] = mx[None, None, :]
    m[1] = my[None, None, :]
    problem = dict(n=(1, ny, nx), cell=(2e-9, 2e-9, 2e-9), pbc=(0, 0, 0), demag=1, exchange=1, zhangli=1,
                   msat=8.6e5, aex=1.3e-11, alpha=0.02, gamma=2.211e5, zl_pol=0.5, xi=0.05,
                   j=(0.0, 0.0, float(current)))
    return problem, m.astype(np.float32).ravel(), x0


def wall_position(avg_mx_user, length):
    """Position of a +x | -x wall from <m_x>: <m_x> = (2 x_w - L) / L."""
    return 0.5 * length * (1.0 + avg_mx_user)
