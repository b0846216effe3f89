"""Shared test inputs: seeded, smooth, float-exact initial states that exercise every term
of the step (flow in all three directions, all pi components, bulk)."""
import numpy as np


def f32(a):
    return np.asarray(a, np.float64).astype(np.float32).astype(np.float64)


def rich_state(lat, seed=0, vel=0.1, pi=0.05, e0=60.0, emin=0.5, spacing=0.3):
    """Primitive fields on the ghosted lattice of `lat` (any object with nx.., ncx.., shear, bulk)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = lat.nx, lat.ny, lat.nz
    x = (np.arange(lat.ncx) - 2 - (nx - 1) / 2) * spacing
    y = (np.arange(lat.ncy) - 2 - (ny - 1) / 2) * spacing
    z = (np.arange(lat.ncz) - 2 - (nz - 1) / 2) * spacing
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    e = e0 * np.exp(-(X ** 2 + 1.3 * Y ** 2) / 8) * np.exp(-Z ** 2 / 2) + emin
    ux = f32(vel * np.tanh(X) * np.exp(-Y ** 2 / 8))
    uy = f32(vel * 0.7 * np.tanh(Y))
    un = f32(vel * 0.2 * np.tanh(Z))
    ut = np.sqrt(1 + ux ** 2 + uy ** 2 + (0.5 ** 2) * un ** 2)
    prim = dict(e=f32(e), ut=ut, ux=ux, uy=uy, un=un)
    if lat.shear:
        p = e / 3
        for k in ["pitt", "pitx", "pity", "pitn", "pixx", "pixy", "pixn", "piyy", "piyn", "pinn"]:
            prim[k] = f32(pi * p * rng.uniform(-1, 1, e.shape) * (0.3 if k.startswith("pit") else 1.0))
    if lat.bulk:
        prim["Pi"] = f32(-pi * 0.3 * e / 3)
    return {k: v.reshape(-1) for k, v in prim.items()}


def rel_err(a, b):
    """max |a-b| / max |b| over the cells (per-field scale-relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / scale)


def interior(lat, a):
    return np.asarray(a).reshape(lat.ncz, lat.ncy, lat.ncx)[2:-2, 2:-2, 2:-2]
