"""Shared test helpers: synthetic particle sets and particle matching."""
from __future__ import annotations

import numpy as np

from fopis_b200 import PARTICLE_DTYPE


def random_particles(n, lo, hi, sigma, seed, species=0, drift=(0.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, PARTICLE_DTYPE)
    for a, key in enumerate("xyz"):
        r[key] = rng.uniform(lo[a], hi[a], n)
    for a, key in enumerate(("vx", "vy", "vz")):
        r[key] = drift[a] + sigma * rng.standard_normal(n)
    r["typeId"] = species
    r["isValid"] = 1
    return r


def as_f32_state(recs):
    """What the GPU holds after loading FP64 records: cell i = floor(x)+1 and an FP32 offset."""
    out = recs.copy()
    for key in ("x", "y", "z"):
        f = np.floor(out[key])
        o = (out[key] - f).astype(np.float32)
        out[key] = f + o.astype(np.float64)
    for key in ("vx", "vy", "vz"):
        out[key] = out[key].astype(np.float32).astype(np.float64)
    return out


def match(a, b, vscale=10.0):
    """Pairs records of a with their nearest records of b in (x, y, z, s*v) space;
    returns (a_sorted, b_matched) and asserts the pairing is one-to-one."""
    from scipy.spatial import cKDTree
    assert len(a) == len(b), (len(a), len(b))
    pa = np.stack([a["x"], a["y"], a["z"], vscale * a["vx"], vscale * a["vy"], vscale * a["vz"]], 1)
    pb = np.stack([b["x"], b["y"], b["z"], vscale * b["vx"], vscale * b["vy"], vscale * b["vz"]], 1)
    d, idx = cKDTree(pb).query(pa)
    assert len(np.unique(idx)) == len(idx), "particle matching is not one-to-one"
    return a, b[idx], d


def rel_err(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
