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


def em_config(n=13, boundary="DDDDDD", ppc=4, te_ev=5.0e3, density=1.0e12, courant=0.5, precision=None,
              boxes=None, photo=False, obj_parser=None):
    """An EM-mode configuration: electrons of te_ev and 1 eV ions (mass 100) at
    `density`, dx = 0.5 m (below the Debye length of those electrons), dt =
    courant * dx / c (Environment::checkCFLCondition needs c dt / dx <= 1);
    electrons move ~0.05 cells per step. boxes: voxel conductors (as
    config.objects_from_boxes)."""
    from fopis_b200 import _abi, config
    from fopis_b200.config import SpeciesInfo, make_params
    dx = 0.5
    dt = courant * dx / config.CLIGHT
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, density, te_ev, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, density, 1.0, ppc)]
    shine = (0.0, 0.0, 0.0)
    if photo:
        import math
        vbar = math.sqrt(8.0 * 10.0 * config.E / (math.pi * config.ME))
        sp.append(SpeciesInfo("Photo", "photoelectron", 1.0, -1.0, density, 10.0, ppc,
                              current_density=10.0 * config.E * density * vbar / 4.0))
        shine = (-1.0, 0.0, 0.0)
    p, norm = make_params((n, n, n), boundary, dx, dt, sp, tol=1e-10, sort_interval=1000000, shine=shine,
                          precision=_abi.FP64 if precision is None else precision, solver="EM")
    objs = []
    if boxes:
        emit = next((k for k, s in enumerate(sp) if s.kind == "photoelectron"), -1)
        objs.append(config.objects_from_boxes(boxes, (n, n, n), emit_species=emit, obj_parser=obj_parser))
    return config.SimConfig(params=p, norm=norm, species=sp, objects=objs, dx=dx, dt=dt)
