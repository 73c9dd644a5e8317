"""GPU sort: brick-then-cell order of the slots, no particle lost or changed,
and steps with a sort between each of them tracking the oracle.

A neutral blob of extra electrons and ions inside one 4x4x8 brick puts that
brick above the 8192 particles the cell pass orders in shared memory, so both
of its paths run.
"""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units

from helpers import as_f32_state, match, random_particles

pytestmark = pytest.mark.gpu

BX, BY, BZ = 4, 4, 8


def cfg_sorted(n=24, ppc=4, sort_interval=1):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, ppc)]
    p, norm = make_params((n, n, n), "PPPPPP", dx, dt, sp, tol=1e-10, sort_interval=sort_interval)
    return config.SimConfig(params=p, norm=norm, species=sp)


def with_blob(n, base, blob, seed, species):
    """Uniform particles plus `blob` more inside node cells 5..7 (x, y) and
    9..15 (z), all in brick (1, 1, 1)."""
    a = random_particles(base, (0, 0, 0), (n, n, n), 0.05, seed, species)
    b = random_particles(blob, (4.0, 4.0, 8.0), (6.99, 6.99, 14.99), 0.05, seed + 1, species)
    return np.concatenate([a, b])


def sort_keys(cell, n):
    i, j, k = (cell >> 20) & 1023, (cell >> 10) & 1023, cell & 1023
    nb = [(n + 2 - 1 + BX - 1) // BX, (n + 2 - 1 + BY - 1) // BY, (n + 2 - 1 + BZ - 1) // BZ]
    brick = ((i // BX) * nb[1] + (j // BY)) * nb[2] + (k // BZ)
    local = ((i % BX) * BY + (j % BY)) * BZ + (k % BZ)
    return brick.astype(np.int64) * (BX * BY * BZ) + local


def records(cell, f):
    return np.sort(np.rec.fromarrays([cell] + [a.view(np.int32) for a in f]), order=None)


def test_sort_orders_by_brick_then_cell_and_keeps_every_particle(gpu_available):
    n = 24
    cfg = cfg_sorted(n)
    g = RootGrid(cfg)
    for s in range(2):
        g.load_particles(s, with_blob(n, n ** 3 * 4, 12000, 70 + 10 * s, s))
    before = [g.getParticlesRaw(s) for s in range(2)]
    g.sort()
    for s in range(2):
        cell, f = g.getParticlesRaw(s)
        assert len(cell) == len(before[s][0])
        key = sort_keys(cell, n)
        assert np.all(np.diff(key) >= 0), "slots not in brick-then-cell order"
        blob_brick = np.bincount(key // (BX * BY * BZ)).max()
        assert blob_brick > 8192
        assert np.array_equal(records(cell, f), records(*before[s]))


def test_steps_with_a_sort_each_step_track_oracle(gpu_available):
    n = 16
    cfg = cfg_sorted(n, sort_interval=1)
    parts = [with_blob(n, n ** 3 * 4, 9000, 90 + 10 * s, s) for s in range(2)]
    g = RootGrid(cfg)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    for s, recs in enumerate(parts):
        g.load_particles(s, recs)
        o.load_particles(s, as_f32_state(recs))
    g.initialize()
    o.initialize()
    for _ in range(4):
        g.mainLoopES(1)
        o.main_loop(1)
    pe_g, fe_g = g.getEnergy()
    pe_o, fe_o = o.energy()
    assert abs(pe_g - pe_o) < 1e-5 * pe_o
    assert abs(fe_g - fe_o) < 2e-3 * fe_o
    for s in range(2):
        cell, _ = g.getParticlesRaw(s)
        assert np.all(np.diff(sort_keys(cell, n)) >= 0)
        a, b, d = match(g.getParticles(s), o.particles(s))
        assert np.max(np.abs(a["x"] - b["x"])) < 1e-4
