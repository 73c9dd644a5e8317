"""FP64 mode (FOPIS_FP64): FP64 particle offsets and velocities, FP64 gather,
push and deposit on the GPU.

* Against the FP64 oracle it agrees to rounding: one step on a periodic box,
  and 30 steps of the conductor path with photoemission and injection.
* It is the reference run for the mixed-precision mode: on the same seed the
  mixed mode's rho, phi and E after one step, and its spacecraft-potential
  history over 100 steps, are compared with the FP64 GPU run (the potential
  within 1 %).
"""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units

from helpers import match, random_particles, rel_err
from test_gpu_conductor import cube_cfg

pytestmark = pytest.mark.gpu


def periodic_fp64(n=16, ppc=4):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, ppc)]
    p, norm = make_params((n, n, n), "PPPPPP", dx, dt, sp, tol=1e-10, sort_interval=1000000,
                          precision=_abi.FP64)
    return config.SimConfig(params=p, norm=norm, species=sp)


def test_fp64_step_matches_oracle_to_rounding(gpu_available):
    cfg = periodic_fp64()
    n = 16 ** 3 * 4
    parts = [random_particles(n, (0, 0, 0), (16, 16, 16), 0.1, 500 + s, s) for s in range(2)]
    g = RootGrid(cfg)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    for s, recs in enumerate(parts):
        g.load_particles(s, recs)
        o.load_particles(s, recs)          # the FP64 records themselves, no FP32 rounding
    g.initialize()
    o.initialize()
    for s in range(2):
        assert rel_err(g.getRho(s), o.field(16 + s)) < 1e-12
    g.mainLoopES(1)
    o.main_loop(1)
    for s in range(2):
        a, b, d = match(g.getParticles(s), o.particles(s))
        for key in ("x", "y", "z"):
            assert np.max(np.abs(a[key] - b[key])) < 1e-11
        for key in ("vx", "vy", "vz"):
            assert np.max(np.abs(a[key] - b[key])) < 1e-11 * np.max(np.abs(b[key]))
        assert rel_err(g.getRho(s), o.field(16 + s)) < 1e-11
    assert rel_err(g.getPhi(), o.field(0)) < 1e-8
    pe_g, fe_g = g.getEnergy()
    pe_o, fe_o = o.energy()
    assert abs(pe_g - pe_o) < 1e-11 * pe_o
    assert abs(fe_g - fe_o) < 1e-7 * fe_o
    g.close()
    o.close()


def test_fp64_conductor_run_tracks_oracle(gpu_available):
    cfg = cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-10, precision=_abi.FP64)
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-12)
    o.set_cmatrix(0, g.get_cmatrix(0))
    g.generate_ambient()
    o.generate_ambient()
    g.initialize()
    o.initialize()
    hist = []
    for _ in range(30):
        g.mainLoopES(1)
        o.main_loop(1)
        hist.append((g.getObject(0)[0], o.get_object(0)[0]) + g.getEnergy() + o.energy())
    h = np.array(hist)
    Vg, Vo = h[:, 0], h[:, 1]
    assert np.max(np.abs(Vg - Vo)) <= 1e-6 * np.max(np.abs(Vo))
    assert np.max(np.abs(h[:, 2] - h[:, 4]) / h[:, 4]) <= 1e-8
    assert np.max(np.abs(h[:, 3] - h[:, 5])) <= 1e-6 * np.max(h[:, 5])
    for s in range(3):
        a, b, d = match(g.getParticles(s), o.particles(s))
        assert np.max(d) < 1e-8
    # surface charge per node and species (Spacecraft charge_map): the same absorptions and
    # emissions, the GPU's bilinear weights in 20-bit fixed point
    cm_g, cm_o = g.getChargeMap(0), o.charge_map(0)
    cm_err = rel_err(cm_g, cm_o)
    assert cm_err < 1e-5, cm_err
    print(f"\nFP64 GPU vs oracle, 30 steps: max |dV|/max|V| {np.max(np.abs(Vg - Vo)) / np.max(np.abs(Vo)):.2e}, "
          f"charge map {cm_err:.2e}")
    g.close()
    o.close()


def test_mixed_mode_error_against_fp64_run(gpu_available):
    mixed = cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-8)
    fp64 = cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-8, precision=_abi.FP64)
    gm, gd = RootGrid(mixed), RootGrid(fp64)
    gm.initializeObjectsCmatrix(0)
    gd.set_cmatrix(0, gm.get_cmatrix(0))
    for g in (gm, gd):
        g.generate_ambient()
        g.initialize()
        g.mainLoopES(1)
    # one step from the same loading: the mixed mode's field errors
    err = {"rho": rel_err(gm.getRho(), gd.getRho()), "phi": rel_err(gm.getPhi(), gd.getPhi())}
    em, ed = gm.getEref(), gd.getEref()
    err["E"] = max(rel_err(a, b) for a, b in zip(em, ed))
    assert err["rho"] < 1e-4 and err["phi"] < 1e-4 and err["E"] < 1e-3
    V = [(gm.getObject(0)[0], gd.getObject(0)[0])]
    for _ in range(99):
        gm.mainLoopES(1)
        gd.mainLoopES(1)
        V.append((gm.getObject(0)[0], gd.getObject(0)[0]))
    V = np.array(V)
    dv = np.max(np.abs(V[:, 0] - V[:, 1])) / np.max(np.abs(V[:, 1]))
    assert dv <= 0.01
    print(f"\nmixed vs FP64 GPU: step-1 rho {err['rho']:.2e}, phi {err['phi']:.2e}, E {err['E']:.2e}; "
          f"100-step potential {dv:.2e}")
    gm.close()
    gd.close()
