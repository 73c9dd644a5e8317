"""Parity on the named workloads at their stated sizes, against the FP64
oracle, at these tolerances:

* the periodic box (32^3 cells fully periodic, electrons + ions, 16 particles per
  cell per species, 100 steps): after the first step every particle's
  position and velocity within 1e-5 relative of the oracle's; over 100 steps
  the kinetic- and field-energy histories within 1 % (mixed precision), and
  much tighter in the FP64 mode;
* the 64^3 spacecraft box (64^3 cells, Dirichlet faces with injection, 8^3-cell cube
  conductor, 32 particles per cell per species, FP64 on the GPU): the
  spacecraft potential within 1e-6 relative of the oracle's for 50 steps;
* a grid with Dirichlet, Neumann and periodic faces: phi (held Neumann faces
  during the solve, then Field::setNeumannPhi, src/Grid/Field.cpp:34-65) and
  nodal E against the oracle's exact solve, from a zero start and from a
  start whose Neumann faces hold the previous solve's values.

Reference path: RootGrid::mainLoopES (src/Grid/RootGrid/RootGrid.cpp:82-143)."""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, _abi, config

from helpers import match, random_particles, rel_err

pytestmark = pytest.mark.gpu


def vec(r, keys):
    return np.stack([r[k] for k in keys], 1)


def particle_errors(g, o, nsp):
    """Largest per-particle |dx|/max(|x|, 1 cell) and |dv|/|v| over the species."""
    ex = ev = 0.0
    for s in range(nsp):
        a, b, _ = match(g.getParticles(s), o.particles(s))
        xa, xb = vec(a, "xyz"), vec(b, "xyz")
        va, vb = vec(a, ("vx", "vy", "vz")), vec(b, ("vx", "vy", "vz"))
        ex = max(ex, float(np.max(np.linalg.norm(xa - xb, axis=1) / np.maximum(np.linalg.norm(xb, axis=1), 1.0))))
        ev = max(ev, float(np.max(np.linalg.norm(va - vb, axis=1) / np.linalg.norm(vb, axis=1))))
    return ex, ev


def energy_histories(g, o, steps):
    h = []
    for _ in range(steps):
        g.mainLoopES(1)
        o.main_loop(1)
        h.append(g.getEnergy() + o.energy())
    return np.array(h)               # pe_g, fe_g, pe_o, fe_o


@pytest.mark.parametrize("precision", [_abi.MIXED, _abi.FP64])
def test_config1_periodic32(gpu_available, precision):
    cfg = config.workload("periodic32", tol=1e-10, precision=precision)
    assert (cfg.params.nx, cfg.params.ny, cfg.params.nz) == (32, 32, 32) and cfg.params.species[0].particle_per_cell == 16
    g = RootGrid(cfg)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    g.generate_ambient()
    o.generate_ambient()
    n = sum(len(g.getParticles(s)) for s in range(2))
    assert n == 2 * 32 ** 3 * 16
    g.initialize()
    o.initialize()
    g.mainLoopES(1)
    o.main_loop(1)
    ex, ev = particle_errors(g, o, 2)
    bound = 1e-5 if precision == _abi.MIXED else 1e-10
    assert ex <= bound and ev <= bound, (ex, ev)
    h = energy_histories(g, o, 99)
    pe = np.abs(h[:, 0] - h[:, 2]) / h[:, 2]
    fe = np.abs(h[:, 1] - h[:, 3]) / np.max(h[:, 3])
    tol = 0.01 if precision == _abi.MIXED else 1e-4
    assert pe.max() <= tol and fe.max() <= tol, (pe.max(), fe.max())
    print(f"\nperiodic 32^3 box ({'mixed' if precision == _abi.MIXED else 'fp64'}): step-1 max |dx|/|x| {ex:.2e}, |dv|/|v| {ev:.2e};"
          f" 100 steps: kinetic energy {pe.max():.2e}, field energy {fe.max():.2e} of its max")
    g.close()
    o.close()


def test_config2_cube64_fp64_potential(gpu_available):
    cfg = config.workload("cube64", tol=1e-10, precision=_abi.FP64)
    assert (cfg.params.nx, cfg.params.ny, cfg.params.nz) == (65, 65, 65)
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    o.set_cmatrix(0, g.get_cmatrix(0))
    g.generate_ambient()
    o.generate_ambient()
    g.initialize()
    o.initialize()
    Vg, Vo = [], []
    for _ in range(50):
        g.mainLoopES(1)
        o.main_loop(1)
        Vg.append(g.getObject(0)[0])
        Vo.append(o.get_object(0)[0])
    Vg, Vo = np.array(Vg), np.array(Vo)
    err = np.abs(Vg - Vo) / np.abs(Vo)
    assert err.max() <= 1e-6, err.max()
    print(f"\n64^3 spacecraft box (fp64, 50 steps): spacecraft potential max rel. error {err.max():.2e}")
    pg, _ = g.getEnergy()
    po, _ = o.energy()
    assert abs(pg - po) <= 1e-6 * po
    g.close()
    o.close()


def mixed_face_cfg():
    from fopis_b200.config import SpeciesInfo, make_params, plasma_units
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, 8),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, 8)]
    # x: Neumann below, Dirichlet above; y periodic; z: Dirichlet below, Neumann above
    p, norm = make_params((25, 24, 27), "NDPPDN", dx, dt, sp, tol=1e-11, sort_interval=1000000)
    return config.SimConfig(params=p, norm=norm, species=sp)


def test_neumann_dirichlet_periodic_faces(gpu_available):
    cfg = mixed_face_cfg()
    p = cfg.params
    g = RootGrid(cfg)
    n = 24 * 24 * 26 * 8
    for s in range(2):
        g.load_particles(s, random_particles(n, (0, 0, 0), (p.nx - 1, p.ny, p.nz - 1), 0.1, 900 + s, s))
    assert g.initialize() == 0
    o = orc.Oracle(p)
    o.set_solver(1, exact_tol=1e-13)
    # zero start: the Neumann faces are held at 0 during the solve, then copied
    o.set_field(1, g.getRho())
    o.solve()
    pg, po = g.getPhi(), o.field(0)
    assert rel_err(pg, po) < 1e-8
    # Neumann copies over the face's own nodes (glue rows keep their earlier values, as in the reference)
    assert np.array_equal(pg[1, 1:-1, 1:-1], pg[2, 1:-1, 1:-1])
    assert np.array_equal(pg[1:-1, 1:-1, -2], pg[1:-1, 1:-1, -3])
    assert np.all(pg[-2, 1:-1, 1:-1] == 0.0) and np.all(pg[1:-1, 1:-1, 1] == 0.0)       # Dirichlet faces
    o.update_efield()
    g.updateEfield()
    for a, e in enumerate(g.getEref()):
        assert rel_err(e, o.field(2 + a)) < 1e-7
    # a second solve holds the Neumann faces at the values the first one copied
    rng = np.random.default_rng(3)
    rho2 = g.getRho() * (1.0 + 0.1 * rng.standard_normal(g.shape))
    g.set_field(_abi.FIELD_RHO0, rho2)
    assert g.solvePoisson() == 0
    o.set_field(0, pg)
    o.set_field(1, rho2)
    o.solve()
    assert rel_err(g.getPhi(), o.field(0)) < 1e-8
    # and the fused steps track the oracle on the same particles
    o3 = orc.Oracle(p)
    o3.set_solver(1, exact_tol=1e-13)
    g3 = RootGrid(cfg)
    for s in range(2):
        recs = random_particles(n, (0, 0, 0), (p.nx - 1, p.ny, p.nz - 1), 0.1, 950 + s, s)
        g3.load_particles(s, recs)
        o3.load_particles(s, recs)
    g3.initialize()
    o3.initialize()
    h = energy_histories(g3, o3, 10)
    assert np.max(np.abs(h[:, 0] - h[:, 2]) / h[:, 2]) < 1e-4
    assert np.max(np.abs(h[:, 1] - h[:, 3])) < 1e-3 * np.max(h[:, 3])
    for gg in (g, g3):
        gg.close()
