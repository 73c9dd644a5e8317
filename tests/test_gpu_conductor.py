"""GPU parity of the conductor path against the FP64 oracle: capacity matrix,
ambient loading, photoemission, boundary injection, absorption and the
equipotential redistribution (RootGrid::injectParticlesFromBoundary,
Spacecraft::emitParticles, distributeInnerParticleCharge, sumWholeCharge,
redistributeChargeForPerfectConductor, RootGrid::initializeObjectsCmatrix)."""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units, objects_from_boxes

from helpers import match, rel_err

pytestmark = pytest.mark.gpu


def cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-10, fixed=None, precision=_abi.MIXED):
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, ppc)]
    shine = (0.0, 0.0, 0.0)
    if photo:
        import math
        vbar = math.sqrt(8.0 * 1.0 * config.E / (math.pi * config.ME))
        sp.append(SpeciesInfo("Photo", "photoelectron", 1.0, -1.0, 1e7, 0.2, ppc,
                              current_density=10.0 * config.E * 1e7 * vbar / 4.0))
        shine = (-1.0, 0.0, 0.0)
    p, norm = make_params((n, n, n), "DDDDDD", dx, dt, sp, shine=shine, tol=tol, sort_interval=1000000, seed=4242,
                          precision=precision)
    emit = 2 if photo else -1
    obj = objects_from_boxes([((-half,) * 3, (half,) * 3)], (n, n, n), emit_species=emit, fixed=fixed)
    return config.SimConfig(params=p, norm=norm, species=sp, objects=[obj])


@pytest.fixture(scope="module")
def pair(gpu_available):
    cfg = cube_cfg()
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    o.build_cmatrix(0)
    return cfg, g, o


def test_capacity_matrix_matches_oracle(pair):
    cfg, g, o = pair
    Cg, Co = g.get_cmatrix(0), o.get_cmatrix(0)
    assert Cg.shape == (98, 98)
    assert rel_err(Cg, Co) < 1e-6
    # C is the inverse of B = phi at the surface nodes for unit charges
    assert abs(Cg.sum() - Co.sum()) < 1e-6 * abs(Co.sum())


def test_ambient_loading_matches_oracle(pair):
    cfg, g, o = pair
    g.generate_ambient()
    o.generate_ambient()
    for s in range(2):
        a, b = g.getParticles(s), o.particles(s)
        assert len(a) == len(b)              # same Philox draws, same body exclusion
        a, b, d = match(a, b)
        assert np.max(d) < 1e-5


def test_phased_step_with_conductor_matches_oracle(pair):
    cfg, g, o = pair
    g.initialize()
    o.initialize()
    V0g, Q0g, _ = g.getObject(0)
    V0o, Q0o, _ = o.get_object(0)
    assert abs(V0g - V0o) <= 1e-6 * max(abs(V0o), 1e-30) + 1e-12
    for step in range(3):
        g.updateParticleVelocity()
        o.reset_objects()
        o.update_velocity()
        g.emitParticlesFromObjects()
        o.emit()
        if step == 0:
            a, b, d = match(g.getParticles(2), o.particles(2))
            assert len(a) > 0 and np.max(d) < 1e-5
        g.updateParticlePosition()
        o.update_position()
        g.injectParticlesFromBoundary()
        o.inject()
        if step == 0:
            for s in range(2):
                a, b, d = match(g.getParticles(s), o.particles(s))
                assert np.max(d) < 1e-4
        g.updateRho()
        o.update_rho()
        g.solvePoisson()
        o.solve()
        g.updateEfield()
        o.update_efield()
        g.advance_timestep()
        o.timestep = o.timestep + 1
        Vg, Qg, Ig = g.getObject(0)
        Vo, Qo, Io = o.get_object(0)
        assert abs(Vg - Vo) <= 1e-3 * abs(Vo), (step, Vg, Vo)
        assert abs(Qg - Qo) <= 1e-3 * abs(Qo) + 1e-6 * abs(cfg.params.species[0].size), (step, Qg, Qo)
        assert np.allclose(Ig, Io, rtol=0.05, atol=abs(cfg.params.species[0].size) * 2.5)
    cm_g, cm_o = g.getChargeMap(0), o.charge_map(0)
    cm_err = rel_err(cm_g.sum(0), cm_o.sum(0))
    print(f"\nmixed precision, 3 phased steps: charge map {cm_err:.2e}")
    assert cm_err < 1e-5
    st = g.stats()
    assert st.device_status & ~_abi.DEV_SURFACE_NOT_FOUND == 0


def test_fused_steps_with_conductor_track_oracle(gpu_available):
    cfg = cube_cfg(n=25, half=2, ppc=8)
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
    for _ in range(8):
        g.mainLoopES(1)
        o.main_loop(1)
        Vg.append(g.getObject(0)[0])
        Vo.append(o.get_object(0)[0])
    Vg, Vo = np.array(Vg), np.array(Vo)
    assert np.max(np.abs(Vg - Vo)) <= 0.01 * np.max(np.abs(Vo))      # spacecraft potential within 1 %
    pg, fg = g.getEnergy()
    po, fo = o.energy()
    assert abs(pg - po) < 1e-3 * po and abs(fg - fo) < 1e-2 * fo
    for s in range(3):
        ng, no = len(g.getParticles(s)), len(o.particles(s))
        assert abs(ng - no) <= max(3, 1e-4 * no)


def test_fixed_potential_object(gpu_available):
    cfg = cube_cfg(n=21, half=2, ppc=4, photo=False, fixed=0.0)
    cfg.objects[0].fixed_potential = -0.02
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    g.generate_ambient()
    g.initialize()
    g.mainLoopES(2)
    V, Q, I = g.getObject(0)
    assert V == -0.02
    # the surface nodes sit at the fixed potential after the second solve
    phi = g.getPhi()
    nodes = cfg.objects[0].nodes
    ps = phi[nodes[:, 0], nodes[:, 1], nodes[:, 2]]
    assert np.max(np.abs(ps - V)) < 1e-6 * max(1.0, abs(V)) + 1e-9 * np.max(np.abs(phi))


def test_capacity_matrix_64_matches_exact(gpu_available):
    """At 64^3 (386 surface nodes) the capacity matrix built by multigrid solves
    on the GPU agrees with the exact sine-basis build."""
    cfg = config.workload("cube64", ppc=1)
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    Cg = g.get_cmatrix(0)
    g.close()
    Cx = orc.dirichlet_capacity_matrix(cfg.params, cfg.objects[0].nodes)
    assert Cg.shape == Cx.shape == (386, 386)
    assert np.abs(Cg - Cx).max() < 1e-8 * np.abs(Cx).max()
