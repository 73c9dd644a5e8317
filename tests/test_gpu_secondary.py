"""GPU parity of the secondary-emission and dielectric-surface path against the
FP64 oracle:

* one incident list (hits of 1-90 eV electrons and ions on the six faces of a
  cube) given to both sides: the same secondaries (elastic, inelastic and true)
  leave from the same points with the same velocities (positions to 2e-6 cells,
  the split-precision offsets; velocities to 1e-6 relative), the same charge
  comes off the same surface nodes (2e-6 of the largest node charge: the GPU
  rounds the in-face coordinates of the bilinear split to 2^-20) and the
  object's current matches;
* fused steps on a cube that emits secondaries, hit by 4 eV electrons (true
  secondaries and elastic backscatter; speeds stay below a cell per step, the
  reference's regime), in the FP64 mode: absorption records the same incidents
  (same count per step, crossing points to 1e-9), the same secondaries live on,
  and the spacecraft potential tracks the oracle (1e-6 relative) over 12 steps;
* a dielectric cube of two materials (Spacecraft::redistributeChargeForDielectric,
  src/Spacecraft/Spacecraft.cpp:641-706), FP64 mode: the spacecraft potential
  within 1e-6 relative of the oracle's over 20 steps and visibly different from
  the same body as a perfect conductor.

Reference path: Spacecraft::emitParticles (Spacecraft.cpp:901-937),
SecondaryParticleType::generateNewParticles (src/Particle/SecondaryParticleType.cpp:16-194),
Spacecraft::distributeInnerParticleCharge with incident events (Spacecraft.cpp:512-592,
src/Spacecraft/SecondaryEmission.cpp:14-33)."""
import math

import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, _abi, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units

from helpers import as_f32_state, match, random_particles
from test_secondary_cpu import incident_records, secondary_cfg

pytestmark = pytest.mark.gpu


def vec(r):
    return np.stack([r[k] for k in ("x", "y", "z", "vx", "vy", "vz")], 1)


def test_secondaries_from_one_incident_list_match_oracle(gpu_available):
    cfg = secondary_cfg()
    p = cfg.params
    n = len(cfg.objects[0].nodes)
    g = RootGrid(cfg)
    g.set_cmatrix(0, np.eye(n))
    o = orc.Oracle(p, cfg.objects)
    o.set_cmatrix(0, np.eye(n))
    recs = incident_records(p.energy_ev)
    g.set_incidents(recs)
    assert np.array_equal(g.get_incidents(), recs)
    o.set_incidents(recs)
    assert g.lib.fopis_set_timestep(g.h, 7) == 0
    o.timestep = 7
    g.emitParticlesFromObjects()
    assert o.emit() == 0
    assert len(g.get_incidents()) == 0
    a, b = g.getParticles(2), o.particles(2)
    assert len(a) == len(b) > 100
    a, b, _ = match(a, b)
    va, vb = vec(a), vec(b)
    assert np.max(np.abs(va[:, :3] - vb[:, :3])) < 2e-6
    assert np.max(np.linalg.norm(va[:, 3:] - vb[:, 3:], axis=1) / np.linalg.norm(vb[:, 3:], axis=1)) < 1e-6
    # the emitted charge, on the surface nodes (moved to the charge map by updateRho)
    g.updateRho()
    o.update_rho()
    cg, co = g.getChargeMap(0), o.charge_map(0)
    assert np.max(np.abs(cg - co)) <= 2e-6 * np.max(np.abs(co))
    assert np.max(np.abs(co[2])) > 0
    _, _, cur_g = g.getObject(0)
    _, _, cur_o = o.get_object(0)
    assert cur_g[2] == pytest.approx(cur_o[2], rel=1e-12)
    g.close()
    o.close()


def fast_electron_cfg(precision=_abi.FP64, dielectric=None, secondary=True, n=25, te=4.0):
    """A 25^3 Dirichlet box with a 4^3 cube; electrons at `te` eV (ions 1 eV); with
    secondary, the cube emits secondaries of 2 eV."""
    dx, dt = plasma_units()
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, te, 4),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, 4)]
    if secondary:
        sp.append(SpeciesInfo("Secondary", "secondary", 1.0, -1.0, 1e7, 2.0, 4))
    p, norm = make_params((n, n, n), "DDDDDD", dx, dt, sp, tol=1e-10, sort_interval=1000000, precision=precision)
    if dielectric:
        import tempfile, os
        text = config.box_obj_text([((-2, -2, -2), (2, 2, 2))])
        text = "\n".join(l.replace("/1/2", "/2/2") if l.startswith("f ") else l for l in text.splitlines()) + "\n"
        fd, path = tempfile.mkstemp(suffix=".obj")
        with os.fdopen(fd, "w") as f:
            f.write(text)
        try:
            nodes, cells = orc.parse_obj(path, n, n, n)
            tex = config.parse_obj_textures(path, n, n, n)
        finally:
            os.unlink(path)
        obj = config.ObjectInfo("Spacecraft", nodes, cells, dielectric=1,
                                capacitance=config.node_capacitance(tex, dielectric, norm))
    else:
        obj = config.objects_from_boxes([((-2, -2, -2), (2, 2, 2))], (n, n, n), obj_parser=orc.parse_obj)
    if secondary:
        obj.secondary_species = 2
    return config.SimConfig(params=p, norm=norm, species=sp, objects=[obj])


def start_pair(cfg, seed=40):
    p = cfg.params
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    o = orc.Oracle(p, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    o.set_cmatrix(0, g.get_cmatrix(0))
    npart = (p.nx - 1) ** 3 * 4
    for s in range(2):
        sig = p.species[s].deviation
        recs = random_particles(npart, (0, 0, 0), (p.nx - 1,) * 3, sig, seed + s, s)
        cells = {tuple(c) for c in cfg.objects[0].cells}
        keep = np.array([tuple(int(math.floor(c)) + 1 for c in (r["x"], r["y"], r["z"])) not in cells for r in recs])
        recs = recs[keep]
        g.load_particles(s, recs)
        o.load_particles(s, recs if p.precision == _abi.FP64 else as_f32_state(recs))
    g.initialize()
    o.initialize()
    return g, o


def test_fused_steps_with_secondaries_track_oracle(gpu_available):
    cfg = fast_electron_cfg()
    g, o = start_pair(cfg)
    Vg, Vo, ng, no, inc = [], [], [], [], []
    for step in range(12):
        g.mainLoopES(1)
        o.main_loop(1)
        ig, io = g.get_incidents(), o.get_incidents()
        assert len(ig) == len(io), (step, len(ig), len(io))
        if len(ig):
            key = lambda r: np.lexsort((r[:, 6], r[:, 5], r[:, 4], r[:, 1]))
            a, b = ig[key(ig)], io[key(io)]
            assert np.array_equal(a[:, :3], b[:, :3])
            assert np.max(np.abs(a[:, 3:] - b[:, 3:])) < 1e-9
        inc.append(len(ig))
        Vg.append(g.getObject(0)[0])
        Vo.append(o.get_object(0)[0])
        ng.append(len(g.getParticles(2)))
        no.append(len(o.particles(2)))
    Vg, Vo = np.array(Vg), np.array(Vo)
    assert sum(inc) > 50 and ng[-1] > 0, (inc, ng)
    assert ng == no, (ng, no)
    assert np.max(np.abs(Vg - Vo) / np.abs(Vo)) <= 1e-6
    print(f"\nsecondaries: incidents per step {inc}, secondaries alive {ng[-1]}, "
          f"potential max rel. error {np.max(np.abs(Vg - Vo) / np.abs(Vo)):.2e}")
    g.close()
    o.close()


def test_dielectric_surface_tracks_oracle(gpu_available):
    mats = {1: "Teflon", 2: "Aluminum"}
    hist = {}
    for name, diel in (("dielectric", mats), ("conductor", None)):
        cfg = fast_electron_cfg(dielectric=diel, secondary=False, te=1.0)
        g, o = start_pair(cfg)
        Vg, Vo = [], []
        for _ in range(20):
            g.mainLoopES(1)
            o.main_loop(1)
            Vg.append(g.getObject(0)[0])
            Vo.append(o.get_object(0)[0])
        Vg, Vo = np.array(Vg), np.array(Vo)
        err = np.max(np.abs(Vg - Vo) / np.abs(Vo))
        assert err <= 1e-6, (name, err)
        hist[name] = Vg
        g.close()
        o.close()
    diff = np.max(np.abs(hist["dielectric"] - hist["conductor"]) / np.abs(hist["conductor"]))
    assert diff > 1e-3, diff
    print(f"\ndielectric: potential tracks the oracle to 1e-6; differs from the conductor's by up to {diff:.2e}")
