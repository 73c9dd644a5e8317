"""GPU parity of the EM mode (RootGrid::mainLoopEM, src/Grid/RootGrid/RootGrid.cpp:145-191)
against the FP64 oracle:

* the FDTD updates alone (RootGrid::updateEfieldFDTDDamping / updateBfieldDamping,
  src/Grid/RootGrid/RootGridField.cpp:594-820, with the periodic glue copies and the
  nodal references of :489-582 and :1102-1127) on random fields and currents, on
  D, mixed and periodic boxes: every Yee array and nodal field to 1e-12 of its
  largest value over three updates;
* the phases of one step on the FP64 GPU path: the E and B gather with Boris
  (GridParticleTreatmentEM.cpp:13-105) to 1e-12, the edge currents of
  updateParticlePositionEM (:107-201, particle.cpp:258-338) to 1e-12 of the largest;
* whole mainLoopEM runs, FP64: a D box with injection and a periodic box (20
  steps) and a floating conductor with photoemission (10 steps): particle sets to
  1e-9 cells, fields to 1e-8 of their largest, the three energies to 1e-9
  (the oracle solves Poisson exactly, the GPU to 1e-10, so the start-up E differs
  at that level and is carried along);
* the mixed mode (FP32 particles) against the same oracle: fields to 1e-4 of their
  largest after 10 steps.
"""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, _abi

from helpers import as_f32_state, em_config, match, random_particles, rel_err

pytestmark = pytest.mark.gpu

YEE = list(range(_abi.FIELD_EX, _abi.FIELD_BZ + 1))
NODAL = [_abi.FIELD_EXREF, _abi.FIELD_EYREF, _abi.FIELD_EZREF, _abi.FIELD_BXREF, _abi.FIELD_BYREF, _abi.FIELD_BZREF]
CURRENTS = [_abi.FIELD_JX, _abi.FIELD_JY, _abi.FIELD_JZ]


@pytest.mark.parametrize("boundary", ["DDDDDD", "PPDDPP", "PPPPPP", "NDPPDN"])
def test_fdtd_updates_match_oracle(gpu_available, boundary):
    cfg = em_config(n=10, boundary=boundary)
    g = RootGrid(cfg)
    o = orc.Oracle(cfg.params)
    rng = np.random.default_rng(7)
    for which in YEE + CURRENTS:
        assert g.field_shape(which) == o.field_shape(which)
        a = rng.standard_normal(o.field_shape(which)[1]) * (1e-3 if which in CURRENTS else 1.0)
        g.set_field(which, a)
        o.set_field(which, a)
    phi = rng.standard_normal((12, 12, 12))
    g.set_field(_abi.FIELD_PHI, phi)
    o.set_field(0, phi)
    for _ in range(3):
        g.updateEfield()
        o.update_efield()
        g.updateBfield()
        o.update_bfield()
    for which in YEE + NODAL:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-12, which
    assert g.getBfieldEnergy() == pytest.approx(o.bfield_energy(), rel=1e-12)
    assert g.getEnergy()[1] == pytest.approx(o.energy()[1], rel=1e-12)
    g.close()
    o.close()


def load_pair(cfg, seed=30, ppc_fill=4, f32=False):
    p = cfg.params
    g = RootGrid(cfg)
    if cfg.objects:
        g.initializeObjectsCmatrix(0)
    o = orc.Oracle(p, cfg.objects)
    o.set_solver(1, exact_tol=1e-13)
    if cfg.objects:
        o.set_cmatrix(0, g.get_cmatrix(0))
    hi = [p.nx - 1 if cfg.params.boundary[2 * a] != b"P"[0] else p.nx for a in range(3)]
    for s in range(2):
        recs = random_particles(int(np.prod(hi)) * ppc_fill, (0, 0, 0), hi, p.species[s].deviation, seed + s, s)
        if cfg.objects:
            cells = {tuple(c) for c in cfg.objects[0].cells}
            keep = np.array([tuple(int(np.floor(v)) + 1 for v in (r["x"], r["y"], r["z"])) not in cells for r in recs])
            recs = recs[keep]
        g.load_particles(s, recs)
        o.load_particles(s, as_f32_state(recs) if f32 else recs)
    g.initialize()
    o.initialize()
    return g, o


def compare_particles(g, o, tol_x, tol_v):
    for s in range(g.nspecies):
        a, b, _ = match(g.getParticles(s), o.particles(s))
        for key in ("x", "y", "z"):
            assert np.max(np.abs(a[key] - b[key]), initial=0.0) <= tol_x, (s, key)
        vmax = max(np.max(np.abs(b[k]), initial=0.0) for k in ("vx", "vy", "vz"))
        for key in ("vx", "vy", "vz"):
            assert np.max(np.abs(a[key] - b[key]), initial=0.0) <= tol_v * vmax, (s, key)


def test_em_phases_match_oracle(gpu_available):
    cfg = em_config(n=13)
    g, o = load_pair(cfg)
    for which in NODAL[:3]:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-8, which
    # B after Grid::initialize is the curl of a gradient: rounding on both sides
    emax = max(np.max(np.abs(o.field(w))) for w in NODAL[:3])
    for which in NODAL[3:]:
        assert np.max(np.abs(g.get_field(which))) <= 1e-12 * emax
        assert np.max(np.abs(o.field(which))) <= 1e-12 * emax
    g.updateParticleVelocity()
    o.update_velocity()
    compare_particles(g, o, 1e-12, 1e-9)
    g.updateParticlePosition()
    o.update_position()
    for which in CURRENTS:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-9, which
    compare_particles(g, o, 1e-12, 1e-9)
    g.injectParticlesFromBoundary()
    o.inject()
    g.updateRho()
    o.update_rho()
    assert rel_err(g.getRho(), o.field(1)) <= 1e-11
    g.updateEfield()
    o.update_efield()
    g.updateBfield()
    o.update_bfield()
    for which in YEE + NODAL:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-8, which
    g.close()
    o.close()


def test_em_mixed_phases_match_oracle(gpu_available):
    """The phase entry points in the mixed mode (FP32 particles): velocity, then the
    position update with the edge currents (FP64 atomics of the FP32 terms), against
    the FP64 oracle on the same FP32-rounded start."""
    cfg = em_config(n=13, precision=_abi.MIXED)
    g, o = load_pair(cfg, f32=True)
    g.updateParticleVelocity()
    o.update_velocity()
    compare_particles(g, o, 1e-6, 1e-5)
    g.updateParticlePosition()
    o.update_position()
    for which in CURRENTS:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-5, which
    compare_particles(g, o, 1e-5, 1e-5)
    g.close()
    o.close()


@pytest.mark.parametrize("boundary,steps", [("DDDDDD", 20), ("PPPPPP", 20)])
def test_em_main_loop_fp64_tracks_oracle(gpu_available, boundary, steps):
    cfg = em_config(n=13, boundary=boundary)
    g, o = load_pair(cfg)
    hist = []
    for _ in range(steps):
        g.mainLoopEM(1)
        o.main_loop(1)
        pe_g, fe_g = g.getEnergy()
        pe_o, fe_o = o.energy()
        hist.append((pe_g / pe_o - 1, fe_g / fe_o - 1, g.getBfieldEnergy() / o.bfield_energy() - 1))
    hist = np.abs(np.array(hist))
    assert np.max(hist) <= 1e-8, hist.max(0)
    compare_particles(g, o, 1e-9, 1e-8)
    for which in YEE + NODAL + CURRENTS:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-8, which
    print(f"\nEM {boundary}: {steps} steps, worst relative energy differences (particles, E, B) "
          f"{hist.max(0)}, B energy {o.bfield_energy():.3e}")
    g.close()
    o.close()


def test_em_conductor_run_tracks_oracle(gpu_available):
    cfg = em_config(n=17, boxes=[((-2, -2, -2), (2, 2, 2))], photo=True, obj_parser=orc.parse_obj)
    g, o = load_pair(cfg)
    V = []
    for _ in range(10):
        g.mainLoopEM(1)
        o.main_loop(1)
        V.append((g.getObject(0)[0], o.get_object(0)[0]))
    V = np.array(V)
    assert np.max(np.abs(V[:, 0] - V[:, 1]) / np.abs(V[:, 1])) <= 1e-8
    compare_particles(g, o, 1e-9, 1e-8)
    for which in YEE + NODAL:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-8, which
    g.close()
    o.close()


@pytest.mark.parametrize("boundary", ["DDDDDD", "PPPPPP"])
def test_em_mixed_precision_tracks_oracle(gpu_available, boundary):
    """The mixed mode's one-pass move with the fixed-point current (the periodic
    folds included on the P box) against the FP64 oracle."""
    cfg = em_config(n=13, boundary=boundary, precision=_abi.MIXED)
    g, o = load_pair(cfg, f32=True)
    for _ in range(10):
        g.mainLoopEM(1)
        o.main_loop(1)
    for which in YEE + NODAL + CURRENTS:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-4, which
    pe_g, fe_g = g.getEnergy()
    pe_o, fe_o = o.energy()
    assert pe_g == pytest.approx(pe_o, rel=1e-5)
    g.close()
    o.close()


def test_em_mixed_conductor_run_tracks_oracle(gpu_available):
    """The mixed mode with a floating conductor and photoemission: emitted particles
    move with their current in the tail pass, injected ones deposit as they are
    created, absorption and the redistribution as in the ES step."""
    cfg = em_config(n=17, boxes=[((-2, -2, -2), (2, 2, 2))], photo=True, obj_parser=orc.parse_obj,
                    precision=_abi.MIXED)
    g, o = load_pair(cfg, f32=True)
    V = []
    for _ in range(10):
        g.mainLoopEM(1)
        o.main_loop(1)
        V.append((g.getObject(0)[0], o.get_object(0)[0]))
    V = np.array(V)
    assert np.max(np.abs(V[:, 0] - V[:, 1]) / np.abs(V[:, 1])) <= 1e-4
    for s in range(3):       # FP32 trajectories may cross a face where the FP64 ones do not
        ng, no = len(g.getParticles(s)), len(o.particles(s))
        assert abs(ng - no) <= max(5, 2e-3 * no), (s, ng, no)
    for which in YEE + NODAL:
        assert rel_err(g.get_field(which), o.field(which)) <= 1e-4, which
    g.close()
    o.close()


def test_em_resume_tracks_uninterrupted_run(gpu_available, tmp_path):
    """Resume data of the EM mode (RootGrid::saveResumeFieldData / loadResumeFieldData,
    RootGridIO.cpp:181-271: the Yee E and B under Efield/ex.. and Bfield/bx..) and
    Grid::initializeForLoad: 3 steps, save, continue 3 steps in a fresh context,
    against 6 uninterrupted steps."""
    from fopis_b200 import resume as R
    cfg = em_config(n=13)

    def fresh():
        g, o = load_pair(cfg)
        o.close()
        return g

    def hist(g, steps):
        out = []
        for _ in range(steps):
            g.mainLoopEM(1)
            out.append(g.getEnergy() + (g.getBfieldEnergy(),))
        return np.array(out)

    a = fresh()
    ha = hist(a, 6)
    b = fresh()
    hist(b, 3)
    R.save_resume(b, tmp_path)
    c = RootGrid(cfg)
    assert R.load_resume(c, tmp_path) == int(b.stats().timestep)
    hc = hist(c, 3)
    assert np.max(np.abs(hc / ha[3:] - 1)) <= 1e-9, hc / ha[3:] - 1
    for which in YEE:
        assert rel_err(c.get_field(which), a.get_field(which)) <= 1e-9, which
    for g in (a, b, c):
        g.close()


def test_fopis_run_em_matches_python_driver(gpu_available, tmp_path):
    """fopis_run on an "EM" input.json: data/energy.txt carries the B-field column
    of IO::plotEnergy (src/Misc/IO.cpp:170-194) and matches the Python driver."""
    import subprocess
    from pathlib import Path
    from fopis_b200 import config
    from host_input import write_input
    run = Path(__file__).resolve().parent.parent / "fopis_b200" / "fopis_run"
    steps = 4
    path = write_input(tmp_path / "case", n=17, ppc=4, photo=True, steps=steps, em=True)
    out = tmp_path / "data"
    r = subprocess.run([str(run), str(path), "--out", str(out), "--resume", str(tmp_path / "resume")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    energy = np.loadtxt(out / "energy.txt", skiprows=1)
    cfg = config.load_input(str(path))
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    g.generate_ambient()
    g.initialize()
    n = cfg.norm
    for t in range(steps):
        g.mainLoopEM(1)
        pe, fe = g.getEnergy()
        be = g.getBfieldEnergy()
        np.testing.assert_allclose(energy[t, 3:6], [n.unenergy(pe), n.unenergy(fe), n.unenergy(be)], rtol=1e-6)
        np.testing.assert_allclose(energy[t, 2], n.unenergy(pe + fe + be), rtol=1e-6)
    assert energy[-1, 5] > 0.0
    g.close()
