"""Two conductors in one box against the FP64 oracle: a floating cube with
photoemission and a second body held at a fixed potential (Spacecraft's
is_potential_fixed), each with its own capacity matrix, absorbing and
redistributing charge through 20 fused steps with boundary injection."""
import math

import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid, config
from fopis_b200.config import SpeciesInfo, make_params, plasma_units, objects_from_boxes

from helpers import rel_err

pytestmark = pytest.mark.gpu


def two_body_cfg(n=29, ppc=8, tol=1e-10):
    dx, dt = plasma_units()
    vbar = math.sqrt(8.0 * 1.0 * config.E / (math.pi * config.ME))
    sp = [SpeciesInfo("Electron", "ambient", 1.0, -1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Ion", "ambient", 100.0, 1.0, 1e7, 1.0, ppc),
          SpeciesInfo("Photo", "photoelectron", 1.0, -1.0, 1e7, 0.2, ppc,
                      current_density=10.0 * config.E * 1e7 * vbar / 4.0)]
    p, norm = make_params((n, n, n), "DDDDDD", dx, dt, sp, shine=(-1.0, 0.0, 0.0), tol=tol,
                          sort_interval=4, seed=777)
    floating = objects_from_boxes([((-8, -2, -2), (-4, 2, 2))], (n, n, n), name="Floating", emit_species=2)
    fixed = objects_from_boxes([((4, -3, -2), (7, 3, 2))], (n, n, n), name="Fixed", fixed=-0.5)
    return config.SimConfig(params=p, norm=norm, species=sp, objects=[floating, fixed])


def test_two_conductors_track_oracle(gpu_available):
    cfg = two_body_cfg()
    g = RootGrid(cfg)
    for o in range(2):
        g.initializeObjectsCmatrix(o)
    o_ = orc.Oracle(cfg.params, cfg.objects)
    o_.set_solver(1, exact_tol=1e-12)
    for o in range(2):
        o_.set_cmatrix(o, g.get_cmatrix(o))
    g.generate_ambient()
    o_.generate_ambient()
    g.initialize()
    o_.initialize()
    hist = []
    for _ in range(20):
        g.mainLoopES(1)
        o_.main_loop(1)
        hist.append([g.getObject(0)[0], o_.get_object(0)[0], g.getObject(1)[0], o_.get_object(1)[0]])
    h = np.array(hist)
    # the fixed body stays at its potential; the floating one tracks the oracle
    assert np.max(np.abs(h[:, 2] - (-0.5))) < 1e-9 and np.max(np.abs(h[:, 3] - (-0.5))) < 1e-9
    assert np.max(np.abs(h[:, 0] - h[:, 1])) <= 1e-3 * np.max(np.abs(h[:, 1]))
    pe_g, fe_g = g.getEnergy()
    pe_o, fe_o = o_.energy()
    assert abs(pe_g - pe_o) < 1e-3 * pe_o
    assert abs(fe_g - fe_o) < 1e-2 * fe_o
    # mixed precision against FP64: a particle at a body face may be absorbed on
    # one side only, so the populations are compared by count
    for s in range(3):
        ng, no = len(g.getParticles(s)), len(o_.particles(s))
        assert abs(ng - no) <= max(2, 1e-3 * no)
    assert rel_err(g.getPhi(), o_.field(0)) < 1e-2
    print(f"\ntwo bodies, 20 steps: floating |dV|/max|V| "
          f"{np.max(np.abs(h[:, 0] - h[:, 1])) / np.max(np.abs(h[:, 1])):.2e}")
    g.close()
    o_.close()
