"""Long-run parity: 100 fused steps of the mixed-precision GPU path against the
FP64 oracle on the same initial particles (25^3 box, voxel cube, photoemission,
injection on all faces): the spacecraft-potential history and the particle and
field energy histories agree within 1 %."""
import numpy as np
import pytest

import oracle as orc
from fopis_b200 import RootGrid

from test_gpu_conductor import cube_cfg

pytestmark = pytest.mark.gpu


def test_hundred_steps_track_fp64_oracle(gpu_available):
    steps = 100
    cfg = cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-8)
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    o = orc.Oracle(cfg.params, cfg.objects)
    o.set_solver(1, exact_tol=1e-10)
    o.set_cmatrix(0, g.get_cmatrix(0))
    g.generate_ambient()
    o.generate_ambient()
    g.initialize()
    o.initialize()
    hist = []
    for _ in range(steps):
        g.mainLoopES(1)
        o.main_loop(1)
        hist.append((g.getObject(0)[0], o.get_object(0)[0]) + g.getEnergy() + o.energy())
    g.close()
    o.close()
    h = np.array(hist)                  # Vg, Vo, pe_g, fe_g, pe_o, fe_o
    Vg, Vo = h[:, 0], h[:, 1]
    assert np.max(np.abs(Vg - Vo)) <= 0.01 * np.max(np.abs(Vo))
    pe_g, fe_g, pe_o, fe_o = h[:, 2], h[:, 3], h[:, 4], h[:, 5]
    assert np.max(np.abs(pe_g - pe_o) / pe_o) <= 0.01
    assert np.max(np.abs(fe_g - fe_o)) <= 0.01 * np.max(fe_o)
    print(f"\n100 steps: max |dV|/max|V| {np.max(np.abs(Vg - Vo)) / np.max(np.abs(Vo)):.2e}, "
          f"max particle-energy rel. error {np.max(np.abs(pe_g - pe_o) / pe_o):.2e}, "
          f"max field-energy error / max {np.max(np.abs(fe_g - fe_o)) / np.max(fe_o):.2e}")
