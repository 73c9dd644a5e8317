"""fopis_run (the C++ host side over the C ABI) on a 25^3 box with a voxel
cube and photoemission: its data/energy.txt, data/object_Spacecraft.txt and
data/total_particle_number.txt match the Python driver stepping the same
input.json through the same library."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fopis_b200 import RootGrid, config

from host_input import write_input

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
RUN = ROOT / "fopis_b200" / "fopis_run"


def test_fopis_run_matches_python_driver(gpu_available, tmp_path):
    steps = 5
    path = write_input(tmp_path / "case", n=25, ppc=4, photo=True, steps=steps)
    out = tmp_path / "data"
    r = subprocess.run([str(RUN), str(path), "--out", str(out), "--resume", str(tmp_path / "resume")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    energy = np.loadtxt(out / "energy.txt", skiprows=1)
    obj = np.loadtxt(out / "object_Spacecraft.txt", skiprows=1)
    num = np.loadtxt(out / "total_particle_number.txt", skiprows=1)
    assert energy.shape == (steps, 6) and obj.shape[0] == steps and num.shape[0] == steps

    cfg = config.load_input(str(path))
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    g.generate_ambient()
    g.initialize()
    n = cfg.norm
    for t in range(steps):
        g.mainLoopES(1)
        pe, fe = g.getEnergy()
        V, Q, I = g.getObject(0)
        st = g.stats()
        assert energy[t, 0] == t + 1
        np.testing.assert_allclose(energy[t, 1], (t + 1) * cfg.dt, rtol=1e-6)
        np.testing.assert_allclose(energy[t, 3], n.unenergy(pe), rtol=1e-6)
        np.testing.assert_allclose(energy[t, 4], n.unenergy(fe), rtol=1e-6)
        np.testing.assert_allclose(obj[t, 2], n.unpotential(V), rtol=1e-6)
        np.testing.assert_allclose(obj[t, 3], n.uncharge(Q), rtol=1e-6, atol=1e-30)
        counts = [int(st.num_particles[s]) for s in range(cfg.params.nspecies)]
        assert list(num[t, 3:].astype(np.int64)) == counts and num[t, 2] == sum(counts)
    g.close()
