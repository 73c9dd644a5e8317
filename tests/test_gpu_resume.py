"""Resume data and the capacity-matrix cache on the GPU.

* A run saved after 3 steps (Environment::saveInfo + RootGrid::saveResumeData,
  src/main.cpp:62-63) and continued in a fresh context (loadInfo,
  loadResumeData, Grid::initializeForLoad: Initialize.cpp:81-95, Grid.cpp:38-50)
  tracks the uninterrupted run: spacecraft potential and energies within 1e-6,
  the same particle counts (the injection carry and the Philox keys continue).
* The capacity-matrix cache (IO::writeCmatrixData / loadCmatrixData,
  IO.cpp:28-120) gives back the built matrix; a cache with another grid
  spacing, or a damaged file, is not used.
* fopis_run writes the resume files at the end of a run and continues from them
  with job_type "load" and use_existing_capacity_matrix; a resume whose dx
  differs from input.json's is refused with the reference's message."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fopis_b200 import RootGrid, _abi
from fopis_b200 import resume as R

from host_input import write_input
from test_gpu_conductor import cube_cfg

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
RUN = ROOT / "fopis_b200" / "fopis_run"


def history(g, steps):
    h = []
    for _ in range(steps):
        g.mainLoopES(1)
        st = g.stats()
        h.append((g.getObject(0)[0],) + g.getEnergy() + tuple(int(st.valid_particles[s]) for s in range(3)))
    return np.array(h)


def test_resumed_run_tracks_uninterrupted_run(gpu_available, tmp_path):
    cfg = cube_cfg(n=25, half=2, ppc=8, photo=True, tol=1e-10)
    a = RootGrid(cfg)
    a.set_guess_mode(_abi.GUESS_WARM)
    a.initializeObjectsCmatrix(0)
    R.write_cmatrix(a, 0, tmp_path)
    a.generate_ambient()
    a.initialize()
    ha = history(a, 6)
    b = RootGrid(cfg)
    b.set_guess_mode(_abi.GUESS_WARM)
    b.set_cmatrix(0, a.get_cmatrix(0))
    b.generate_ambient()
    b.initialize()
    history(b, 3)
    R.save_resume(b, tmp_path)
    b.close()
    c = RootGrid(cfg)
    c.set_guess_mode(_abi.GUESS_WARM)
    assert R.load_cmatrix(c, 0, tmp_path)
    assert R.load_resume(c, tmp_path) == 4
    hc = history(c, 3)
    rel = np.abs(hc[:, :3] - ha[3:, :3]) / np.abs(ha[3:, :3])
    assert rel.max() < 1e-6, rel
    assert np.array_equal(hc[:, 3:], ha[3:, 3:])
    for g in (a, c):
        g.close()


def test_capacity_matrix_cache(gpu_available, tmp_path):
    cfg = cube_cfg(n=21, half=2, ppc=1, photo=False)
    g = RootGrid(cfg)
    g.initializeObjectsCmatrix(0)
    R.write_cmatrix(g, 0, tmp_path)
    h = RootGrid(cfg)
    assert R.load_cmatrix(h, 0, tmp_path)
    assert np.array_equal(h.get_cmatrix(0), g.get_cmatrix(0))
    other = cube_cfg(n=21, half=2, ppc=1, photo=False)
    other.dx = cfg.dx * 1.01
    k = RootGrid(other)
    assert not R.load_cmatrix(k, 0, tmp_path)                 # another grid spacing (IO.cpp:88-90)
    f = R.cmatrix_file(tmp_path, cfg.objects[0])
    raw = bytearray(f.read_bytes())
    raw[100] ^= 1
    f.write_bytes(bytes(raw))
    assert not R.load_cmatrix(h, 0, tmp_path)                 # damaged file
    for x in (g, h, k):
        x.close()


def run(args, timeout=600):
    return subprocess.run([str(RUN)] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)


def test_fopis_run_resume_and_cache(gpu_available, tmp_path):
    case = tmp_path / "case"
    path = write_input(case, n=21, ppc=4, photo=True, steps=7)
    js = json.loads(path.read_text())
    js["Options"]["use_existing_capacity_matrix"] = True
    path.write_text(json.dumps(js))
    # uninterrupted: 7 steps
    r = run([path, "--out", tmp_path / "full", "--resume", tmp_path / "res_full", "--guess", "warm"])
    assert r.returncode == 0, r.stderr
    full = np.loadtxt(tmp_path / "full" / "object_Spacecraft.txt", skiprows=1)
    assert (tmp_path / "res_full" / "objects" / "cube.obj.bin").exists()
    # 4 steps, then a load job for 3 more, with the capacity matrix from the cache
    r = run([path, "--steps", 4, "--out", tmp_path / "part", "--resume", tmp_path / "res", "--guess", "warm"])
    assert r.returncode == 0, r.stderr
    js["Environment"]["job_type"] = "load"
    path.write_text(json.dumps(js))
    r = run([path, "--steps", 3, "--out", tmp_path / "part", "--resume", tmp_path / "res", "--guess", "warm"])
    assert r.returncode == 0, r.stderr
    assert "Resume Data (t = 5)" in r.stdout
    part = np.loadtxt(tmp_path / "part" / "object_Spacecraft.txt", skiprows=1)
    assert part.shape[0] == 7 and list(part[:, 0]) == list(full[:, 0])
    np.testing.assert_allclose(part[4:, 2], full[4:, 2], rtol=1e-6, atol=1e-6 * np.abs(full[:, 2]).max())
    # a resume written with another dx is refused (Environment::loadInfo)
    js["Environment"]["dx"] = js["Environment"]["dx"] * 1.5
    path.write_text(json.dumps(js))
    r = run([path, "--steps", 1, "--out", tmp_path / "bad", "--resume", tmp_path / "res"])
    assert r.returncode == 1 and "does not match the dx" in r.stderr
