"""CPU: the named-dataset files of the resume data and the capacity-matrix
cache (the reference keeps them as HDF5: RootGridIO.cpp:25-290, IO.cpp:28-120,
Environment.cpp:379-438). The Python reader and writer and the C++ host's
(fopis_run --datafile-echo) agree byte for byte; a corrupted or truncated file
is rejected by both; environment data with another dx or dt is rejected."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fopis_b200 import config
from fopis_b200 import resume as R

ROOT = Path(__file__).resolve().parent.parent
RUN = ROOT / "fopis_b200" / "fopis_run"


@pytest.fixture(scope="module")
def built():
    if not RUN.exists():
        subprocess.run(["make", "-C", str(ROOT / "fopis_b200")], check=True, capture_output=True)
    return RUN


def sample():
    rng = np.random.default_rng(3)
    return {"capacity_matrix": rng.standard_normal((7, 7)), "grid_spacing": np.float64(2.35),
            "time_spacing": np.float64(1.8e-6), "Electron/x": rng.uniform(0, 30, 1001),
            "Electron/generated_counts": np.array([12345, 9], np.int64), "Potential/phi": rng.standard_normal((5, 4, 6)),
            "Spacecraft/charge_map": rng.standard_normal((3, 11))}


def test_round_trip_and_cpp_agree(built, tmp_path):
    sets = sample()
    a = tmp_path / "a.bin"
    R.write(a, sets)
    got = R.read(a)
    assert set(got) == set(sets)
    for k, v in sets.items():
        assert got[k].dtype.kind == np.asarray(v).dtype.kind
        assert np.array_equal(got[k], np.asarray(v).reshape(got[k].shape))
    b = tmp_path / "b.bin"
    r = subprocess.run([str(built), "--datafile-echo", str(a), str(b)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.parametrize("damage", ["flip", "truncate", "magic"])
def test_corrupt_files_are_rejected(built, tmp_path, damage):
    a = tmp_path / "a.bin"
    R.write(a, sample())
    raw = bytearray(a.read_bytes())
    if damage == "flip":
        raw[len(raw) // 2] ^= 0x10
    elif damage == "truncate":
        raw = raw[:-20]
    else:
        raw[0:8] = b"HDF5XXXX"
    a.write_bytes(bytes(raw))
    with pytest.raises(R.CorruptFile):
        R.read(a)
    r = subprocess.run([str(built), "--datafile-echo", str(a), str(tmp_path / "b.bin")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "corrupt" in r.stderr


def test_environment_spacing_mismatch_is_rejected(tmp_path):
    cfg = config.workload("periodic32", ppc=1)
    R.save_info(cfg, 42, tmp_path)
    assert R.load_info(cfg, tmp_path) == 42
    other = config.workload("periodic32", ppc=1)
    other.dx = cfg.dx * (1 + 1e-12)
    with pytest.raises(ValueError, match="dx"):
        R.load_info(other, tmp_path)
    other = config.workload("periodic32", ppc=1)
    other.dt = cfg.dt * 2
    with pytest.raises(ValueError, match="dt"):
        R.load_info(other, tmp_path)
    with pytest.raises(ValueError, match="does not exist"):
        R.load_info(cfg, tmp_path / "elsewhere")
