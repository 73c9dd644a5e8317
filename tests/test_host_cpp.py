"""The C++ host side (fopis_b200/host): its input.json loader gives the same
normalised parameters and object node lists as the Python loader, for a
generated input and for the reference's own sample input."""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fopis_b200 import _abi, config

from host_input import write_input

ROOT = Path(__file__).resolve().parent.parent
RUN = ROOT / "fopis_b200" / "fopis_run"
# the reference checkout's sample input (FOPIS_REFERENCE), where given
_REF = os.environ.get("FOPIS_REFERENCE")
SAMPLE = Path(_REF) / "input_samples" / "input.json" if _REF else None


def dump(path, tmp_path):
    out = tmp_path / "params.bin"
    subprocess.run([str(RUN), str(path), "--dump-params", str(out)], check=True, capture_output=True, timeout=120)
    raw = out.read_bytes()
    size = C.sizeof(_abi.Params)
    p = _abi.Params.from_buffer_copy(raw[:size])
    off = size
    nobj = int(np.frombuffer(raw, np.int32, 1, off)[0])
    off += 4
    objs = []
    for _ in range(nobj):
        nn, nc, fixed, emit = np.frombuffer(raw, np.int32, 4, off)
        off += 16
        pot = np.frombuffer(raw, np.float64, 2, off)
        off += 16
        nodes = np.frombuffer(raw, np.int32, 3 * nn, off).reshape(-1, 3)
        off += 12 * nn
        cells = np.frombuffer(raw, np.int32, 3 * nc, off).reshape(-1, 3)
        off += 12 * nc
        sec, diel = np.frombuffer(raw, np.int32, 2, off)
        off += 8
        cap = None
        if diel:
            cap = np.frombuffer(raw, np.float64, nn, off)
            off += 8 * nn
        objs.append((nodes, cells, int(fixed), int(emit), pot, int(sec), int(diel), cap))
    p.plot_energy_width = int(np.frombuffer(raw, np.int32, 1, off)[0])
    return p, objs


def compare(cpp, py):
    p, objs = cpp
    q = py.params
    assert bytes(p) == bytes(q), [(f, getattr(p, f), getattr(q, f)) for f, _ in q._fields_ if
                                  not isinstance(getattr(q, f), (int, float)) or getattr(p, f) != getattr(q, f)]
    assert p.plot_energy_width == py.plot_energy_width
    assert len(objs) == len(py.objects)
    for (nodes, cells, fixed, emit, pot, sec, diel, cap), o in zip(objs, py.objects):
        assert np.array_equal(nodes, o.nodes) and np.array_equal(cells, o.cells)
        assert fixed == o.is_potential_fixed and emit == o.emit_species
        assert pot[0] == o.fixed_potential and pot[1] == o.initial_potential_offset
        assert sec == o.secondary_species and diel == o.dielectric
        if diel:
            assert np.array_equal(cap, o.capacitance)


@pytest.fixture(scope="module")
def built():
    if not RUN.exists():
        subprocess.run(["make", "-C", str(ROOT / "fopis_b200")], check=True, capture_output=True)
    return RUN


@pytest.mark.parametrize("photo", [True, False])
def test_cpp_loader_matches_python(built, tmp_path, photo):
    path = write_input(tmp_path, photo=photo, drift=(50.0, 0.0, -20.0))
    compare(dump(path, tmp_path), config.load_input(str(path)))


def test_cpp_loader_dielectric_and_secondary(built, tmp_path):
    # a dielectric cube of two materials emitting photoelectrons and secondaries
    path = write_input(tmp_path, photo=True, secondary=True, dielectric={"1": "Teflon", "2": "Aluminum"})
    py = config.load_input(str(path))
    assert [s.kind for s in py.species] == ["ambient", "ambient", "photoelectron", "secondary"]
    o = py.objects[0]
    assert o.dielectric == 1 and o.secondary_species == 3 and o.emit_species == 2
    compare(dump(path, tmp_path), py)


@pytest.mark.parametrize("io", [{"plot_energy_width": 7}, {"plot_energy_width": 3.0, "plot_rho_width": 0}, None])
def test_cpp_loader_energy_log_width(built, tmp_path, io):
    """IO.plot_energy_width, cast from a number as Initializer does (Initialize.cpp:219-250);
    without it the energy log is never written (Environment::isPlotTimestep, environment.hpp:266-278)."""
    import json
    path = write_input(tmp_path, photo=False)
    js = json.loads(path.read_text())
    js.pop("IO", None)
    if io is not None:
        js["IO"] = io
    path.write_text(json.dumps(js))
    py = config.load_input(str(path))
    assert py.plot_energy_width == (int(io["plot_energy_width"]) if io else 0)
    compare(dump(path, tmp_path), py)


def test_cpp_loader_on_reference_sample(built, tmp_path):
    if SAMPLE is None or not SAMPLE.exists():
        pytest.skip("reference sample input not available")
    compare(dump(SAMPLE, tmp_path), config.load_input(str(SAMPLE)))


def test_cpp_loader_em_mode(built, tmp_path):
    """solver_type "EM": the solver and the normalised mu0 (include/normalizer.hpp:219-221)
    in the parameters; a time step above the Courant limit is refused by both loaders
    (Environment::checkCFLCondition, src/Misc/Environment.cpp:193-203)."""
    path = write_input(tmp_path / "ok", photo=True, em=True)
    py = config.load_input(str(path))
    assert py.params.solver == _abi.SOLVER_EM and py.params.mu0 > 0
    compare(dump(path, tmp_path), py)
    bad = write_input(tmp_path / "bad", photo=False, em=True, courant=1.5)
    with pytest.raises(ValueError, match="Courant number exceeds 1.0"):
        config.load_input(str(bad))
    r = subprocess.run([str(RUN), str(bad), "--dump-params", str(tmp_path / "x.bin")], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode != 0 and "Courant number exceeds 1.0" in (r.stderr + r.stdout)
