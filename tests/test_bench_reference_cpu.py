"""CPU: `bench.py --impl reference` prints the reference arm's one JSON line with
the metric, unit, sample description and end-to-end block the bench contract
asks for, on the CPU-runnable periodic 32^3 workload (no GPU involved); the
arm never loads libfopis_gpu.so, and its bodies come from the oracle's own
.obj loader, which gives the same nodes as the product's."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent

# Runs bench.py's reference arm in this interpreter, then reports whether the
# product library was mapped into the process.
_PROBE = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "periodic32", "--steps", "2", "--warmup", "3"]
runpy.run_path(sys.argv[0], run_name="__main__")
maps = open("/proc/self/maps").read()
print("PRODUCT_LIB_LOADED" if "libfopis_gpu" in maps else "PRODUCT_LIB_ABSENT")
"""


def test_reference_arm_prints_contract_line():
    out = subprocess.run([sys.executable, "-c", _PROBE], capture_output=True, text=True, timeout=600, check=True,
                         cwd=str(ROOT))
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "step" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the config block names only the workload, identical on both arms
    assert set(d["config"]) == {"workload", "parallelism", "sort_interval"}
    assert d["config"]["workload"].startswith("periodic32")
    assert "PRODUCT_LIB_ABSENT" in out.stdout


def test_oracle_body_parser_matches_product():
    code = """
import sys
sys.path.insert(0, "oracle")
import numpy as np
import oracle as orc
from fopis_b200 import _abi, config
cfg = config.workload("cube64", obj_parser=orc.parse_obj)
assert _abi._lib is None, "product library loaded"
o = cfg.objects[0]
np.save(sys.argv[1], np.concatenate([o.nodes.ravel(), [-1], o.cells.ravel()]))
"""
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        f = Path(td) / "geom.npy"
        subprocess.run([sys.executable, "-c", code, str(f)], check=True, cwd=str(ROOT), timeout=300)
        got = np.load(f)
    from fopis_b200 import config
    o = config.workload("cube64").objects[0]
    want = np.concatenate([o.nodes.ravel(), [-1], o.cells.ravel()])
    assert np.array_equal(got, want)
