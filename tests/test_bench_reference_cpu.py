"""CPU: `bench.py --impl reference` prints the reference arm's one JSON line with
the metric, unit, sample description and end-to-end block the bench contract
asks for, on the CPU-runnable periodic 32^3 workload (no GPU involved)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "periodic32",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "step" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("periodic32")
