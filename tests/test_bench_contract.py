"""The JSON line of bench.py's reference arm (the CPU path timed beside the
GPU one): it runs on the host cores only, so it is checked here on CPU."""
import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"],
                         capture_output=True, text=True, timeout=600, cwd=REPO, check=True).stdout
    d = json.loads(out.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["metric"].startswith("external-mode cell-iter/s") and d["unit"] == "cell-iter/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert cb["unit"] == d["unit"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["members"] == 256 and d["config"]["workload"]
