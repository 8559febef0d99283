"""bench.py's reference arm on the CPU: one JSON line with every key the
benchmark contract asks for, the CPU baseline describing the run, and an
end-to-end figure with no host/device traffic."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BENCH = os.path.join(HERE, "..", "bench.py")
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def test_reference_arm_json_line(oracle_lib):
    out = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--n", "32", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["n"] == 32          # the arm runs the configuration its line names
    assert d["value"] > 0 and d["higher_is_better"] is True and d["dtype"] == "f64"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
