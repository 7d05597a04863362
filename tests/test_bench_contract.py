"""bench.py's output contract, checked on the CPU: the reference arm of the
build workload, on a small sample, prints one JSON line with the keys and
meanings the benchmark driver reads."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--cpu-sample", "2000", "--fit-rows", "5000", "--n", "100000"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    j = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in j, key
    assert j["impl"] == "reference" and j["n_gpus"] == 1 and j["steps"] == 1
    assert j["unit"] == "s" and j["higher_is_better"] is False and j["value"] > 0
    assert "workload" in j["config"] and "model" not in j["config"]
    cb = j["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == j["value"]
    assert j["e2e"]["value"] == j["value"] and j["e2e"]["unit"] == j["unit"]
    assert j["e2e"]["h2d_bytes_per_step"] == 0 and j["e2e"]["d2h_bytes_per_step"] == 0
    # extrapolated by the power law through the two measured sizes
    c = j["config"]
    assert c["sample_rows"] == 2000 and c["fit_rows"] == 5000
    assert abs(c["t_fit_rows_s"] * (100000 / 5000) ** c["alpha"] - j["value"]) <= 1e-9 * j["value"]
