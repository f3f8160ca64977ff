"""The benchmark's reference arm (`bench.py --impl reference`) on a small case: it runs on the
host cores only and prints one JSON line with the keys of the benchmark contract."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--n", "8192",
                        "--steps", "1", "--warmup", "1", "--cpu-sample-seconds", "1"],
                       capture_output=True, text=True, timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["unit"] == "particles/s" and line["value"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["config"]["n"] == 8192
    # ms_per_step is the measured sample step, not an extrapolation: steps x ms_per_step fits the run
    assert 0 < line["ms_per_step"] < 60e3
    assert 0 < line["sample"]["fraction_of_matvec_evals"] <= 1.0
