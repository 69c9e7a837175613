"""The reference arm of bench.py on CPU: it times the oracle (the CPU
restatement of the reference's codec; the reference itself has no CPU
codec) on every frame of the mix (scaled down to 12 frames here) and prints
one JSON line with the same metric, unit and workload as the GPU arm."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--frames", "12"], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Gpix/s encode+decode" and d["unit"] == "Gpix/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 1, 1)
    assert d["scaling"] == "weak" and d["vs_baseline"] is None and d["dtype"] == "u16"
    assert d["config"]["workload"].startswith("mixed96")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == "Gpix/s" and cb["kind"] == "port" and cb["cores"] >= 1
    assert "all 12 frames" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
