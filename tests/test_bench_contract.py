"""bench.py's reference arm runs on the host cores and prints the one JSON
line the benchmark contract asks for (same metric, unit and workload as the
GPU arm, a cpu_baseline record and a host-only e2e record)."""

import json
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    import bench

    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "trajectories/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] >= 3
    assert d["config"]["workload"] == bench.WORKLOAD
    # warm-up and timed steps each take the next block of theta rows
    per = d["config"]["sample_theta_per_step"]
    assert d["config"]["theta_rows_covered"] == min(bench.N_THETA, 4 * per)
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
