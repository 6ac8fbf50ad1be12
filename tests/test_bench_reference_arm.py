"""bench.py's reference arm on CPU (no GPU needed): `--impl reference` times the reference algorithm's CPU
path (the oracle port, OpenMP on all host cores) on the bench workload and prints one JSON line with the
same metric, unit and direction as the GPU arm, a cpu_baseline describing the run and an e2e entry with no
host-device traffic."""
import json
import os
import subprocess
import sys


def test_reference_arm_prints_the_contract_line():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"],
                         cwd=root, capture_output=True, text=True, timeout=900, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    sys.path.insert(0, root)
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["n_gpus"] == 1 and line["warmup"] >= 3
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and isinstance(cb["sample"], str)
    assert cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == bench.WORKLOADS["contact64"]
    assert line["steps"] == 1
