"""The bench's reference arm on the CPU: the oracle's timed sample prints one JSON line with the
keys the reference arm must carry (impl, metric, value, unit, e2e, cpu_baseline)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("approach", ["tree", "list"])
def test_reference_arm_line(approach):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--approach", approach, "--workload", "plain_64m",
                        "--cpu-sample-bytes", str(8 << 20)], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == f"{approach}-dedup ingest GB/s"
    assert line["unit"] == "GB/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["config"]["approach"] == approach
    # the line's config names the buffer size it actually timed
    assert line["config"]["nbytes"] == 8 << 20 and "0.0078125 GiB" in cb["sample"]
