"""bench.py's reference arm runs only the reference CPU path, so its JSON line
is checked here on a tiny field loop: the keys the benchmark contract asks
for, the reference kind and a positive throughput."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line():
    if not (ROOT / "oracle" / "_ref" / "athref_field_loop_roe").exists():
        pytest.skip("oracle/_ref not built")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--nx", "64", "--ny", "32",
                        "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "field_loop 64x32"
