"""The reference arm of ``bench.py`` on the host cores (CPU, no GPU needed).

``bench.py --impl reference`` times the oracle restatement of the reference
path on each workload and prints one JSON line; the line must carry the
metric, unit and value of the workload, ``"impl": "reference"``, a
``cpu_baseline`` describing the run and an ``e2e`` object with zero copy
bytes, or an ``unavailable`` reason where the reference has no counterpart.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(workload):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          workload, "--steps", "1", "--warmup", "0", "--cpu-per-b", "1"], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["energy_batch", "plain_large", "large_mixed", "bcr_batch"])
def test_reference_arm_line(workload):
    line = _run(workload)
    assert line["impl"] == "reference"
    assert line["unit"] == "matrices/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["metric"]
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["cores"] >= 1 and cpu["kind"] in ("port", "reference")
    assert cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("workload", ["gradient_set", "lesser_batch"])
def test_reference_arm_without_counterpart(workload):
    line = _run(workload)
    assert line["impl"] == "reference" and "unavailable" in line
