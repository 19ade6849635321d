"""The benchmark's JSON contract on the CPU: the per-cell byte counts behind
the roofline figure, and one short run of the reference arm (the reference's
own RHS on the host cores) printing the fields a reader of the bench line
relies on."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle  # noqa: E402


def test_algorithmic_bytes_per_cell_update():
    # P = 12 phase field, no chemistry: 130 B mixed (4-byte phi/T), 234 B FP64
    assert bench.survey_bytes_per_cell(12, 0, 0, 4) == 130
    assert bench.survey_bytes_per_cell(12, 0, 0, 8) == 234


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
