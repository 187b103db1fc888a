"""The reference arm of bench.py on the host (CPU).

`bench.py --impl reference` times the reference path (the oracle port of the
reference's DF-RHF) on the host cores and prints one JSON line with the same
metric as the B200 arm. This checks the line's contract: impl, metric, unit,
direction, a positive value, and the cpu_baseline and e2e objects.
"""

from __future__ import annotations

import json
import subprocess
import sys

from tests.conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--fit-waters", "4"], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    import bench

    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    assert line["unit"] == "s" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert [p["waters"] for p in line["measured"]] == [8, 4]
    assert line["cpu_baseline"]["extrapolated"] is True and "fit" in line
