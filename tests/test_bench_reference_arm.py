"""bench.py's reference arm on the host cores (no GPU): the compiled
reference engine runs the frame-buffer and sequence-window workloads and
prints one JSON line with the keys the bench contract asks for."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("workload", ["frames8-ntsc", "window6-ntsc"])
def test_reference_arm_json_line(workload):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference engine not built")
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), "--workload", workload,
                          "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "frames/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
