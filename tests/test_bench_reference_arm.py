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


def test_reference_sample_rotation_covers_the_workload():
    """The reference arm's per-step samples: four rotating quarters of the
    64-field workload whose work-weighted field counts add up to exactly
    the workload's 64 fields, so any multiple of four steps times the same
    configuration as the GPU arm."""
    sys.path.insert(0, str(REPO))
    import bench
    fields = bench.workload(1000)
    qs = bench.quarter_samples(fields)
    assert len(qs) == 4 and sum(len(q) for q in qs) == len(fields) == 64
    assert [f for q in qs for f in q] == fields
    eq = [bench.field_equivalents(q, fields) for q in qs]
    assert abs(sum(eq) - 64.0) < 1e-9
    assert all(e > 0 for e in eq)
