"""bench.py's reference arm and cache note on the CPU.

`bench.py --impl reference` times the CPU restatement of the reference's hydro
path (the oracle) and prints one JSON line with the keys the benchmark
contract names; a small mesh keeps the run to seconds.  The cache note says
whether a stage's working set exceeds L2 for the mesh actually run.
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "32", "--nb", "16",
                        "--steps", "1", "--warmup", "3"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["cells"] == 32 ** 3 and d["config"]["meshblocks"] == 8
    assert d["config"]["cache"].startswith("inputs smaller than L2")


def test_cache_note_follows_the_mesh():
    sys.path.insert(0, str(ROOT))
    try:
        import bench
    finally:
        sys.path.pop(0)
    assert bench.state_vs_l2(256, 32).startswith("inputs larger than L2 (256^3 state: 671 MB FP64, 336 MB FP32;")
    assert bench.state_vs_l2(128, 32).startswith("inputs larger than L2")
    assert bench.state_vs_l2(32, 16).startswith("inputs smaller than L2")
