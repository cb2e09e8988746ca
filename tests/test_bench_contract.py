"""Host-side pieces of the benchmark that run without a GPU: the DRAM traffic
figure the roofline reports comes from the committed ncu summary, and the
reference arm's line keeps the contract's keys."""
import json
import subprocess
import sys
import os

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_roofline_traffic_comes_from_the_committed_ncu_summary():
    t = bench.profiled_traffic("search_stage_copy_8patterns_256mib.md", "traffic_bytes_per_1gib_pass")
    assert t is not None and 1_400_000_000 < t < 2_000_000_000  # about 1.04x the pass's algorithmic bytes
    assert bench.profiled_traffic("search_stage_copy_8patterns_256mib.md", "no_such_key") is None
    assert bench.profiled_traffic("no_such_profile.md", "traffic_bytes_per_1gib_pass") is None


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--bytes", str(64 << 20)], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
