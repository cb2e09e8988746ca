"""Host-side pieces of the benchmark that run without a GPU: the DRAM traffic
figure the roofline reports comes from the committed ncu summary, the
reference arm's line keeps the contract's keys and times the GPU line's
config, and the parity checkers find differences."""
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
    assert d["config"]["text_bytes"] == 64 << 20  # the whole document, the GPU line's config
    assert set(d["cpu_baseline"]["stage_ms"]) == {"parse_par", "build_links", "find_all_par"}


def test_first_mismatch_names_the_first_difference():
    import numpy as np

    a = np.arange(10, dtype=np.uint32)
    assert bench.first_mismatch("x", a, a.copy()) is None
    b = a.copy()
    b[7] = 0
    b[9] = 1
    assert bench.first_mismatch("x", b, a) == "x[7]: 0 vs 7 (2 differ)"
    assert "entries" in bench.first_mismatch("x", a[:5], a)


def test_device_hit_digest_equals_the_cpu_ports_digest():
    """The checker's torch digest (run here on a CPU tensor) of the oracle's sorted
    hit list equals the CPU port's digest, and a swapped pair changes it."""
    import numpy as np
    import torch

    import oracle
    from oneline_b200 import datagen

    text = datagen.corpus(1 << 20, 8)
    pats = datagen.patterns_dictionary(text, 8, n=100)
    counts, hp, ho = oracle.find_many(text, pats)
    hits = np.empty(2 * len(hp), np.uint32)
    hits[0::2], hits[1::2] = hp, ho
    t = torch.from_numpy(hits.view(np.int32).copy())
    _, total, dg = oracle.CpuBaseline(threads=2).many(pats).digest_par(text)
    assert total == len(hp)
    assert bench.device_hit_digest(t, total, chunk=1000) == dg
    hits[2:4], hits[4:6] = hits[4:6].copy(), hits[2:4].copy()
    assert bench.device_hit_digest(torch.from_numpy(hits.view(np.int32).copy()), total) != dg


def test_serve_client_buffers_have_room_and_are_reused():
    """The serve client's result buffers: every parse gets a set with room for
    its lines (the serve corpus has fewer than one line per 8 bytes), sets are
    pooled per room, and search sets hold SERVE_MAX_HITS hits."""
    import numpy as np

    from oneline_b200 import HIT_DTYPE

    for n in (0, 1, 1000, 64 << 10, (64 << 20) - 1, 64 << 20):
        room = bench.serve_room(n)
        assert room >= n // 8 + 4096 and room & (room - 1) == 0 and room >= 1 << 12
    reqs = [("parse", 0.0, np.zeros(n, np.uint8)) for n in (1000, 1000, 5 << 20)]
    reqs += [("search", 0.1, [b"abcd"], 0)]
    pool = bench.serve_buffer_pool(reqs)
    assert len(pool["search"]) == 128 and pool["search"][0]["hits"].dtype == HIT_DTYPE
    assert pool["search"][0]["hits"].size == bench.SERVE_MAX_HITS
    small, big = bench.serve_room(1000), bench.serve_room(5 << 20)
    assert len(pool[small]) == 2 and len(pool[big]) == 1
    s = pool[big][0]
    assert all(a.size == big for a in s.values()) and s["kinds"].dtype == np.uint8 and s["offsets"].dtype == np.uint32
