"""Benchmark of the oneline parse-and-search hot path on B200.

Default workload (one step): a 1 GiB synthetic oneline document (seed 1), full
parse (newline scan + classification, tree links) and an 8-pattern substring
search with pattern lengths 4..1024 B (even indices sampled from the text, odd
indices random bytes). Inputs (1 GiB) are larger than L2, so no flush is needed.

  value   : text GB/s of the device pipeline with the text resident in HBM
            (CUDA events on the engine's stream, max over ranks, whole job);
  e2e     : the same through the C ABI with host buffers (pinned upload, parse,
            tree, searches, download of offsets/kinds/tree arrays/hits);
  roofline: the dominant kernel's algorithmic bytes per launch / its average
            launch time, against the measured HBM copy bandwidth;
  cpu_baseline: the multi-threaded C++ port of the reference's CPU engine on the
            same 1 GiB document, on all host cores, with per-stage times;
  parity  : after the timed region, every output of the last timed step
            (offsets, kinds, 16-byte nodes, parent, subtree_end, first_child,
            next_sibling, every hit of the 8 patterns) compared element by
            element with the CPU port's outputs on the same document;
  dictionary: the 10,000-pattern dictionary search of a 1 GiB document (seed 2)
            as a sub-record, with its own roofline, e2e, CPU baseline and
            parity (exact per-pattern counts, an order-checking digest of all
            hits, and the full hit lists of sampled patterns).

`--impl reference` times that CPU port alone (rank 0; other ranks exit).
Multi-GPU (torchrun): each rank parses and searches its own document (replicas,
weak scaling); there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "parse+search GB/s vs HBM peak"


def profiled_traffic(name: str, key: str):
    """DRAM bytes per launch recorded from an ncu capture in a profiles/
    summary (a line `key: <bytes>`), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return int(line.split(":", 1)[1].strip())
    except (OSError, ValueError):
        pass
    return None


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bytes", type=int, default=1 << 30, help="document size (default 1 GiB)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-workers", type=int, default=3, help="concurrent end-to-end steps (contexts)")
    ap.add_argument("--cpu-reps", type=int, default=2, help="timed CPU-port steps in the cpu_baseline leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and the parity check")
    ap.add_argument("--no-dictionary", action="store_true",
                    help="skip the dictionary sub-record of the default workload")
    ap.add_argument("--dict-bytes", type=int, default=1 << 30, help="dictionary document size (default 1 GiB)")
    ap.add_argument("--dict-cpu-sample-mb", type=int, default=128,
                    help="prefix of the dictionary document timed on the CPU port")
    ap.add_argument("--clock-log", default=None,
                    help="file for the nvidia-smi clock log of the timed region (default: a temp file)")
    ap.add_argument("--no-graph", action="store_true", help="enqueue the headline step call by call, no CUDA graph")
    ap.add_argument("--profile-launches", action="store_true",
                    help="one short run for an ncu launch list (no e2e, no CPU leg)")
    ap.add_argument("--workload", default="parse_search", choices=["parse_search", "dictionary", "batch", "serve"],
                    help="parse_search: 1 GiB parse + 8-pattern search (the headline); dictionary: 1 GiB x "
                         "10,000 patterns; batch: 10,000 uneven documents, batched vs one call per document; "
                         "serve: open-loop Poisson parse/search requests, concurrent workers vs one")
    ap.add_argument("--pattern-source-bytes", type=int, default=0,
                    help="sample the 8 patterns from the document of this size (the text is its prefix)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="length of the serve workload's arrival stream")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch sub-record of the default workload")
    ap.add_argument("--no-serve", action="store_true", help="skip the serve sub-record of the default workload")
    ap.add_argument("--serve-workers", type=int, default=8)
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="mean arrivals per second")
    ap.add_argument("--serve-overload-rate", type=float, default=8000.0,
                    help="arrival rate of the second, overloaded serve stream (0: skip it)")
    ap.add_argument("--serve-overload-seconds", type=float, default=10.0)
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 2 ms from a thread (read-only queries), plus a
    nvidia-smi log (100 ms) written to `log_path` (default: a temp file)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    log_path = None  # set from --clock-log

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.samples = []
        self.max_mhz = None
        base = ClockSampler.log_path or os.path.join(tempfile.gettempdir(), "oneline_clocks.csv")
        root, ext = os.path.splitext(base)
        self.path = f"{root}_rank{index}{ext or '.csv'}"

    def _poll(self):
        import pynvml

        h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        while not self._stop.is_set():
            sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
            r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, r))
            self._stop.wait(0.002)

    def __enter__(self):
        import threading

        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join()
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        import pynvml

        if self.samples:
            names = [n for n, attr in self.REASONS if any(r & getattr(pynvml, attr) for _, r in self.samples)]
            return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": names, "samples": len(self.samples), "source": "NVML every 2 ms"}
        try:  # nvidia-smi log only
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
            sm = [float(r[1]) for r in rows]
            mx = float(rows[0][2]) if rows else None
            names = [n for n, _ in self.REASONS]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                    "samples": len(rows), "source": "nvidia-smi every 100 ms"}
        except Exception as e:  # nvidia-smi missing
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)[:80]}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def _reduce_device():
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def allreduce_max(x: float, world: int) -> float:
    """The largest value over the ranks (step times: the job is as slow as its slowest replica)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float, world: int) -> float:
    """The sum over the ranks (bytes processed by all replicas)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------ workload

def make_workload(nbytes: int, seed: int, pattern_source_bytes: int = 0):
    """The document and its 8 patterns. With pattern_source_bytes > nbytes the
    patterns are those of the larger document of the same seed, of which the text
    is the prefix (profiling the full-size patterns on a smaller text)."""
    from oneline_b200 import datagen

    if pattern_source_bytes > nbytes:
        big = datagen.corpus(pattern_source_bytes, seed)
        return np.ascontiguousarray(big[:nbytes]), datagen.patterns_eight(big, seed)
    text = datagen.corpus(nbytes, seed)
    pats = datagen.patterns_eight(text, seed)
    return text, pats


class CpuPort:
    """The reference's CPU path on one document: the multi-threaded C++ port of
    oneline-simd (parse_par, build_links + first_child/next_sibling, one
    find_all_par per pattern) on `threads` host cores. Outputs are allocated
    once and reused by every step, as ParseBuffers does
    (crates/oneline-simd/src/lib.rs:445-469); each search writes into a buffer
    sized by a first run. The outputs of the last step are the parity reference
    for the GPU's."""

    STAGES = ("parse_par", "build_links", "find_all_par")

    def __init__(self, text: np.ndarray, pats, threads: int | None = None):
        import oracle

        self.base = oracle.CpuBaseline(threads)
        self.threads = self.base.threads
        self.text = np.ascontiguousarray(text)
        self.pats = [bytes(x) for x in pats]
        n = self.base.line_count(self.text)
        self.lines = n
        self.offsets = np.empty(max(n, 1), np.uint32)
        self.nodes = np.empty(max(n, 1), oracle.NODE_DTYPE)
        self.tree = {k: np.empty(max(n, 1), np.uint32) for k in TREE_KEYS}
        self.totals = [self.base.find_all_par(self.text, x, np.empty(1, np.uint32))[0] for x in self.pats]
        self.hits = [np.empty(max(t, 1), np.uint32) for t in self.totals]

    def step(self) -> dict:
        """One pass of the path; returns the seconds per stage."""
        t0 = time.perf_counter()
        got = self.base.parse_par_into(self.text.ctypes.data, self.text.size, self.offsets, self.nodes)
        assert got == self.lines
        t1 = time.perf_counter()
        self.base.build_links(self.nodes[: self.lines], out=self.tree)
        t2 = time.perf_counter()
        for i, x in enumerate(self.pats):
            total, _ = self.base.find_all_par(self.text, x, self.hits[i])
            assert total == self.totals[i]
        t3 = time.perf_counter()
        return {"parse_par": t1 - t0, "build_links": t2 - t1, "find_all_par": t3 - t2, "step": t3 - t0}


TREE_KEYS = ("parent", "subtree_end", "first_child", "next_sibling")

# The reference's published CPU figures for these stages (RTX 3060 host, 12
# threads; .agents/tasks/*.md), scaled per thread for comparison.
PUBLISHED_CPU = {
    "parse_par": {"value": "1 GiB HTML in 64 ms (16.8 GB/s) on 12 threads",
                  "source": ".agents/tasks/gpu-profiling-and-overhead.md:139"},
    "build_links": {"value": "1 GiB mixed (13 M lines) in 40.2 ms on 12 threads",
                    "source": ".agents/tasks/gpu-tree-construction.md:14"},
    "find_all_par": {"value": "1 GiB, one sparse pattern, 27 ms on 12 threads",
                     "source": ".agents/tasks/gpu-substring-search.md:151"},
}


def cpu_leg(text: np.ndarray, pats, reps: int = 2) -> tuple[dict, CpuPort]:
    """The reference CPU path (port) on all host cores over the whole document:
    one warm-up step, then the median of `reps` steps, with per-stage times."""
    port = CpuPort(text, pats)
    port.step()
    runs = [port.step() for _ in range(max(reps, 1))]
    med = {k: statistics.median(r[k] for r in runs) for k in runs[0]}
    n = port.text.size
    stages = {k: {"ms": round(med[k] * 1e3, 2), "published": PUBLISHED_CPU[k]} for k in CpuPort.STAGES}
    stages["parse_par"]["gb_per_s"] = round(n / med["parse_par"] / 1e9, 3)
    stages["build_links"]["ns_per_line_thread"] = round(med["build_links"] * 1e9 * port.threads / max(port.lines, 1), 1)
    stages["find_all_par"]["patterns"] = len(port.pats)
    rec = {"value": round(n / med["step"] / 1e9, 4), "unit": "GB/s", "cores": port.threads, "kind": "port",
           "sample": f"the whole {n}-byte document (the same config as the GPU line): parse_par + build_links + "
                     f"children + {len(port.pats)} x find_all_par into preallocated outputs, median of {len(runs)} "
                     "after 1 warm-up (C++ port of oneline-simd; the Rust reference cannot be built here)",
           "seconds_per_rep": round(med["step"], 4), "stages": stages}
    return rec, port


def first_mismatch(name: str, got: np.ndarray, want: np.ndarray):
    """None when equal, else a one-line description of the first difference."""
    got, want = np.asarray(got), np.asarray(want)
    if got.shape != want.shape:
        return f"{name}: {got.size} entries vs {want.size}"
    bad = np.flatnonzero(got != want)
    if bad.size == 0:
        return None
    i = int(bad[0])
    return f"{name}[{i}]: {got[i]} vs {want[i]} ({bad.size} differ)"


def parity_parse_search(doc, tree, parser, hit_outs, d_totals, port: CpuPort) -> dict:
    """Every output of the GPU's last step against the CPU port on the same
    document, element by element (the port is itself checked against the oracle
    in the CPU tests)."""
    L = port.lines
    checks = []
    got_offs = doc.read_offsets()
    checks.append(first_mismatch("offsets", got_offs, port.offsets[:L]))
    checks.append(first_mismatch("kinds", doc.read_kinds(), port.nodes["kind"][:L].astype(np.uint8)))
    nodes = doc.read_nodes()
    for f in ("depth", "kind", "span_start", "span_len"):
        checks.append(first_mismatch(f"nodes.{f}", nodes[f], port.nodes[f][:L]))
    t = parser.download_tree(tree)
    for k in TREE_KEYS:
        checks.append(first_mismatch(k, t[k], port.tree[k][:L]))
    tots = d_totals.cpu().numpy().view(np.uint32)
    for i, (o, want_t) in enumerate(zip(hit_outs, port.totals)):
        checks.append(None if int(tots[i]) == want_t else f"total[{i}]: {int(tots[i])} vs {want_t}")
        checks.append(first_mismatch(f"hits[{i}]", o[:want_t].cpu().numpy().view(np.uint32), port.hits[i][:want_t]))
    bad = [c for c in checks if c]
    return {"result": "bit-exact" if not bad else "MISMATCH", "first_mismatch": bad[0] if bad else None,
            "compared": f"{L} offsets, kinds and 16-byte nodes; parent, subtree_end, first_child, next_sibling; "
                        f"{sum(port.totals)} hits of {len(port.totals)} patterns",
            "against": f"the CPU port of oneline-simd on the same document ({port.threads} threads)"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    text, pats = make_workload(args.bytes, args.seed)
    port = CpuPort(text, pats)
    for _ in range(args.warmup):
        port.step()
    t0 = time.perf_counter()
    runs = [port.step() for _ in range(args.steps)]
    dt = (time.perf_counter() - t0) / args.steps
    v = text.size / dt / 1e9
    med = {k: round(statistics.median(r[k] for r in runs) * 1e3, 2) for k in CpuPort.STAGES}
    line = {"metric": METRIC, "value": round(v, 4), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(args, text.size, pats, port.lines),
            "cpu_baseline": {"value": round(v, 4), "unit": "GB/s", "cores": port.threads, "kind": "port",
                             "sample": f"the whole {text.size}-byte document every step: parse_par + build_links + "
                                       f"children + {len(pats)} x find_all_par into preallocated outputs (C++ port "
                                       "of oneline-simd on all host threads)",
                             "stage_ms": med},
            "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args, nbytes, pats, lines):
    return {"workload": f"{nbytes}-byte synthetic oneline document: full parse (newline scan, classify, tree "
                        f"parent/first_child/next_sibling/subtree_end) + {len(pats)}-pattern substring search "
                        f"(lengths {[len(p) for p in pats]})",
            "text_bytes": int(nbytes), "lines": lines, "seed": args.seed,
            "l2": "inputs larger than L2 (no flush needed)" if nbytes > (126 << 20) else "L2 flushed between steps",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU"}


# ------------------------------------------------------------------ our arm

def run_ours(args, world, rank, local):
    import torch

    from oneline_b200 import GpuParser, _lib

    L = _lib.load()
    text, pats = make_workload(args.bytes, args.seed + rank, args.pattern_source_bytes)
    N = text.size
    torch.cuda.set_device(local)
    p = GpuParser(local)
    host = torch.empty(N, dtype=torch.uint8, pin_memory=True)
    host.numpy()[:] = text

    # Resident document and tree; exact hit counts for the output buffers.
    doc = p.upload(host.numpy())
    tree = p.build_tree(doc)
    lines = doc.line_count()
    totals = [p.search_document(doc, pt, 0, max_pattern_len=None).total_matches for pt in pats]
    outs = [torch.empty(max(t, 1), dtype=torch.int32, device=f"cuda:{local}") for t in totals]
    d_tot = torch.zeros(len(pats), dtype=torch.int32, device=f"cuda:{local}")
    pbufs = [np.frombuffer(pt, np.uint8) for pt in pats]
    stream = torch.cuda.ExternalStream(L.ol_ctx_stream(p.ctx), device=f"cuda:{local}")

    def chk(s):
        if s != 0:
            raise RuntimeError(L.ol_last_error(p.ctx).decode())

    def enqueue_parse():
        chk(L.ol_doc_reparse_async(p.ctx, doc.handle))

    def enqueue_tree():
        chk(L.ol_tree_rebuild_async(p.ctx, doc.handle, tree.handle))

    n_p = len(pats)
    P = (ctypes.c_void_p * n_p)(*[b.ctypes.data for b in pbufs])
    lens = np.array([len(x) for x in pats], np.uint32)
    maxes = np.array(totals, np.uint32)
    O = (ctypes.c_void_p * n_p)(*[o.data_ptr() for o in outs])

    def enqueue_search():
        chk(L.ol_search_multi_async(p.ctx, doc.handle, P, lens.ctypes.data, n_p, maxes.ctypes.data,
                                    d_tot.data_ptr(), O))

    def step():
        enqueue_parse()
        enqueue_tree()
        enqueue_search()

    if args.profile_launches:
        for _ in range(args.warmup + args.steps):
            step()
        p.sync()
        return

    # Per-kernel timing pass (outside the timed region): events around each launch group.
    def timed(fn, reps=3):
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                a.record()
            fn()
            with torch.cuda.stream(stream):
                b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    for _ in range(2):
        step()
    p.sync()
    t_parse = timed(enqueue_parse)
    t_tree = timed(enqueue_tree)
    t_search = timed(enqueue_search)

    # Timed region: the step replayed as one CUDA graph (or, with --no-graph,
    # enqueued call by call).
    run_step, tstream, per_step = step, stream, None
    if not args.no_graph:
        pipe = p.capture_pipeline(doc, tree, pats, maxes, d_tot.data_ptr(), [o.data_ptr() for o in outs])
        run_step = pipe.launch
        tstream = torch.cuda.ExternalStream(pipe.stream, device=f"cuda:{local}")
        per_step = pipe.kernels
    for _ in range(args.warmup):
        run_step()
    p.sync()
    torch.cuda.synchronize(local)
    if not args.no_graph:
        pipe.sync()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = L.ol_launch_count()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(tstream):
            ev0.record()
        for _ in range(args.steps):
            run_step()
        with torch.cuda.stream(tstream):
            ev1.record()
        ev1.synchronize()
    # graph replays launch the captured kernels without passing the library's counter
    launches = per_step * args.steps if per_step is not None else L.ol_launch_count() - l0
    torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = allreduce_max(ms, world)
    bytes_all = allreduce_sum(float(N), world)
    value = bytes_all / (ms_max * 1e-3) / 1e9

    # Check the timed outputs once more against the first (blocking) results.
    got_tot = d_tot.cpu().numpy().astype(np.int64)
    assert list(got_tot) == totals, "search totals changed between runs"

    # Roofline of the dominant kernel group.
    peak, peak_kind = hbm_peak()
    hits = sum(totals)
    # algorithmic bytes: text read once per launch + every output byte once
    groups = {"parse pass (newline_count, scan, parse_tiles, fixup)": (t_parse, N + 6 * lines),
              "tree pass (summary, scan, resolve)": (t_tree, 2 * lines + 16 * lines),
              "8-pattern search pass (search_stage, scan, search_copy, search_write)": (t_search, N + 4 * hits)}
    dom = max(groups, key=lambda k: groups[k][0])
    t_launch = groups[dom][0]
    alg = groups[dom][1]
    achieved = alg / (t_launch * 1e-3) / 1e9
    traffic = None
    if dom.startswith("8-pattern search") and N == 1 << 30 and args.seed == 1 and args.pattern_source_bytes in (0, N):
        traffic = profiled_traffic("search_stage_copy_8patterns_256mib.md", "traffic_bytes_per_1gib_pass")
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind, "traffic": traffic,
                "traffic_source": "ncu dram read+write of the pass's kernels at 256 MiB, x4 (profiles/)"
                if traffic else None,
                "alg_bytes_per_launch": int(alg), "ms_per_launch": round(t_launch, 4),
                "ms_parse": round(t_parse, 4), "ms_tree": round(t_tree, 4),
                "ms_search": round(t_search, 4)}

    # End to end through the C ABI with host buffers: `e2e_workers` host threads,
    # each with its own context (stream) and pinned output buffers, run whole
    # steps concurrently. One lock per copy direction keeps one upload and one
    # download in flight at a time: each gets the link to itself, and one
    # step's upload overlaps another's downloads instead of the threads
    # uploading (then downloading) at the same time.
    e2e = None
    if args.e2e_steps > 0:
        import threading

        workers = max(1, args.e2e_workers)
        ctxs = [p] + [GpuParser(local) for _ in range(workers - 1)]
        h2d_lock, d2h_lock = threading.Lock(), threading.Lock()

        def make_step(q):
            offs_h = torch.empty(lines, dtype=torch.int32, pin_memory=True).numpy()
            kinds_h = torch.empty(lines, dtype=torch.uint8, pin_memory=True).numpy()
            tree_h = [torch.empty(lines, dtype=torch.int32, pin_memory=True).numpy() for _ in range(4)]
            hits_h = [torch.empty(max(t, 1), dtype=torch.int32, pin_memory=True).numpy() for t in totals]
            tots_h = np.zeros(n_p, np.uint32)
            OH = (ctypes.c_void_p * n_p)(*[a.ctypes.data for a in hits_h])

            def e2e_step():
                h = ctypes.c_void_p()
                with h2d_lock:
                    chk(L.ol_doc_upload(q.ctx, host.data_ptr(), N, ctypes.byref(h)))
                t = ctypes.c_void_p()
                chk(L.ol_tree_build(q.ctx, h.value, 1, ctypes.byref(t)))
                with d2h_lock:
                    chk(L.ol_search_multi(q.ctx, h.value, P, lens.ctypes.data, n_p, maxes.ctypes.data,
                                          tots_h.ctypes.data, OH))
                    chk(L.ol_doc_read_offsets(q.ctx, h.value, offs_h.ctypes.data, lines))
                    chk(L.ol_doc_read_kinds(q.ctx, h.value, kinds_h.ctypes.data, lines))
                    chk(L.ol_tree_read(q.ctx, t.value, *[a.ctypes.data for a in tree_h], lines))
                L.ol_tree_free(t.value)
                L.ol_doc_free(h.value)
                assert list(tots_h) == totals
            return e2e_step

        steps = [make_step(q) for q in ctxs]
        for f in steps:
            f()  # warm-up: every context's buffers and kernels
        barrier(world)
        threads = [threading.Thread(target=lambda f=f: [f() for _ in range(args.e2e_steps)]) for f in steps]
        t0 = time.perf_counter()
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        dt = (time.perf_counter() - t0) / (args.e2e_steps * workers)
        dt = allreduce_max(dt, world)
        for q in ctxs[1:]:
            q.close()
        e2e = {"value": round(bytes_all / dt / 1e9, 4), "unit": "GB/s", "ms_per_step": round(dt * 1e3, 3),
               "h2d_bytes_per_step": int(N), "d2h_bytes_per_step": int(21 * lines + 4 * hits),
               "workers": workers,
               "timing": "host wall clock around blocking C-ABI calls (steps of all workers / wall time), max over ranks",
               "path": "per step: ol_doc_upload (pinned) + ol_tree_build + ol_search_multi (8 patterns) + "
                       "ol_doc_read_offsets/kinds + ol_tree_read (4 arrays), on `workers` contexts at once, "
                       "one upload and one download in flight at a time"}

    # CPU baseline (rank 0, all host cores, while the other ranks wait), then
    # parity on every rank: the outputs of the last timed step against the CPU
    # port on the same document (rank 0 reuses its timed port's outputs).
    cpu, parity = None, None
    if not args.no_cpu:
        port = None
        if rank == 0:
            cpu, port = cpu_leg(text, pats, args.cpu_reps)
        barrier(world)
        if port is None:
            port = CpuPort(text, pats, threads=max(1, (os.cpu_count() or 1) // world))
            port.step()
        parity = parity_parse_search(doc, tree, p, outs, d_tot, port)
        bad = allreduce_sum(0.0 if parity["result"] == "bit-exact" else 1.0, world)
        if world > 1:
            parity["ranks_checked"] = world
            parity["ranks_mismatched"] = int(bad)
        del port

    # Sub-records of the other workloads, at N = 1 only (a scaling run times the
    # headline alone).
    dict_rec = batch_rec = serve_rec = None
    if not args.no_graph:
        pipe.free()
    del outs
    def sub_record(fn, *a):
        # a sub-record that fails is reported as such; the headline line stands
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            import traceback

            traceback.print_exc()
            return {"error": f"{type(e).__name__}: {e}"[:300]}

    if world == 1 and not args.no_dictionary:
        dict_rec = sub_record(dictionary_record, args, world, rank, local, p)
    if world == 1 and not args.no_batch:
        batch_rec = sub_record(batch_record, args, world, rank, local, p)
    if world == 1 and not args.no_serve:
        serve_rec = sub_record(serve_record, args, local)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                "config": {**workload_config(args, N, pats, lines), "hits": totals},
                "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "e2e": e2e,
                "gpu_launches": int(launches), "clocks": clocks.summary(),
                "step_form": "CUDA graph (ol_pipeline_launch)" if not args.no_graph else "enqueued calls",
                "dictionary": dict_rec, "batch": batch_rec, "serve": serve_rec, "device": p.adapter_name()}
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------ dictionary

_U64 = (1 << 64) - 1


def _i64(c: int) -> int:
    """A 64-bit constant as torch's signed int64."""
    return c - (1 << 64) if c >= 1 << 63 else c


def device_hit_digest(hits_i32, total: int, chunk: int = 1 << 27) -> int:
    """The order-checking digest of a device hit list {pattern u32, offset u32}[total]:
    the sum over slots i of the CPU port's hit_digest(i, pattern, offset) mod 2^64,
    computed with torch on the device in chunks (int64 arithmetic wraps)."""
    import torch

    def lsr(x, k):  # logical shift right of int64
        return (x >> k) & ((1 << (64 - k)) - 1)

    v64 = hits_i32.view(torch.int64)[:total]
    k0, k1, k2 = _i64(0x9E3779B97F4A7C15), _i64(0xBF58476D1CE4E5B9), _i64(0x94D049BB133111EB)
    acc = 0
    for s0 in range(0, total, chunk):
        v = v64[s0: s0 + chunk]
        slot = torch.arange(s0, s0 + v.numel(), dtype=torch.int64, device=v.device)
        x = ((v << 32) | lsr(v, 32)) ^ (slot * k0)  # (pattern << 32) | offset
        del slot
        x = x ^ lsr(x, 30)
        x = x * k1
        x = x ^ lsr(x, 27)
        x = x * k2
        x = x ^ lsr(x, 31)
        acc += int(x.sum().item())
        del x
    return acc & _U64


def parity_dictionary(text: np.ndarray, pats, counts: np.ndarray, total: int, d_hits, threads: int) -> dict:
    """The GPU's dictionary result over the whole document against the CPU port:
    every pattern's count, the total and the order-checking digest of all hits
    (hit_digest summed over the (pattern, offset)-ordered slots, without
    building the list on the host), plus, element by element, the full hit lists
    of the three most frequent patterns and five others (find_all_par on the
    whole document)."""
    import oracle

    base = oracle.CpuBaseline(threads)
    many = base.many(pats)
    t0 = time.perf_counter()
    want_counts, want_total, want_digest = many.digest_par(text)
    t_digest = time.perf_counter() - t0
    checks = [first_mismatch("counts", counts.astype(np.uint64), want_counts),
              None if total == want_total else f"total: {total} vs {want_total}"]
    got_digest = device_hit_digest(d_hits, total)
    checks.append(None if got_digest == want_digest else f"digest: {got_digest:#x} vs {want_digest:#x}")
    base_of = np.concatenate([[0], np.cumsum(want_counts.astype(np.int64))])
    order = np.argsort(-want_counts.astype(np.int64), kind="stable")
    rng = np.random.default_rng(7)
    sampled = [int(i) for i in order[:3]] + [int(i) for i in rng.choice(len(pats), 5, replace=False)]
    listed = 0
    for i in sampled:
        c = int(want_counts[i])
        want = np.empty(max(c, 1), np.uint32)
        n_found, _ = base.find_all_par(text, pats[i], want)
        got = d_hits[2 * int(base_of[i]): 2 * (int(base_of[i]) + c)].cpu().numpy().view(np.uint32).reshape(-1, 2)
        checks.append(None if n_found == c else f"pattern {i}: find_all_par {n_found} vs count {c}")
        checks.append(first_mismatch(f"hits of pattern {i} (pattern field)", got[:, 0], np.full(c, i, np.uint32)))
        checks.append(first_mismatch(f"hits of pattern {i} (offsets)", got[:, 1], want[:c]))
        listed += c
    bad = [c for c in checks if c]
    return {"result": "bit-exact" if not bad else "MISMATCH", "first_mismatch": bad[0] if bad else None,
            "compared": f"counts of all {len(pats)} patterns, the total ({total} hits) and a 64-bit order-checking "
                        f"digest of every (pattern, offset) hit in order; {listed} hits of {len(sampled)} patterns "
                        "element by element",
            "against": f"the CPU port's Aho-Corasick DFA ({many.states} states) and find_all_par on the same "
                       f"document ({threads} threads)",
            "cpu_check_s": round(t_digest, 2)}


def dictionary_record(args, world, rank, local, p=None) -> dict:
    """A synthetic oneline document (seed 2, 1 GiB) against 10,000 patterns of
    4..64 B: every (pattern id, offset) hit in (pattern, offset) order, left in
    HBM (value) or downloaded (e2e). Returns the record (all ranks take part in
    the collectives; the record is meaningful on rank 0)."""
    import torch

    from oneline_b200 import GpuParser, _lib, datagen

    L = _lib.load()
    seed = 2 + rank
    text = datagen.corpus(args.dict_bytes, seed)
    pats = datagen.patterns_dictionary(text, seed, n=10_000)
    N = text.size
    torch.cuda.set_device(local)
    p = p or GpuParser(local)
    host = torch.empty(N, dtype=torch.uint8, pin_memory=True)
    host.numpy()[:] = text
    doc = p.upload(host.numpy())
    ps = p.compile_patterns(doc, pats, max_patterns=None)
    counts, total = p.search_many_device(doc, ps, 0, 0)
    hits = torch.empty(2 * max(total, 1), dtype=torch.int32, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(L.ol_ctx_stream(p.ctx), device=f"cuda:{local}")

    def step():
        c, t = p.search_many_device(doc, ps, hits.data_ptr(), total)
        assert t == total
        return c

    if args.profile_launches:
        for _ in range(args.warmup + args.steps):
            step()
        p.sync()
        return {}
    for _ in range(args.warmup):
        step()
    p.sync()
    barrier(world)
    torch.cuda.synchronize()
    l0 = L.ol_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            ev0.record()
        for _ in range(args.steps):
            counts = step()
        with torch.cuda.stream(stream):
            ev1.record()
        ev1.synchronize()
    launches = L.ol_launch_count() - l0
    work = p.dict_stats()
    ms = allreduce_max(ev0.elapsed_time(ev1) / args.steps, world)
    bytes_all = allreduce_sum(float(N), world)
    value = bytes_all / (ms * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    alg = N + 8 * total  # text once + every ManyHit {pattern u32, offset u32} once
    achieved = alg / (ms * 1e-3) / 1e9

    def chk(s):
        if s != 0:
            raise RuntimeError(L.ol_last_error(p.ctx).decode())

    e2e = None
    if args.e2e_steps > 0:
        out_h = torch.empty(2 * max(total, 1), dtype=torch.int32, pin_memory=True)
        cnt_h = np.zeros(len(pats), np.uint32)
        tot_h = ctypes.c_uint64()

        def e2e_step():
            h = ctypes.c_void_p()
            chk(L.ol_doc_upload(p.ctx, host.data_ptr(), N, ctypes.byref(h)))
            chk(L.ol_search_many(p.ctx, h.value, ps.handle, total, cnt_h.ctypes.data, ctypes.byref(tot_h),
                                 out_h.data_ptr()))
            L.ol_doc_free(h.value)

        e2e_step()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        dt = allreduce_max((time.perf_counter() - t0) / args.e2e_steps, world)
        assert int(tot_h.value) == total
        del out_h
        e2e = {"value": round(bytes_all / dt / 1e9, 4), "unit": "GB/s", "ms_per_step": round(dt * 1e3, 2),
               "h2d_bytes_per_step": int(N), "d2h_bytes_per_step": int(8 * total + 4 * len(pats) + 8),
               "timing": "host wall clock around blocking C-ABI calls, max over ranks",
               "path": "ol_doc_upload (pinned text) + ol_search_many (counts and every hit to pinned host memory)"}

    cpu, parity = None, None
    if not args.no_cpu:
        import oracle

        if rank == 0:
            n = min(N, args.dict_cpu_sample_mb << 20)
            sample = np.ascontiguousarray(text[:n])
            many = oracle.CpuBaseline().many(pats)
            ts = []
            for _ in range(2):
                t0 = time.perf_counter()
                many.find_all_par(sample)
                ts.append(time.perf_counter() - t0)
            t = ts[-1]
            cpu = {"value": round(n / t / 1e9, 4), "unit": "GB/s", "cores": many.threads, "kind": "port",
                   "sample": f"first {n} bytes of the same document x the same 10,000 patterns: Aho-Corasick DFA "
                             "(byte classes), every hit, ordered by (pattern, offset); the second of 2 runs (the "
                             "whole 1 GiB would hold 30 GB of hits in host memory)",
                   "dfa_states": int(many.states)}
            del many
        barrier(world)
        parity = parity_dictionary(text, pats, counts, total, hits, max(1, (os.cpu_count() or 1) // world))
        bad = allreduce_sum(0.0 if parity["result"] == "bit-exact" else 1.0, world)
        if world > 1:
            parity["ranks_checked"] = world
            parity["ranks_mismatched"] = int(bad)

    return {"metric": "dictionary search GB/s vs HBM peak", "value": round(value, 3), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {"workload": f"{N}-byte synthetic oneline document (seed {seed}) x 10,000-pattern "
                                   f"dictionary (4..64 B, 60% sampled from the text): every (pattern, offset)",
                       "text_bytes": int(N), "patterns": len(pats), "unique_patterns": ps.unique(),
                       "total_hits": int(total), "hit_bytes": int(8 * total),
                       "walked_per_byte": round(work["walked"] / N, 4),
                       "nodes_per_walk": round(work["nodes"] / max(work["walked"], 1), 2),
                       "bitmap_patterns": work["heavy_patterns"], "sorted_key_hits": work["light_hits"],
                       "l2": "inputs and outputs larger than L2 (no flush needed)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": "dictionary pass (match, rank, sort, emit)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind, "traffic": None,
                         "alg_bytes_per_launch": int(alg), "ms_per_launch": round(ms, 3)},
            "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks.summary(), "device": p.adapter_name()}


def run_dictionary(args, world, rank, local):
    rec = dictionary_record(args, world, rank, local)
    if rank == 0 and rec:
        print(json.dumps(rec), flush=True)


# ----------------------------------------------------------------- batch

def batch_record(args, world, rank, local, p=None) -> dict:
    """10,000 documents (seeds 3..10002, log-normal sizes, median 16 KiB, sigma 1.5,
    256 B..64 MiB): full parse, tree links and a 1,000-pattern dictionary search of
    every document, batched (one upload, one parse, one tree build, one search) vs
    one call per document, both end to end from host memory."""
    import torch

    from oneline_b200 import GpuParser, _lib, datagen

    L = _lib.load()
    n_docs = 10_000
    sizes = datagen.lognormal_sizes(3, n_docs, 16384.0, 1.5, 256, 64 << 20)
    docs = [datagen.corpus(int(sz), 3 + i) for i, sz in enumerate(sizes)]
    offs = np.zeros(n_docs + 1, np.uint64)
    offs[1:] = np.cumsum(sizes)
    data_np = np.concatenate(docs)
    total_bytes = int(offs[-1])
    dict_text = datagen.corpus(1 << 30, 2)
    pats = datagen.patterns_dictionary(dict_text, 2, n=10_000)[:1000]
    del dict_text
    torch.cuda.set_device(local)
    p = p or GpuParser(local)
    data = torch.empty(total_bytes, dtype=torch.uint8, pin_memory=True)
    data.numpy()[:] = data_np
    ps = p.compile_patterns(None, pats)
    cnt = np.zeros(len(pats), np.uint32)
    tot = ctypes.c_uint64()

    def chk(s):
        if s != 0:
            raise RuntimeError(L.ol_last_error(p.ctx).decode())

    # output room: the hits of the batched pass (same total as the per-document calls)
    b0 = p.upload_batch((data.numpy(), offs))
    _, total = p.batch_search_many(b0, ps, 0, 0)
    b0.free()
    hits = torch.empty(2 * max(total, 1), dtype=torch.int32, device=f"cuda:{local}")

    def batched():
        h = ctypes.c_void_p()
        chk(L.ol_batch_upload(p.ctx, data.data_ptr(), offs.ctypes.data, n_docs, ctypes.byref(h)))
        chk(L.ol_batch_build_trees(p.ctx, h.value))
        chk(L.ol_batch_search_many(p.ctx, h.value, ps.handle, total, 0, cnt.ctypes.data, ctypes.byref(tot),
                                   hits.data_ptr()))
        L.ol_batch_free(h.value)
        return int(tot.value)

    def plain():
        got = 0
        base = data.data_ptr()
        for i in range(n_docs):
            h = ctypes.c_void_p()
            t = ctypes.c_void_p()
            chk(L.ol_doc_upload(p.ctx, base + int(offs[i]), int(sizes[i]), ctypes.byref(h)))
            chk(L.ol_tree_build(p.ctx, h.value, 0, ctypes.byref(t)))
            chk(L.ol_search_many_device(p.ctx, h.value, ps.handle, total - got, 0, cnt.ctypes.data, ctypes.byref(tot),
                                        hits.data_ptr() + 8 * got))
            got += int(tot.value)
            L.ol_tree_free(t.value)
            L.ol_doc_free(h.value)
        return got

    for _ in range(args.warmup):
        batched()
    p.sync()
    barrier(world)
    l0 = L.ol_launch_count()
    step_ms = []
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ts = time.perf_counter()
            got = batched()
            step_ms.append((time.perf_counter() - ts) * 1e3)
        p.sync()
        dt = (time.perf_counter() - t0) / args.steps
    launches = L.ol_launch_count() - l0
    assert got == total
    dt = allreduce_max(dt, world)
    # where one batched step's time goes: CUDA-event passes, and each call's
    # host wall time
    _, prof = p._profiled(batched)
    passes = {}
    for label, sec in prof.gpu_passes:
        passes[label] = round(passes.get(label, 0.0) + sec * 1e3, 3)
    host_steps = [(label, round(sec * 1e3, 3)) for label, sec in prof.host_steps]
    calls = {}
    h = ctypes.c_void_p()
    t_0 = time.perf_counter()
    chk(L.ol_batch_upload(p.ctx, data.data_ptr(), offs.ctypes.data, n_docs, ctypes.byref(h)))
    t_1 = time.perf_counter()
    chk(L.ol_batch_build_trees(p.ctx, h.value))
    t_2 = time.perf_counter()
    chk(L.ol_batch_search_many(p.ctx, h.value, ps.handle, total, 0, cnt.ctypes.data, ctypes.byref(tot), hits.data_ptr()))
    t_3 = time.perf_counter()
    L.ol_batch_free(h.value)
    p.sync()
    t_4 = time.perf_counter()
    calls = {"ol_batch_upload": round((t_1 - t_0) * 1e3, 2), "ol_batch_build_trees": round((t_2 - t_1) * 1e3, 2),
             "ol_batch_search_many": round((t_3 - t_2) * 1e3, 2), "ol_batch_free": round((t_4 - t_3) * 1e3, 2)}
    t0 = time.perf_counter()
    got_plain = plain()
    p.sync()
    dt_plain = allreduce_max(time.perf_counter() - t0, world)
    assert got_plain == total, (got_plain, total)
    bytes_all = allreduce_sum(float(total_bytes), world)
    value = bytes_all / dt / 1e9
    line = {}
    if rank == 0:
        plain_v = bytes_all / dt_plain / 1e9
        line = {"metric": "batched parse+dictionary GB/s vs one call per document", "value": round(value, 3),
                "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u8", "data": "synthetic",
                "config": {"workload": f"{n_docs} documents (seeds 3..{2 + n_docs}, log-normal sizes median 16 KiB, "
                                       f"sigma 1.5, 256 B..64 MiB, {total_bytes} bytes): parse + tree links + "
                                       f"1,000-pattern dictionary search of every document",
                           "docs": n_docs, "text_bytes": total_bytes, "patterns": len(pats), "total_hits": int(total),
                           "l2": "inputs larger than L2", "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "plain": {"value": round(plain_v, 4), "unit": "GB/s", "ms_per_step": round(dt_plain * 1e3, 1),
                          "path": "per document: ol_doc_upload + ol_tree_build + ol_search_many_device"},
                "speedup_vs_plain": round(value / plain_v, 2),
                "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": total_bytes,
                        "d2h_bytes_per_step": 4 * len(pats) + 8,
                        "timing": "host wall clock around the blocking batch calls (the value itself)",
                        "path": "ol_batch_upload (pinned) + ol_batch_build_trees + ol_batch_search_many (hits in HBM)"},
                "gpu_launches": int(launches), "launches_per_step": round(launches / max(args.steps, 1), 1),
                "step_ms": {"min": round(min(step_ms), 2), "median": round(statistics.median(step_ms), 2),
                            "max": round(max(step_ms), 2)},
                "passes_ms": passes, "host_steps_ms": host_steps, "calls_ms": calls, "clocks": clocks.summary(),
                "device": p.adapter_name()}
    return line


def run_batch(args, world, rank, local):
    line = batch_record(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- serve

def serve_stream(seconds: float, seed: int = 4, rate: float = 2000.0):
    """The request stream: Poisson arrivals at 2,000 req/s; 30% parse requests
    (log-normal sizes, median 64 KiB, sigma 2, 1 KiB..64 MiB, cut from a seeded
    corpus), 70% searches of 1..64 patterns (4..64 B) against resident documents."""
    from oneline_b200 import datagen

    n = int(rate * seconds)
    t = datagen.poisson_arrivals(seed, n, rate)
    rng = datagen.Rng(seed)
    is_parse = np.array([rng.below(100) < 30 for _ in range(n)])
    sizes = datagen.lognormal_sizes(seed, n, 65536.0, 2.0, 1024, 64 << 20)
    base = datagen.corpus(256 << 20, seed)
    pool = datagen.patterns_dictionary(base[: 64 << 20], seed, n=20_000)
    reqs = []
    for i in range(n):
        if is_parse[i]:
            size = int(sizes[i])
            at = rng.below(base.size - size) if base.size > size else 0
            reqs.append(("parse", float(t[i]), base[at: at + size]))
        else:
            k = 1 + rng.below(64)
            first = rng.below(len(pool) - k)
            reqs.append(("search", float(t[i]), pool[first: first + k], rng.below(1 << 30)))
    return reqs, base


SERVE_MAX_HITS = 1 << 18  # hits a search request gets back


def serve_room(nbytes: int) -> int:
    """Lines of room the client gives a parse of `nbytes` bytes: a power of two
    at least nbytes / 8 + 4096 (the serve corpus has fewer lines)."""
    return 1 << max(12, (int(nbytes) // 8 + 4096 - 1).bit_length())


def serve_parse_set(room: int) -> dict:
    from oneline_b200.serving import LINK_NAMES

    out = {"offsets": np.zeros(room, np.uint32), "kinds": np.zeros(room, np.uint8),
           **{k: np.zeros(room, np.uint32) for k in LINK_NAMES}}
    for a in out.values():
        a.fill(0)  # touch every page now, not in a worker's copy during the stream
    return out


def serve_search_set() -> dict:
    from oneline_b200 import HIT_DTYPE

    out = {"counts": np.zeros(64, np.uint32), "hits": np.zeros(SERVE_MAX_HITS, HIT_DTYPE)}
    out["hits"].view(np.uint8).fill(0)
    return out


def serve_buffer_pool(*streams) -> dict:
    """The result buffers a serving client keeps and reuses, made and touched
    before any timed stream: per parse room (serve_room) as many sets as the
    streams have parses of that room, at most 64 (rooms up to 2^16 lines), 16
    (up to 2^20) or 4 (larger), and 128 search sets. A stream that needs more
    at once makes them as it goes."""
    from collections import Counter

    need = Counter(serve_room(r[2].size) for reqs in streams for r in reqs if r[0] == "parse")
    pool = {"search": [serve_search_set() for _ in range(128)]}
    for room, n in sorted(need.items()):
        keep = 64 if room <= 1 << 16 else 16 if room <= 1 << 20 else 4
        pool[room] = [serve_parse_set(room) for _ in range(min(n, keep))]
    return pool


def serve_run(reqs, workers: int, warm_docs, coalesce: bool, pool: dict, warm_stream=()):
    """Plays the stream open-loop against a server; returns per-request latencies
    and the bytes processed. Every request gets its results back in host arrays
    (a parse: offsets, kinds and the four tree arrays; a search: counts and up
    to SERVE_MAX_HITS hits), so the latency covers the download. The arrays
    come from `pool` (serve_buffer_pool) and go back to it once the result has
    been collected, as a serving client that reuses its buffers does."""
    import threading

    from oneline_b200 import _lib
    from oneline_b200.serving import GpuServer

    L = _lib.load()
    free_bufs = pool

    with GpuServer(workers=workers, store_budget=4 << 30, max_hits=SERVE_MAX_HITS, coalesce=coalesce) as srv:
        # warm-up outside the timed stream: resident documents to search, and
        # every kernel launched once (the first launch of a kernel loads it)
        ready = [srv.wait(r).doc_id for r in [srv.submit_parse(d) for d in warm_docs]]
        sizes = {d: int(len(w)) for d, w in zip(ready, warm_docs)}
        for r in [srv.submit_search(d, [b"||||", b"| @", b"abcd"][: 1 + d % 3]) for d in ready]:
            srv.wait(r)
        lock = threading.Lock()

        def play(stream):
            """Submits `stream` open-loop (each request at its arrival time) and
            collects every result; returns them and the wall time."""
            pending = []  # (request id, kind, text bytes of a parse, buffer pool key, buffers)
            done = threading.Event()
            results = []

            def collect():
                i = 0
                while True:
                    with lock:
                        item = pending[i] if i < len(pending) else None
                    if item is None:
                        if done.is_set():
                            with lock:
                                if i >= len(pending):
                                    return
                        time.sleep(0.0002)
                        continue
                    rid, kind, nbytes, key, bufs = item
                    r = srv.wait(rid)
                    srv.results(rid, r)  # the arrays are in host memory; the buffers go back to the pool
                    with lock:
                        free_bufs.setdefault(key, []).append(bufs)
                    if kind == "parse" and r.status == 0:
                        with lock:
                            ready.append(r.doc_id)
                            sizes[r.doc_id] = nbytes
                    results.append((kind, r.status, r.latency_ns, nbytes if kind == "parse" else sizes.get(r.doc_id, 0),
                                    r.start_ns, r.end_ns, r.submit_ns))
                    i += 1

            col = threading.Thread(target=collect)
            col.start()
            t0 = time.perf_counter()
            for req in stream:
                delay = t0 + req[1] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                if req[0] == "parse":
                    room = serve_room(req[2].size)
                    with lock:
                        lst = free_bufs.get(room)
                        bufs = lst.pop() if lst else None
                    if bufs is None:
                        bufs = serve_parse_set(room)
                    rid = srv.submit_parse(req[2], out=bufs)
                    with lock:
                        pending.append((rid, "parse", int(req[2].size), room, bufs))
                else:
                    with lock:
                        doc = ready[req[3] % len(ready)]
                    with lock:
                        lst = free_bufs.get("search")
                        bufs = lst.pop() if lst else None
                    if bufs is None:
                        bufs = serve_search_set()
                    rid = srv.submit_search(doc, req[2], out=bufs)
                    with lock:
                        pending.append((rid, "search", 0, "search", bufs))
            done.set()
            col.join()
            wall = time.perf_counter() - t0
            return results, wall

        if warm_stream:
            play(warm_stream)  # not timed: the server and the client settle first
        s0, l0 = srv.steps(), L.ol_launch_count()
        results, wall = play(reqs)
        s1, l1 = srv.steps(), L.ol_launch_count()
        stats = {**srv.stats(), "steps": s1["steps"] - s0["steps"], "requests": s1["requests"] - s0["requests"],
                 "largest_step": s1["largest_step"], "launches": l1 - l0}
    return results, wall, stats


def serve_timeline(ok, windows: int = 6) -> list:
    """Latency over the stream: per window of submit time, the requests, their
    p99 latency, the longest service (ms) and the kind and bytes of that request."""
    t0 = min(r[6] for r in ok)
    span = max(r[6] for r in ok) - t0 + 1
    out = []
    for w in range(windows):
        sel = [r for r in ok if (r[6] - t0) * windows // span == w]
        if not sel:
            continue
        lat = np.array([r[2] for r in sel], np.float64) / 1e6
        slow = max(sel, key=lambda r: r[5] - r[4])
        out.append({"from_s": round(w * span / windows / 1e9, 1), "requests": len(sel),
                    "p99_ms": round(float(np.percentile(lat, 99)), 3),
                    "max_service_ms": round((slow[5] - slow[4]) / 1e6, 3), "slowest": [slow[0], int(slow[3])]})
    return out


def serve_record(args, local) -> dict:
    """The serving workload: the same open-loop stream against the served form
    (`serve_workers` workers, continuous batching) and the plain form (one
    worker, one request per step: every request its own launches)."""
    import gc

    from oneline_b200 import GpuParser, _lib

    L = _lib.load()
    reqs, base = serve_stream(args.serve_seconds, rate=args.serve_rate)
    warm = [base[i << 20: (i << 20) + (64 << 10)] for i in range(64)]
    oreqs = serve_stream(args.serve_overload_seconds, seed=5, rate=args.serve_overload_rate)[0] \
        if args.serve_overload_rate > 0 else []
    # every form first serves 8 s of the same traffic (another seed), not timed
    wreqs = serve_stream(8.0, seed=6, rate=args.serve_rate)[0]
    gc.collect()  # the earlier workloads' garbage goes now, not during a timed stream
    pool = serve_buffer_pool(reqs, oreqs, wreqs)
    out = {}
    for name, workers, coalesce in (("served", args.serve_workers, True), ("plain", 1, False)):
        with ClockSampler(local) as clocks:
            res, wall, stats = serve_run(reqs, workers, warm, coalesce, pool, wreqs)
        launches = stats.pop("launches")
        ok = [r for r in res if r[1] == 0]
        lat = np.array([r[2] for r in ok], np.float64) / 1e6
        wait = np.array([r[4] - r[6] for r in ok], np.float64) / 1e6  # queued before a worker took it
        svc = np.array([r[5] - r[4] for r in ok], np.float64) / 1e6
        by_kind = {k: np.array([r[2] for r in ok if r[0] == k], np.float64) / 1e6 for k in ("parse", "search")}
        span = (max(r[5] for r in ok) - min(r[6] for r in ok)) / 1e9
        nbytes = sum(r[3] for r in ok)
        out[name] = {"workers": workers, "coalesce": coalesce, "requests": len(res), "ok": len(ok),
                     "gpu_launches": int(launches), "launches_per_request": round(launches / max(len(res), 1), 2),
                     "refused": sum(1 for r in res if r[1] == 6), "not_found": sum(1 for r in res if r[1] == 9),
                     "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                     "queue_p99_ms": round(float(np.percentile(wait, 99)), 3),
                     "p99_ms_second_half": round(float(np.percentile(lat[len(lat) // 2:], 99)), 3),
                     "service_p99_ms": round(float(np.percentile(svc, 99)), 3),
                     "p99_ms_by_kind": {k: round(float(np.percentile(v, 99)), 3) for k, v in by_kind.items() if v.size},
                     "req_per_s": round(len(ok) / wall, 1), "gb_per_s": round(nbytes / span / 1e9, 3),
                     "wall_s": round(wall, 2), "store": stats, "clocks": clocks.summary(),
                     "timeline": serve_timeline(ok)}
    sv, pl = out["served"], out["plain"]
    # the same mix offered faster than one request per step can serve
    overload = {}
    if args.serve_overload_rate > 0:
        for name, workers, coalesce in (("served", args.serve_workers, True), ("plain", 1, False)):
            res, wall, stats = serve_run(oreqs, workers, warm, coalesce, pool, wreqs)
            ok = [r for r in res if r[1] == 0]
            lat = np.array([r[2] for r in ok], np.float64) / 1e6
            overload[name] = {"req_per_s": round(len(ok) / wall, 1), "ok": len(ok), "requests": len(res),
                              "p50_ms": round(float(np.percentile(lat, 50)), 3),
                              "p99_ms": round(float(np.percentile(lat, 99)), 3),
                              "largest_step": stats.get("largest_step"), "steps": stats.get("steps")}
        overload["offered_req_per_s"] = args.serve_overload_rate
        overload["seconds"] = args.serve_overload_seconds
    return {"metric": "served req/s at p99 vs per-request launches", "value": sv["req_per_s"], "unit": "req/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": round(sv["wall_s"] * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"open-loop Poisson stream, {args.serve_rate:g} req/s for {args.serve_seconds} s: 30% parse "
                                   "(log-normal 64 KiB median, sigma 2, 1 KiB..64 MiB), 70% search (1..64 patterns "
                                   "of 4..64 B) against resident documents; 4 GiB store with HBM-budget admission",
                       "requests": len(reqs), "parallelism": "single GPU",
                       "warmup": "every form first serves 8 s of the same traffic (seed 6), not timed"},
            "served": sv, "plain": pl, "overload": overload,
            "p99_speedup_vs_plain": round(pl["p99_ms"] / max(sv["p99_ms"], 1e-9), 2),
            "gbps_vs_plain": round(sv["gb_per_s"] / max(pl["gb_per_s"], 1e-9), 2),
            "results": "every request's arrays downloaded to host memory, into result buffers the client reuses, "
                       "before it completes",
            "device": GpuParser(local).adapter_name()}


def run_serve(args, world, rank, local):
    if rank != 0:
        return
    print(json.dumps(serve_record(args, local)), flush=True)


def main():
    args = parse_args()
    ClockSampler.log_path = args.clock_log
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "dictionary":
            run_dictionary(args, world, rank, local)
        elif args.workload == "batch":
            run_batch(args, world, rank, local)
        elif args.workload == "serve":
            run_serve(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
