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
  cpu_baseline: the multi-threaded C++ port of the reference's CPU engine on a
            bounded sample of the same document.

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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "parse+search GB/s vs HBM peak"


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bytes", type=int, default=1 << 30, help="document size (default 1 GiB)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-mb", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-launches", action="store_true",
                    help="one short run for an ncu launch list (no e2e, no CPU leg)")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
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
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
            sm = [float(r[1]) for r in rows]
            mx = float(rows[0][2]) if rows else None
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                    "samples": len(rows)}
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


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------ workload

def make_workload(nbytes: int, seed: int):
    from oneline_b200 import datagen

    text = datagen.corpus(nbytes, seed)
    pats = datagen.patterns_eight(text, seed)
    return text, pats


def cpu_leg(text: np.ndarray, pats, sample_mb: int, reps: int = 2) -> dict:
    """The reference CPU path (port) on all host cores over a bounded prefix."""
    import oracle

    n = min(text.size, sample_mb << 20)
    sample = text[:n]
    # cut at a line boundary so the sample is a document of its own
    cut = int(np.nonzero(sample == 10)[0][-1]) + 1
    sample = np.ascontiguousarray(sample[:cut])
    base = oracle.CpuBaseline()
    times = []
    for _ in range(reps + 1):
        t0 = time.perf_counter()
        offs, nodes = base.parse_par(sample)
        base.build_links(nodes)
        for p in pats:
            base.find_all_par(sample, p)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times[1:])
    return {"value": round(sample.size / t / 1e9, 4), "unit": "GB/s", "cores": base.threads, "kind": "port",
            "sample": f"first {sample.size} bytes of the same document (line-aligned): parse_par + build_links + "
                      f"children + {len(pats)} x find_all_par, median of {reps} after 1 warm-up "
                      "(C++ port of oneline-simd; the Rust reference cannot be built here)",
            "seconds_per_rep": round(t, 4)}


def run_reference(args, world, rank):
    if rank != 0:
        return
    text, pats = make_workload(args.bytes, args.seed)
    import oracle

    n = min(text.size, args.cpu_sample_mb << 20)
    cut = int(np.nonzero(text[:n] == 10)[0][-1]) + 1
    sample = np.ascontiguousarray(text[:cut])
    base = oracle.CpuBaseline()

    def step():
        offs, nodes = base.parse_par(sample)
        base.build_links(nodes)
        for p in pats:
            base.find_all_par(sample, p)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    v = sample.size / dt / 1e9
    line = {"metric": METRIC, "value": round(v, 4), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(args, sample.size, pats, None),
            "cpu_baseline": {"value": round(v, 4), "unit": "GB/s", "cores": base.threads, "kind": "port",
                             "sample": f"first {sample.size} bytes of the {args.bytes}-byte document per step "
                                       "(C++ port of oneline-simd on all host threads)"},
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
    text, pats = make_workload(args.bytes, args.seed + rank)
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

    # parse: count, scan, tiles, fix-up; tree: summary, scan, resolve; search: count, scan, write per 8 patterns
    launches_per_step = 4 + 3 + 3 * ((n_p + 7) // 8)
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

    # Timed region.
    for _ in range(args.warmup):
        step()
    p.sync()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            ev0.record()
        for _ in range(args.steps):
            step()
        with torch.cuda.stream(stream):
            ev1.record()
        ev1.synchronize()
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
    groups = {"parse_tiles_kernel": (t_parse, N + 6 * lines),
              "tree_forward+backward": (t_tree, 2 * lines + 5 * lines + 3 * lines + 16 * lines),
              "search_kernel<8>": (t_search, N + 4 * hits)}
    dom = max(groups, key=lambda k: groups[k][0])
    launches = 1
    t_launch = groups[dom][0] / launches
    alg = groups[dom][1] / launches
    achieved = alg / (t_launch * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind, "traffic": None,
                "alg_bytes_per_launch": int(alg), "ms_per_launch": round(t_launch, 4),
                "ms_parse": round(t_parse, 4), "ms_tree": round(t_tree, 4),
                "ms_search": round(t_search, 4)}

    # End to end through the C ABI with host buffers.
    e2e = None
    if args.e2e_steps > 0:
        from oneline_b200 import NODE_DTYPE  # noqa: F401

        offs_h = torch.empty(lines, dtype=torch.int32, pin_memory=True).numpy()
        kinds_h = torch.empty(lines, dtype=torch.uint8, pin_memory=True).numpy()
        tree_h = [torch.empty(lines, dtype=torch.int32, pin_memory=True).numpy() for _ in range(4)]
        hits_h = [torch.empty(max(t, 1), dtype=torch.int32, pin_memory=True).numpy() for t in totals]

        tots_h = np.zeros(n_p, np.uint32)
        OH = (ctypes.c_void_p * n_p)(*[a.ctypes.data for a in hits_h])

        def e2e_step():
            h = ctypes.c_void_p()
            chk(L.ol_doc_upload(p.ctx, host.data_ptr(), N, ctypes.byref(h)))
            t = ctypes.c_void_p()
            chk(L.ol_tree_build(p.ctx, h.value, 1, ctypes.byref(t)))
            chk(L.ol_search_multi(p.ctx, h.value, P, lens.ctypes.data, n_p, maxes.ctypes.data,
                                  tots_h.ctypes.data, OH))
            chk(L.ol_doc_read_offsets(p.ctx, h.value, offs_h.ctypes.data, lines))
            chk(L.ol_doc_read_kinds(p.ctx, h.value, kinds_h.ctypes.data, lines))
            chk(L.ol_tree_read(p.ctx, t.value, *[a.ctypes.data for a in tree_h], lines))
            L.ol_tree_free(t.value)
            L.ol_doc_free(h.value)

        e2e_step()
        p.sync()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        p.sync()
        dt = (time.perf_counter() - t0) / args.e2e_steps
        dt = allreduce_max(dt, world)
        e2e = {"value": round(bytes_all / dt / 1e9, 4), "unit": "GB/s", "ms_per_step": round(dt * 1e3, 3),
               "h2d_bytes_per_step": int(N), "d2h_bytes_per_step": int(21 * lines + 4 * hits),
               "timing": "host wall clock around blocking C-ABI calls, max over ranks",
               "path": "ol_doc_upload (pinned) + ol_tree_build + ol_search_multi (8 patterns) + ol_doc_read_offsets/kinds + "
                       "ol_tree_read (4 arrays)"}

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_leg(text, pats, args.cpu_sample_mb)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                "config": {**workload_config(args, N, pats, lines), "hits": totals},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches_per_step * args.steps, "clocks": clocks.summary(),
                "device": p.adapter_name()}
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
