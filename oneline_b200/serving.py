"""GpuServer: the serving loop of the CUDA library (ol_server_* in
include/oneline_cuda.h), for parse and search requests of mixed sizes.

Worker threads in the library each own a context and a stream. A worker that
frees up takes every queued request and serves them as one step (continuous
batching): parse requests are admitted against the HBM budget before any
upload, then parsed and linked as one batch; searches of the same document
share one dictionary pass. Steps of different workers overlap on the device.
Parsed documents stay resident in the budgeted store and are searched without
uploading their text again. Results are downloaded into the caller's arrays
before a request completes. No reference counterpart: the reference offers one
blocking call per document (crates/oneline-gpu/src/parser.rs).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import OnelineError

KIND_PARSE, KIND_SEARCH = 0, 1


class RequestResult(ctypes.Structure):
    """ol_request_result: one finished request."""

    _fields_ = [("id", ctypes.c_uint64), ("kind", ctypes.c_uint32), ("status", ctypes.c_int32),
                ("worker", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("doc_id", ctypes.c_uint64),
                ("line_count", ctypes.c_uint64), ("total_hits", ctypes.c_uint64), ("digest", ctypes.c_uint64),
                ("submit_ns", ctypes.c_uint64), ("start_ns", ctypes.c_uint64), ("end_ns", ctypes.c_uint64)]

    @property
    def latency_ns(self) -> int:
        return int(self.end_ns - self.submit_ns)


class ParseDest(ctypes.Structure):
    """ol_parse_dest."""

    _fields_ = [("cap", ctypes.c_uint64), ("offsets", ctypes.c_void_p), ("kinds", ctypes.c_void_p),
                ("parent", ctypes.c_void_p), ("subtree_end", ctypes.c_void_p), ("first_child", ctypes.c_void_p),
                ("next_sibling", ctypes.c_void_p)]


class SearchDest(ctypes.Structure):
    """ol_search_dest."""

    _fields_ = [("max_hits", ctypes.c_uint64), ("counts", ctypes.c_void_p), ("hits", ctypes.c_void_p)]


NO_COALESCE = 1  # OL_SERVER_NO_COALESCE
HIT_DTYPE = np.dtype([("pattern", "<u4"), ("offset", "<u4")])
LINK_NAMES = ("parent", "subtree_end", "first_child", "next_sibling")


class GpuServer:
    """The serving loop. ``coalesce=False`` serves one request per step (the
    plain per-request form)."""

    def __init__(self, device: int = 0, workers: int = 8, store_budget: int = 4 << 30, max_hits: int = 1 << 22,
                 coalesce: bool = True):
        h = ctypes.c_void_p()
        st = _lib.load().ol_server_create_ex(device, workers, store_budget, max_hits, 0 if coalesce else NO_COALESCE,
                                             ctypes.byref(h))
        if st != 0:
            raise OnelineError(st, "could not start the server")
        self._h = h.value
        self.max_hits = max_hits
        self._keep = {}  # request id -> buffers that must outlive the request
        self._out = {}   # request id -> result arrays

    def submit_parse(self, text, *, results: bool = False, cap: int | None = None, out: dict | None = None) -> int:
        """Queues a parse. With ``results``, the document's offsets, kinds and four
        tree arrays come back with the result (``cap`` lines of room; default: one
        line per byte, always enough). ``out`` (implies ``results``): arrays to
        write them into instead of new ones, as ``results`` returns them (u32
        offsets and links, u8 kinds, all of one length, the room), so a client can
        reuse its buffers; they must not be touched until the request is waited on."""
        buf = np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray)) else np.ascontiguousarray(text, np.uint8)
        rid = ctypes.c_uint64()
        dest = None
        if out is not None:
            n = int(out["offsets"].size)
            for k, dt in (("offsets", np.uint32), ("kinds", np.uint8)) + tuple((k, np.uint32) for k in LINK_NAMES):
                a = out[k]
                if a.dtype != dt or a.size < n or not a.flags.c_contiguous:
                    raise ValueError(f"out[{k!r}] must be a contiguous {np.dtype(dt).name} array of at least {n} entries")
        elif results:
            n = int(cap if cap is not None else buf.size + 1)
            out = {"offsets": np.zeros(max(n, 1), np.uint32), "kinds": np.zeros(max(n, 1), np.uint8)}
            for k in LINK_NAMES:
                out[k] = np.zeros(max(n, 1), np.uint32)
        if out is not None:
            dest = ParseDest(n, *[out[k].ctypes.data for k in ("offsets", "kinds") + LINK_NAMES])
        st = _lib.load().ol_server_submit_parse_to(self._h, buf.ctypes.data, buf.size,
                                                   ctypes.byref(dest) if dest is not None else None,
                                                   ctypes.byref(rid))
        if st != 0:
            raise OnelineError(st, "submit_parse")
        self._keep[rid.value] = (buf, dest)
        if out is not None:
            self._out[rid.value] = out
        return rid.value

    def submit_search(self, doc_id: int, patterns, *, results: bool = False, max_hits: int | None = None,
                      out: dict | None = None) -> int:
        """Queues a search of a resident document. With ``results``, the counts
        and the first ``max_hits`` hits (pattern = index in ``patterns``) come back.
        ``out`` (implies ``results``): {"counts": u32 array with room for every
        pattern, "hits": HIT_DTYPE array} to write them into, for a client that
        reuses its buffers (the hits array's size is the room)."""
        pats = [bytes(p) for p in patterns]
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        P = (ctypes.c_void_p * len(pats))(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats], np.uint32)
        rid = ctypes.c_uint64()
        dest = None
        if out is not None:
            out = dict(out)
            if (out["counts"].dtype != np.uint32 or out["counts"].size < len(pats) or out["hits"].dtype != HIT_DTYPE
                    or not out["counts"].flags.c_contiguous or not out["hits"].flags.c_contiguous):
                raise ValueError("out needs a contiguous u32 'counts' array with room for every pattern and a "
                                 "contiguous HIT_DTYPE 'hits' array")
            dest = SearchDest(int(out["hits"].size), out["counts"].ctypes.data, out["hits"].ctypes.data)
        elif results:
            mh = int(max_hits if max_hits is not None else self.max_hits)
            out = {"counts": np.zeros(max(len(pats), 1), np.uint32), "hits": np.zeros(max(mh, 1), HIT_DTYPE)}
            dest = SearchDest(mh, out["counts"].ctypes.data, out["hits"].ctypes.data)
        st = _lib.load().ol_server_submit_search_to(self._h, int(doc_id), P, lens.ctypes.data, len(pats),
                                                    ctypes.byref(dest) if dest is not None else None,
                                                    ctypes.byref(rid))
        if st != 0:
            raise OnelineError(st, "submit_search")
        self._keep[rid.value] = dest  # the patterns are copied at submission
        if out is not None:
            out["n_patterns"] = len(pats)
            self._out[rid.value] = out
        return rid.value

    def wait(self, request_id: int) -> RequestResult:
        r = RequestResult()
        st = _lib.load().ol_server_wait(self._h, request_id, ctypes.byref(r))
        if st != 0:
            raise OnelineError(st, "wait")
        self._keep.pop(request_id, None)
        return r

    def results(self, request_id: int, result: RequestResult) -> dict | None:
        """The arrays of a finished request submitted with ``results=True``, cut to
        their lengths (None when it failed or its arrays had no room)."""
        out = self._out.pop(request_id, None)
        if out is None or result.status != 0:
            return None
        if result.kind == KIND_PARSE:
            L = int(result.line_count)
            if L > out["offsets"].size:
                return None
            return {k: v[:L] for k, v in out.items()}
        k = min(int(result.total_hits), out["hits"].size)
        return {"counts": out["counts"][: out["n_patterns"]], "hits": out["hits"][:k]}

    def stats(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(4)]
        _lib.load().ol_server_stats(self._h, *[ctypes.byref(x) for x in v])
        return dict(zip(("resident_docs", "resident_bytes", "evictions", "refusals"), (int(x.value) for x in v)))

    def pause(self, paused: bool = True) -> None:
        """Workers take no new request while paused (requests still queue)."""
        _lib.load().ol_server_pause(self._h, 1 if paused else 0)

    def steps(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(3)]
        _lib.load().ol_server_steps(self._h, *[ctypes.byref(x) for x in v])
        return dict(zip(("steps", "requests", "largest_step"), (int(x.value) for x in v)))

    def close(self) -> None:
        if self._h:
            _lib.load().ol_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_K = np.uint64(0x9E3779B97F4A7C15)


def _mix64(x: np.ndarray) -> np.ndarray:
    x = x ^ (x >> np.uint64(30))
    x = x * np.uint64(0xBF58476D1CE4E5B9)
    x = x ^ (x >> np.uint64(27))
    x = x * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def array_digest(a: np.ndarray, seed: int) -> int:
    """The server's device digest of one array, computed on the host: the sum
    (mod 2^64) of splitmix64(seed << 56 ^ i << 24 ^ a[i] * 0x9E3779B97F4A7C15)."""
    with np.errstate(over="ignore"):
        i = np.arange(a.size, dtype=np.uint64)
        v = a.astype(np.uint64) * _K
        h = _mix64((np.uint64(seed) << np.uint64(56)) ^ (i << np.uint64(24)) ^ v)
        return int(h.sum(dtype=np.uint64))


def parse_digest(offsets, kinds, parent, subtree_end, first_child, next_sibling) -> int:
    """Digest of a parse request's outputs (what ol_request_result.digest holds)."""
    total = 0
    for seed, a in enumerate((offsets, kinds, parent, subtree_end, first_child, next_sibling), start=1):
        total = (total + array_digest(np.asarray(a), seed)) & 0xFFFFFFFFFFFFFFFF
    return total ^ ((len(offsets) * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF)


def search_digest(counts, hit_patterns, hit_offsets, total: int) -> int:
    """Digest of a search request's outputs: the hits (pattern, offset) as u32
    pairs, then the per-pattern counts folded in on the host, then the total."""
    pairs = np.empty(2 * len(hit_patterns), np.uint32)
    pairs[0::2] = hit_patterns
    pairs[1::2] = hit_offsets
    h = array_digest(pairs, 7)
    for c in counts:
        h = ((h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF) ^ int(c)
    return h ^ int(total)
