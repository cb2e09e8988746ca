"""GpuServer: the serving loop of the CUDA library (ol_server_* in
include/oneline_cuda.h), for parse and search requests of mixed sizes.

Worker threads in the library each own a context and a stream; requests queue
as they arrive and start as soon as a worker frees up, so their kernels overlap
on the device. Parsed documents stay resident in an HBM-budgeted store and are
searched without uploading their text again. No reference counterpart: the
reference offers one blocking call per document (crates/oneline-gpu/src/parser.rs).
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


class GpuServer:
    def __init__(self, device: int = 0, workers: int = 8, store_budget: int = 4 << 30, max_hits: int = 1 << 22):
        h = ctypes.c_void_p()
        st = _lib.load().ol_server_create(device, workers, store_budget, max_hits, ctypes.byref(h))
        if st != 0:
            raise OnelineError(st, "could not start the server")
        self._h = h.value
        self._keep = {}  # request id -> buffers that must outlive the request

    def submit_parse(self, text) -> int:
        buf = np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray)) else np.ascontiguousarray(text, np.uint8)
        rid = ctypes.c_uint64()
        st = _lib.load().ol_server_submit_parse(self._h, buf.ctypes.data, buf.size, ctypes.byref(rid))
        if st != 0:
            raise OnelineError(st, "submit_parse")
        self._keep[rid.value] = buf
        return rid.value

    def submit_search(self, doc_id: int, patterns) -> int:
        pats = [bytes(p) for p in patterns]
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        P = (ctypes.c_void_p * len(pats))(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats], np.uint32)
        rid = ctypes.c_uint64()
        st = _lib.load().ol_server_submit_search(self._h, int(doc_id), P, lens.ctypes.data, len(pats),
                                                 ctypes.byref(rid))
        if st != 0:
            raise OnelineError(st, "submit_search")
        return rid.value  # the patterns are copied at submission

    def wait(self, request_id: int) -> RequestResult:
        r = RequestResult()
        st = _lib.load().ol_server_wait(self._h, request_id, ctypes.byref(r))
        if st != 0:
            raise OnelineError(st, "wait")
        self._keep.pop(request_id, None)
        return r

    def stats(self) -> dict:
        v = [ctypes.c_uint64() for _ in range(4)]
        _lib.load().ol_server_stats(self._h, *[ctypes.byref(x) for x in v])
        return dict(zip(("resident_docs", "resident_bytes", "evictions", "refusals"), (int(x.value) for x in v)))

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
