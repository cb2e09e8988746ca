"""ORACLE — test infrastructure only.

CPU restatement of the reference's parse-and-search algorithms (tomet-lang/oneline,
crates oneline-core + oneline-simd), used as the checker by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py``. The product package ``oneline_b200`` never imports this module.

* ``oracle.c``        single-threaded restatement (file:line citations inside);
* ``cpu_baseline.cpp`` multi-threaded port of oneline-simd, timed as the CPU baseline.

Parity pinning: the reference is Rust and cannot be compiled here (no cargo), so
the restatement is pinned by the reference's own known-answer and differential
tests, transcribed into ``tests/golden/reference_kat.json``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboneline_oracle.so")
NONE = 0xFFFFFFFF

NODE_DTYPE = np.dtype([("depth", "<u4"), ("kind", "<u4"), ("span_start", "<u4"), ("span_len", "<u4")])


def build(force: bool = False) -> str:
    """Compile oracle.c + cpu_baseline.cpp into liboneline_oracle.so (gcc/g++)."""
    srcs = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "cpu_baseline.cpp")]
    if not force and os.path.exists(LIB_PATH):
        lib_m = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(s) <= lib_m for s in srcs):
            return LIB_PATH
    obj_c = os.path.join(HERE, "_oracle_c.o")
    subprocess.run(["gcc", "-O2", "-fPIC", "-c", srcs[0], "-o", obj_c], check=True)
    subprocess.run(
        ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", srcs[1], obj_c, "-o", LIB_PATH],
        check=True,
    )
    os.remove(obj_c)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        u8p = ctypes.c_void_p
        u64 = ctypes.c_uint64
        L.olo_parse_line.argtypes = [u8p, u64, ctypes.c_uint32, ctypes.c_void_p]
        L.olo_parse_line_bytewise.argtypes = [u8p, u64, ctypes.c_uint32, ctypes.c_void_p]
        L.olo_count_lines.argtypes = [u8p, u64]
        L.olo_count_lines.restype = u64
        L.olo_scan_line_offsets.argtypes = [u8p, u64, ctypes.c_void_p, u64]
        L.olo_scan_line_offsets.restype = u64
        L.olo_parse.argtypes = [u8p, u64, ctypes.c_void_p, ctypes.c_void_p, u64]
        L.olo_parse.restype = u64
        L.olo_tree.argtypes = [ctypes.c_void_p, u64, ctypes.c_void_p, ctypes.c_void_p]
        L.olo_tree_children.argtypes = [ctypes.c_void_p, u64] + [ctypes.c_void_p] * 4
        L.olo_find_all.argtypes = [u8p, u64, u8p, u64, ctypes.c_void_p, u64]
        L.olo_find_all.restype = u64
        L.olo_find_many.argtypes = [u8p, u64, u8p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, u64]
        L.olo_find_many.restype = u64
        L.olb_parse_par.argtypes = [u8p, u64, ctypes.c_void_p, ctypes.c_void_p, u64, ctypes.c_int]
        L.olb_parse_par.restype = u64
        L.olb_build_links.argtypes = [ctypes.c_void_p, u64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.olb_children.argtypes = [ctypes.c_void_p, u64] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.olb_find_all_par.argtypes = [u8p, u64, u8p, u64, ctypes.c_void_p, u64, ctypes.c_int]
        L.olb_find_all_par.restype = u64
        L.olb_many_new.argtypes = [u8p, ctypes.c_void_p, ctypes.c_uint32]
        L.olb_many_new.restype = ctypes.c_void_p
        L.olb_many_free.argtypes = [ctypes.c_void_p]
        L.olb_many_states.argtypes = [ctypes.c_void_p]
        L.olb_many_states.restype = ctypes.c_uint32
        L.olb_many_find_all_par.argtypes = [ctypes.c_void_p, u8p, u64, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, u64, ctypes.c_int]
        L.olb_many_find_all_par.restype = u64
        L.olb_many_digest_par.argtypes = [ctypes.c_void_p, u8p, u64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.olb_many_digest_par.restype = u64
        L.olb_hit_digest.argtypes = [u64, ctypes.c_uint32, ctypes.c_uint32]
        L.olb_hit_digest.restype = u64
        _lib = L
    return _lib


def _buf(data) -> tuple:
    """(pointer, length, keepalive) for bytes / bytearray / uint8 numpy arrays."""
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.uint8)
        return a.ctypes.data, a.size, a
    b = bytes(data)
    a = np.frombuffer(b, dtype=np.uint8) if b else np.zeros(1, np.uint8)
    return a.ctypes.data, len(b), a


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ---------------------------------------------------------------- single line

def parse_line(line: bytes, line_start: int = 0) -> tuple:
    """(depth, kind, span_start, span_len) of one line (line.rs:8-81)."""
    out = np.zeros(1, NODE_DTYPE)
    p, n, _k = _buf(line)
    lib().olo_parse_line(p, n, line_start, _ptr(out))
    return tuple(int(v) for v in out[0])


def parse_line_bytewise(line: bytes, line_start: int = 0) -> tuple:
    """The reference's byte-loop oracle classifier (line.rs:89-142)."""
    out = np.zeros(1, NODE_DTYPE)
    p, n, _k = _buf(line)
    lib().olo_parse_line_bytewise(p, n, line_start, _ptr(out))
    return tuple(int(v) for v in out[0])


# ---------------------------------------------------------------- documents

def scan_line_offsets(text) -> np.ndarray:
    p, n, _k = _buf(text)
    cnt = lib().olo_count_lines(p, n)
    out = np.zeros(max(cnt, 1), np.uint32)
    got = lib().olo_scan_line_offsets(p, n, _ptr(out), cnt)
    assert got == cnt
    return out[:cnt]


def parse(text) -> tuple:
    """(offsets u32[L], nodes NODE_DTYPE[L]) — reference() of lib.rs:493-513."""
    p, n, _k = _buf(text)
    cnt = lib().olo_count_lines(p, n)
    offs = np.zeros(max(cnt, 1), np.uint32)
    nodes = np.zeros(max(cnt, 1), NODE_DTYPE)
    got = lib().olo_parse(p, n, _ptr(offs), _ptr(nodes), cnt)
    assert got == cnt
    return offs[:cnt], nodes[:cnt]


def tree(nodes: np.ndarray) -> tuple:
    """(parent, subtree_end) — TreeLinks::from_nodes_sequential (core links.rs:52-82)."""
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    n = nodes.size
    parent = np.zeros(max(n, 1), np.uint32)
    end = np.zeros(max(n, 1), np.uint32)
    lib().olo_tree(_ptr(nodes), n, _ptr(parent), _ptr(end))
    return parent[:n], end[:n]


def tree_children(nodes: np.ndarray, parent: np.ndarray, subtree_end: np.ndarray) -> tuple:
    """(first_child, next_sibling) derived from the links."""
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    n = nodes.size
    parent = np.ascontiguousarray(parent, np.uint32)
    subtree_end = np.ascontiguousarray(subtree_end, np.uint32)
    fc = np.zeros(max(n, 1), np.uint32)
    ns = np.zeros(max(n, 1), np.uint32)
    lib().olo_tree_children(_ptr(nodes), n, _ptr(parent), _ptr(subtree_end), _ptr(fc), _ptr(ns))
    return fc[:n], ns[:n]


def full_tree(nodes: np.ndarray) -> dict:
    parent, end = tree(nodes)
    fc, ns = tree_children(nodes, parent, end)
    return {"parent": parent, "subtree_end": end, "first_child": fc, "next_sibling": ns}


def find_all(text, pattern: bytes) -> np.ndarray:
    """Every overlapping occurrence, ascending (search.rs:106-114)."""
    p, n, _k = _buf(text)
    q, m, _k2 = _buf(pattern)
    total = lib().olo_find_all(p, n, q, m, 0, 0)
    out = np.zeros(max(total, 1), np.uint32)
    got = lib().olo_find_all(p, n, q, m, _ptr(out), total)
    assert got == total
    return out[:total]


def hit_digest(slot: int, pattern: int, offset: int) -> int:
    """The per-hit term of CpuMany.digest_par (for checking other implementations of it)."""
    return int(lib().olb_hit_digest(slot, pattern, offset))


def _pack(patterns) -> tuple:
    lens = np.array([len(x) for x in patterns], np.uint32)
    blob = b"".join(bytes(x) for x in patterns)
    arr = np.frombuffer(blob, np.uint8) if blob else np.zeros(1, np.uint8)
    return arr, lens


def find_many(text, patterns) -> tuple:
    """(counts u64[n], hit_pattern u32[H], hit_offset u32[H]) sorted by (pattern, offset)."""
    p, n, _k = _buf(text)
    arr, lens = _pack(patterns)
    counts = np.zeros(max(len(patterns), 1), np.uint64)
    total = lib().olo_find_many(p, n, _ptr(arr), _ptr(lens), len(patterns), _ptr(counts), 0, 0, 0)
    hp = np.zeros(max(total, 1), np.uint32)
    ho = np.zeros(max(total, 1), np.uint32)
    got = lib().olo_find_many(p, n, _ptr(arr), _ptr(lens), len(patterns), _ptr(counts), _ptr(hp), _ptr(ho), total)
    assert got == total
    return counts[: len(patterns)], hp[:total], ho[:total]


# ------------------------------------------------- multi-threaded CPU baseline

class CpuBaseline:
    """The timed CPU path: multi-threaded port of oneline-simd on `threads` cores."""

    def __init__(self, threads: int | None = None):
        self.threads = int(threads or os.cpu_count() or 1)

    def line_count(self, text) -> int:
        """Lines of the text, counted per chunk in parallel (the count pass of parse_par)."""
        p, n, _k = _buf(text)
        return int(lib().olb_parse_par(p, n, 0, 0, 0, self.threads)) if n else 0

    def parse_par(self, text) -> tuple:
        p, n, _k = _buf(text)
        cap = self.line_count(text)
        offs = np.zeros(max(cap, 1), np.uint32)
        nodes = np.zeros(max(cap, 1), NODE_DTYPE)
        got = lib().olb_parse_par(p, n, _ptr(offs), _ptr(nodes), cap, self.threads)
        assert got == cap
        return offs[:cap], nodes[:cap]

    def parse_par_into(self, text_ptr: int, n: int, offs: np.ndarray, nodes: np.ndarray) -> int:
        """parse_par into caller-sized outputs (ParseBuffers reuse, lib.rs:445-469); returns the line count."""
        return lib().olb_parse_par(text_ptr, n, _ptr(offs), _ptr(nodes), offs.size, self.threads)

    def build_links(self, nodes: np.ndarray, out: dict | None = None) -> dict:
        n = nodes.size
        out = out or {k: np.zeros(max(n, 1), np.uint32) for k in ("parent", "subtree_end", "first_child", "next_sibling")}
        lib().olb_build_links(_ptr(nodes), n, _ptr(out["parent"]), _ptr(out["subtree_end"]), self.threads)
        lib().olb_children(_ptr(nodes), n, _ptr(out["parent"]), _ptr(out["subtree_end"]),
                           _ptr(out["first_child"]), _ptr(out["next_sibling"]), self.threads)
        return {k: v[:n] for k, v in out.items()}

    def find_all_par(self, text, pattern: bytes, out: np.ndarray | None = None) -> tuple:
        p, n, _k = _buf(text)
        q, m, _k2 = _buf(pattern)
        if out is None:
            total = lib().olb_find_all_par(p, n, q, m, 0, 0, self.threads)
            out = np.zeros(max(total, 1), np.uint32)
        total = lib().olb_find_all_par(p, n, q, m, _ptr(out), out.size, self.threads)
        return total, out[: min(total, out.size)]

    def many(self, patterns) -> "CpuMany":
        return CpuMany(patterns, self.threads)


class CpuMany:
    def __init__(self, patterns, threads: int):
        self.n = len(patterns)
        arr, lens = _pack(patterns)
        self._h = lib().olb_many_new(_ptr(arr), _ptr(lens), self.n)
        self.threads = threads

    @property
    def states(self) -> int:
        return lib().olb_many_states(self._h)

    def find_all_par(self, text, cap: int | None = None) -> tuple:
        p, n, _k = _buf(text)
        counts = np.zeros(max(self.n, 1), np.uint64)
        if cap is None:
            cap = lib().olb_many_find_all_par(self._h, p, n, _ptr(counts), 0, 0, 0, self.threads)
        hp = np.zeros(max(cap, 1), np.uint32)
        ho = np.zeros(max(cap, 1), np.uint32)
        total = lib().olb_many_find_all_par(self._h, p, n, _ptr(counts), _ptr(hp), _ptr(ho), cap, self.threads)
        k = min(total, cap)
        return counts[: self.n], hp[:k], ho[:k], total

    def digest_par(self, text) -> tuple:
        """(counts u64[n], total, digest): the per-pattern counts and the order-checking
        digest of the whole (pattern, offset)-ordered hit list (hit_digest summed over
        the slots), without materialising the list."""
        p, n, _k = _buf(text)
        counts = np.zeros(max(self.n, 1), np.uint64)
        total = ctypes.c_uint64()
        dg = lib().olb_many_digest_par(self._h, p, n, _ptr(counts), ctypes.addressof(total), self.threads)
        return counts[: self.n], int(total.value), int(dg)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.olb_many_free(h)
            self._h = None
