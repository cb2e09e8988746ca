"""GpuParser and friends: the public API of crates/oneline-gpu, over the C ABI.

Method names, argument meaning and error behaviour follow the reference:

* ``GpuParser.upload`` / ``GpuDocument``               document.rs:16-90, 111-127
* ``GpuParser.parse_raw`` / ``parse`` / ``scan_line_offsets``  parse.rs:86-125, scan.rs:127-136
* ``GpuParser.build_tree`` / ``build_tree_reusing`` / ``download_links`` / ``GpuTree``
                                                        tree.rs:34-67, 278-290
* ``GpuParser.search_document`` / ``search_raw`` / ``SearchResult``  search.rs:12-140
* ``GpuParser.query_document`` / ``query_subtree`` / ``query_raw`` / ``query`` / ``QueryResult``
                                                        document.rs:94-127, tree.rs:292-313, query.rs:10-19, 228-329
* ``GpuParser.compile_patterns`` / ``search_many`` / ``GpuPatternSet`` / ``ManyResult``
                                                        many.rs:14-18, 76-94, 139-176, 391-399
* ``GpuParser.profile_*`` / ``Profile``                 timing.rs:109-124, document.rs:136-157, search.rs:143-173,
                                                        many.rs:401-410, tree.rs:69-82, query.rs:275
* limits ``MAX_PATTERN_LEN``, ``MAX_TREE_DEPTH``, ``MAX_GPU_INPUT_LEN``  lib.rs:66, tree.rs:12, util.rs:8

Errors are raised as ``OnelineError`` (the reference returns ``anyhow::Error``);
a failed call leaves the parser usable. Every computation runs in the CUDA
library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import OnelineError, check
from .core import NODE_DTYPE, NONE, FlatTree, TreeLinks

MAX_PATTERN_LEN = 64
MAX_PATTERNS = 2048           # many.rs:14 (drop-in set size)
MIN_SET_PATTERN_LEN = 4       # many.rs:17
MAX_SET_PATTERN_LEN = 64      # many.rs:18
MAX_DICT_PATTERNS = 65536     # this engine's set size limit
HIT_DTYPE = np.dtype([("pattern", "<u4"), ("offset", "<u4")])  # ManyHit (many.rs:76-82)
MAX_TREE_DEPTH = 32
MAX_GPU_INPUT_LEN = 0xFFFFFFFF - 3
TREE_STRICT_DEPTH = 1


def _as_bytes_view(data) -> tuple[int, int, object, bytes | np.ndarray]:
    """(pointer, length, keepalive, source) for str / bytes / bytearray / uint8 arrays."""
    if isinstance(data, str):
        data = data.encode("utf-8")
    if isinstance(data, np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        return a.ctypes.data, a.size, a, a
    if isinstance(data, (bytes, bytearray, memoryview)):
        b = bytes(data)
        if not b:
            return 0, 0, b, b
        a = np.frombuffer(b, dtype=np.uint8)
        return a.ctypes.data, a.size, a, b
    raise TypeError(f"expected str, bytes or a uint8 array, got {type(data).__name__}")


def _check_len(n: int) -> None:
    if n > MAX_GPU_INPUT_LEN:
        raise OnelineError(2, f"input is {n} bytes; the GPU path addresses at most {MAX_GPU_INPUT_LEN} bytes "
                              "(32-bit offsets)")


class _ProfileStep(ctypes.Structure):
    _fields_ = [("label", ctypes.c_char * 40), ("ns", ctypes.c_uint64)]


class _Profile(ctypes.Structure):
    """ol_profile (include/oneline_cuda.h)."""

    _fields_ = [("wall_ns", ctypes.c_uint64), ("gpu_total_ns", ctypes.c_uint64), ("n_host_steps", ctypes.c_uint32),
                ("n_gpu_passes", ctypes.c_uint32), ("host_steps", _ProfileStep * 32), ("gpu_passes", _ProfileStep * 32)]


@dataclass
class Profile:
    """Where the time of one run went (timing.rs:109-124): host wall clock, the
    host steps in order (time since the previous step) and the GPU passes with
    their device time (CUDA events), all in seconds."""

    wall: float
    host_steps: list
    gpu_passes: list

    def gpu_total(self) -> float:
        return sum(d for _, d in self.gpu_passes)

    @staticmethod
    def _from(raw: _Profile) -> "Profile":
        steps = [(raw.host_steps[i].label.decode(), raw.host_steps[i].ns / 1e9) for i in range(raw.n_host_steps)]
        passes = [(raw.gpu_passes[i].label.decode(), raw.gpu_passes[i].ns / 1e9) for i in range(raw.n_gpu_passes)]
        return Profile(raw.wall_ns / 1e9, steps, passes)


@dataclass
class SearchResult:
    """Substring search result (search.rs:12-21). ``offsets`` ascend; when
    truncated by ``max_matches`` they are the lowest ``max_matches`` offsets."""

    total_matches: int
    offsets: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))

    def __eq__(self, other) -> bool:
        return (isinstance(other, SearchResult) and self.total_matches == other.total_matches
                and np.array_equal(self.offsets, other.offsets))


class GpuDocument:
    """A document parsed once and kept in device memory (document.rs:16-127)."""

    def __init__(self, parser: "GpuParser", handle: int, source):
        self._parser = parser
        self._h = handle
        self._source = source
        parser._children.add(self)

    @property
    def handle(self) -> int:
        return self._h

    def line_count(self) -> int:
        return int(_lib.load().ol_doc_line_count(self._h))

    def text_len(self) -> int:
        return int(_lib.load().ol_doc_text_len(self._h))

    def max_depth(self) -> int:
        return int(_lib.load().ol_doc_max_depth(self._h))

    def read_offsets(self) -> np.ndarray:
        n = self.line_count()
        out = np.zeros(max(n, 1), np.uint32)
        check(_lib.load().ol_doc_read_offsets(self._parser._ctx, self._h, out.ctypes.data, out.size), self._parser._ctx)
        return out[:n]

    def read_kinds(self) -> np.ndarray:
        n = self.line_count()
        out = np.zeros(max(n, 1), np.uint8)
        check(_lib.load().ol_doc_read_kinds(self._parser._ctx, self._h, out.ctypes.data, out.size), self._parser._ctx)
        return out[:n]

    def read_nodes(self) -> np.ndarray:
        n = self.line_count()
        out = np.zeros(max(n, 1), NODE_DTYPE)
        check(_lib.load().ol_doc_read_nodes(self._parser._ctx, self._h, out.ctypes.data, out.size), self._parser._ctx)
        return out[:n]

    def free(self) -> None:
        # A document never outlives its parser's context: GpuParser.close()
        # frees the documents and trees it still owns before destroying it.
        if self._h and self._parser._ctx:
            _lib.load().ol_doc_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GpuTree:
    """Tree links of a resident document (tree.rs:29-46)."""

    def __init__(self, parser: "GpuParser", handle: int):
        self._parser = parser
        self._h = handle
        parser._children.add(self)

    @property
    def handle(self) -> int:
        return self._h

    def line_count(self) -> int:
        return int(_lib.load().ol_tree_line_count(self._h))

    def _take(self) -> int:
        h, self._h = self._h, None
        return h

    def free(self) -> None:
        if self._h and self._parser._ctx:
            _lib.load().ol_tree_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Tuning(ctypes.Structure):
    """ol_tuning: the kernel variants a context uses (speed only, never results)."""

    _fields_ = [("dict_slice", ctypes.c_uint32), ("dict_blocks_per_sm", ctypes.c_uint32),
                ("dict_heavy_divisor", ctypes.c_uint32), ("search_staged", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


@dataclass
class QueryResult:
    """Result of a node query (query.rs:10-19): the number of matching lines and
    the first ``max_matches`` of them in ascending order."""

    total_matches: int
    indices: np.ndarray


@dataclass
class ManyResult:
    """Result of a dictionary search (many.rs:84-94). ``hits`` is a structured
    array (``pattern``, ``offset``) sorted by (pattern, offset); when there are more
    than ``max_hits`` it holds the first ``max_hits`` of that order."""

    counts: np.ndarray
    total_hits: int
    hits: np.ndarray = field(default_factory=lambda: np.zeros(0, HIT_DTYPE))


class GpuPatternSet:
    """A compiled dictionary (many.rs:116-147)."""

    def __init__(self, parser: "GpuParser", handle: int, n: int):
        self._parser = parser
        self._h = handle
        self._n = n
        parser._children.add(self)

    @property
    def handle(self) -> int:
        return self._h

    def __len__(self) -> int:
        return self._n

    def len(self) -> int:
        return self._n

    def is_empty(self) -> bool:
        return self._n == 0

    def unique(self) -> int:
        return int(_lib.load().ol_patset_unique(self._h))

    def free(self) -> None:
        if self._h and self._parser._ctx:
            _lib.load().ol_patset_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GpuPipeline:
    """A captured re-parse + tree + multi-pattern search of one resident document,
    replayed as one CUDA graph launch (no reference counterpart)."""

    def __init__(self, parser: "GpuParser", handle: int, keep):
        self._parser = parser
        self._h = handle
        self._keep = keep
        parser._children.add(self)

    def launch(self) -> None:
        check(_lib.load().ol_pipeline_launch(self._h))

    def sync(self) -> None:
        check(_lib.load().ol_pipeline_sync(self._h))

    @property
    def stream(self) -> int:
        return int(_lib.load().ol_pipeline_stream(self._h) or 0)

    @property
    def kernels(self) -> int:
        return int(_lib.load().ol_pipeline_kernels(self._h))

    def free(self) -> None:
        if self._h and self._parser._ctx:
            _lib.load().ol_pipeline_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GpuBatch:
    """Many documents resident as one text (no reference counterpart: per document
    the results equal upload / build_tree / search_many on that document alone)."""

    def __init__(self, parser: "GpuParser", handle: int):
        self._parser = parser
        self._h = handle
        parser._children.add(self)

    @property
    def handle(self) -> int:
        return self._h

    def __len__(self) -> int:
        return int(_lib.load().ol_batch_docs(self._h))

    def text_len(self) -> int:
        return int(_lib.load().ol_batch_text_len(self._h))

    def doc_info(self, i: int) -> tuple[int, int, int, int]:
        """(text_start, text_len, first_line, line_count) of document i."""
        v = [ctypes.c_uint64() for _ in range(4)]
        check(_lib.load().ol_batch_doc_info(self._h, i, *[ctypes.byref(x) for x in v]))
        return tuple(int(x.value) for x in v)

    def free(self) -> None:
        if self._h and self._parser._ctx:
            _lib.load().ol_batch_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GpuParser:
    """Parser and search engine on one CUDA device (parser.rs:8-142)."""

    def __init__(self, device: int = 0):
        L = _lib.load()
        h = ctypes.c_void_p()
        st = L.ol_ctx_create(device, ctypes.byref(h))
        if st != 0:
            raise OnelineError(st, f"cannot create a CUDA context on device {device}")
        self._ctx = h.value
        self._children = weakref.WeakSet()  # documents and trees that hold device memory

    @classmethod
    def new(cls, device: int = 0) -> "GpuParser":
        return cls(device)

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            for child in list(self._children):
                child.free()
            _lib.load().ol_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ctx(self) -> int:
        return self._ctx

    def adapter_name(self) -> str:
        buf = ctypes.create_string_buffer(256)
        check(_lib.load().ol_ctx_device_name(self._ctx, buf, 256), self._ctx)
        return buf.value.decode()

    def is_software(self) -> bool:
        return False

    def timestamps_supported(self) -> bool:
        return True

    def sync(self) -> None:
        check(_lib.load().ol_ctx_sync(self._ctx), self._ctx)

    # ------------------------------------------------------------ documents

    def upload(self, text) -> GpuDocument:
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        h = ctypes.c_void_p()
        check(_lib.load().ol_doc_upload(self._ctx, p, n, ctypes.byref(h)), self._ctx)
        return GpuDocument(self, h.value, src)

    def upload_device(self, dev_ptr: int, n: int) -> GpuDocument:
        """Upload from this device's memory (e.g. a torch CUDA uint8 tensor's data_ptr)."""
        _check_len(n)
        h = ctypes.c_void_p()
        check(_lib.load().ol_doc_upload_device(self._ctx, dev_ptr, n, ctypes.byref(h)), self._ctx)
        return GpuDocument(self, h.value, None)

    def parse_raw(self, text) -> FlatTree:
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        L = _lib.load()
        cnt = ctypes.c_uint64()
        check(L.ol_parse_raw(self._ctx, p, n, None, None, 0, ctypes.byref(cnt)), self._ctx)
        lines = cnt.value
        offs = np.zeros(max(lines, 1), np.uint32)
        nodes = np.zeros(max(lines, 1), NODE_DTYPE)
        if lines:
            check(L.ol_parse_raw(self._ctx, p, n, offs.ctypes.data, nodes.ctypes.data, lines, ctypes.byref(cnt)), self._ctx)
        return FlatTree(src if isinstance(src, bytes) else bytes(src), nodes[:lines], offs[:lines])

    def parse(self, text, line_offsets) -> FlatTree:
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        offs = np.ascontiguousarray(line_offsets, np.uint32)
        nodes = np.zeros(max(offs.size, 1), NODE_DTYPE)
        if offs.size:
            check(_lib.load().ol_parse_with_offsets(self._ctx, p, n, offs.ctypes.data, offs.size, nodes.ctypes.data),
                  self._ctx)
        return FlatTree(src if isinstance(src, bytes) else bytes(src), nodes[: offs.size], offs.copy())

    def scan_line_offsets(self, text) -> np.ndarray:
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        L = _lib.load()
        cnt = ctypes.c_uint64()
        check(L.ol_scan_line_offsets(self._ctx, p, n, None, 0, ctypes.byref(cnt)), self._ctx)
        out = np.zeros(max(cnt.value, 1), np.uint32)
        if cnt.value:
            check(L.ol_scan_line_offsets(self._ctx, p, n, out.ctypes.data, out.size, ctypes.byref(cnt)), self._ctx)
        return out[: cnt.value]

    # ----------------------------------------------------------------- tree

    def build_tree(self, doc: GpuDocument, *, strict_depth: bool = True) -> GpuTree:
        """Tree links of `doc`. Like the reference, a content line nested 32 or more
        levels deep is an error unless ``strict_depth=False`` (then any depth works)."""
        return self.build_tree_reusing(doc, None, strict_depth=strict_depth)

    def build_tree_reusing(self, doc: GpuDocument, previous: GpuTree | None, *, strict_depth: bool = True) -> GpuTree:
        h = ctypes.c_void_p()
        prev = previous._take() if previous is not None else None
        flags = TREE_STRICT_DEPTH if strict_depth else 0
        check(_lib.load().ol_tree_build_reusing(self._ctx, doc.handle, prev, flags, ctypes.byref(h)), self._ctx)
        return GpuTree(self, h.value)

    def _read_tree(self, tree: GpuTree, which: tuple[str, ...]) -> dict:
        n = tree.line_count()
        arrs = {k: np.zeros(max(n, 1), np.uint32) for k in which}
        ptr = lambda k: arrs[k].ctypes.data if k in arrs else None  # noqa: E731
        check(_lib.load().ol_tree_read(self._ctx, tree.handle, ptr("parent"), ptr("subtree_end"), ptr("first_child"),
                                       ptr("next_sibling"), max(n, 1)), self._ctx)
        return {k: v[:n] for k, v in arrs.items()}

    def download_links(self, tree: GpuTree) -> TreeLinks:
        a = self._read_tree(tree, ("parent", "subtree_end"))
        return TreeLinks(a["parent"], a["subtree_end"])

    def download_tree(self, tree: GpuTree) -> dict:
        """parent, subtree_end, first_child and next_sibling of every line."""
        return self._read_tree(tree, ("parent", "subtree_end", "first_child", "next_sibling"))

    # ------------------------------------------------------------ .olb files

    def save_olb(self, doc: GpuDocument, path: str) -> None:
        """Writes the resident document's text, nodes and line offsets as an .olb file."""
        check(_lib.load().ol_doc_save_olb(self._ctx, doc.handle, path.encode()), self._ctx)

    def load_olb(self, path: str, *, verify: bool = False) -> GpuDocument:
        """A resident document from an .olb file, without parsing its text
        (``verify`` also checks the file's CRC-32)."""
        h = ctypes.c_void_p()
        check(_lib.load().ol_doc_load_olb(self._ctx, path.encode(), 1 if verify else 0, ctypes.byref(h)), self._ctx)
        return GpuDocument(self, h.value, path)

    # --------------------------------------------------------------- search

    @staticmethod
    def _check_pattern(pattern: bytes, max_len: int | None) -> bytes:
        pattern = pattern.encode() if isinstance(pattern, str) else bytes(pattern)
        if not pattern or (max_len is not None and len(pattern) > max_len):
            lim = max_len if max_len is not None else "any"
            raise OnelineError(3, f"pattern must be 1..={lim} bytes, got {len(pattern)}")
        return pattern

    def search_document(self, doc: GpuDocument, pattern: bytes, max_matches: int, *,
                        max_pattern_len: int | None = MAX_PATTERN_LEN) -> SearchResult:
        """Every (overlapping) occurrence of `pattern` in a resident document.
        The reference accepts 1..=64 bytes; pass ``max_pattern_len=None`` for any length."""
        pattern = self._check_pattern(pattern, max_pattern_len)
        if max_matches > 0xFFFFFFFF:
            raise OnelineError(1, f"max_matches {max_matches} does not fit in u32")
        out = np.zeros(max(max_matches, 1), np.uint32)
        total = ctypes.c_uint32()
        pa = np.frombuffer(pattern, np.uint8)
        check(_lib.load().ol_search(self._ctx, doc.handle, pa.ctypes.data, len(pattern), max_matches,
                                    ctypes.byref(total), out.ctypes.data), self._ctx)
        k = min(total.value, max_matches)
        return SearchResult(total.value, out[:k].copy())

    def search_document_multi(self, doc: GpuDocument, patterns, max_matches) -> list:
        """Several patterns at once (up to eight share each pass over the text).
        `max_matches` is one int for all or one per pattern. Any pattern length."""
        pats = [self._check_pattern(p, None) for p in patterns]
        n = len(pats)
        if n == 0:
            return []
        maxes = [int(max_matches)] * n if np.isscalar(max_matches) else [int(m) for m in max_matches]
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        outs = [np.zeros(max(m, 1), np.uint32) for m in maxes]
        P = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats], np.uint32)
        mx = np.array(maxes, np.uint32)
        tot = np.zeros(n, np.uint32)
        O = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        check(_lib.load().ol_search_multi(self._ctx, doc.handle, P, lens.ctypes.data, n, mx.ctypes.data,
                                          tot.ctypes.data, O), self._ctx)
        return [SearchResult(int(t), o[: min(int(t), m)].copy()) for t, o, m in zip(tot, outs, maxes)]

    def search_raw(self, text, pattern: bytes, max_matches: int, *,
                   max_pattern_len: int | None = MAX_PATTERN_LEN) -> SearchResult:
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        pattern = self._check_pattern(pattern, max_pattern_len)
        out = np.zeros(max(max_matches, 1), np.uint32)
        total = ctypes.c_uint32()
        pa = np.frombuffer(pattern, np.uint8)
        check(_lib.load().ol_search_raw(self._ctx, p, n, pa.ctypes.data, len(pattern), max_matches,
                                        ctypes.byref(total), out.ctypes.data), self._ctx)
        k = min(total.value, max_matches)
        return SearchResult(total.value, out[:k].copy())

    @staticmethod
    def _filter(kind, depth) -> tuple[int, int]:
        # query.rs:138-139: None -> 0 (any kind), None -> 0xFFFFFFFF (any depth)
        k = 0 if kind is None else int(kind)
        d = 0xFFFFFFFF if depth is None else int(depth)
        return k, d

    def _query_out(self, fn, *args, max_matches: int) -> QueryResult:
        if not 0 <= max_matches <= 0xFFFFFFFF:
            raise OnelineError(1, f"max_matches {max_matches} does not fit in u32")
        out = np.zeros(max(max_matches, 1), np.uint32)
        total = ctypes.c_uint32()
        check(fn(self._ctx, *args, max_matches, ctypes.byref(total), out.ctypes.data), self._ctx)
        return QueryResult(total.value, out[: min(total.value, max_matches)].copy())

    def query_document(self, doc: GpuDocument, kind=None, depth=None, max_matches: int = 1 << 20) -> QueryResult:
        """Lines of a resident document with the given kind and depth (document.rs:94-102)."""
        k, d = self._filter(kind, depth)
        return self._query_out(_lib.load().ol_query_document, doc.handle, k, d, max_matches=max_matches)

    def query_subtree(self, doc: GpuDocument, tree: GpuTree, root: int, kind=None, depth=None,
                      max_matches: int = 1 << 20) -> QueryResult:
        """The same over the subtree of `root`, lines [root, subtree_end[root]) (tree.rs:292-313)."""
        k, d = self._filter(kind, depth)
        return self._query_out(_lib.load().ol_query_subtree, doc.handle, tree.handle, int(root), k, d,
                               max_matches=max_matches)

    def query_raw(self, text, kind=None, depth=None, max_matches: int = 1 << 20) -> np.ndarray:
        """One-shot query on raw text (query.rs:230-242): the matching line indices."""
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        k, d = self._filter(kind, depth)
        return self._query_out(_lib.load().ol_query_raw, p, n, k, d, max_matches=max_matches).indices

    def query(self, text, line_offsets, kind=None, depth=None, max_matches: int = 1 << 20) -> np.ndarray:
        """One-shot query with line offsets computed elsewhere (query.rs:287-312)."""
        p, n, keep, src = _as_bytes_view(text)
        _check_len(n)
        offs = np.ascontiguousarray(line_offsets, dtype=np.uint32)
        k, d = self._filter(kind, depth)
        return self._query_out(_lib.load().ol_query, p, n, offs.ctypes.data, offs.size, k, d,
                               max_matches=max_matches).indices

    def compile_patterns(self, doc: GpuDocument | None, patterns, *,
                         max_patterns: int | None = MAX_PATTERNS) -> GpuPatternSet:
        """Compiles a dictionary (many.rs:158-176): 1..=2048 patterns of 4..=64 bytes, like
        the reference; ``max_patterns=None`` allows up to 65,536."""
        pats = [p.encode("utf-8") if isinstance(p, str) else bytes(p) for p in patterns]
        limit = MAX_DICT_PATTERNS if max_patterns is None else min(max_patterns, MAX_DICT_PATTERNS)
        if not 1 <= len(pats) <= limit:
            raise OnelineError(3, f"pattern count {len(pats)} is outside 1..={limit}")
        for i, p in enumerate(pats):
            if not MIN_SET_PATTERN_LEN <= len(p) <= MAX_SET_PATTERN_LEN:
                raise OnelineError(3, f"pattern {i} has {len(p)} bytes; set patterns need "
                                      f"{MIN_SET_PATTERN_LEN}..={MAX_SET_PATTERN_LEN}")
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        P = (ctypes.c_void_p * len(pats))(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats], np.uint32)
        h = ctypes.c_void_p()
        check(_lib.load().ol_patset_compile(self._ctx, doc.handle if doc is not None else None, P,
                                            lens.ctypes.data, len(pats), ctypes.byref(h)), self._ctx)
        return GpuPatternSet(self, h.value, len(pats))

    def search_many(self, doc: GpuDocument, pattern_set: GpuPatternSet, max_hits: int) -> ManyResult:
        """Every (pattern, offset) of the set in ``doc`` (many.rs:391-399): counts per
        pattern, the total, and up to ``max_hits`` hits in (pattern, offset) order."""
        if max_hits < 0:
            raise OnelineError(1, "max_hits must not be negative")
        n = len(pattern_set)
        counts = np.zeros(n, np.uint32)
        total = ctypes.c_uint64()
        hits = np.zeros(max(int(max_hits), 1), HIT_DTYPE)
        check(_lib.load().ol_search_many(self._ctx, doc.handle, pattern_set.handle, int(max_hits),
                                         counts.ctypes.data, ctypes.byref(total), hits.ctypes.data), self._ctx)
        k = min(int(total.value), int(max_hits))
        return ManyResult(counts, int(total.value), hits[:k].copy())

    def search_many_device(self, doc: GpuDocument, pattern_set: GpuPatternSet, d_hits: int, max_hits: int, *,
                           heavy_min_hits: int = 0) -> tuple[np.ndarray, int]:
        """``search_many`` with the hits left in device memory at ``d_hits`` (room for
        ``max_hits``); returns (counts, total_hits). ``heavy_min_hits`` tunes how hits
        are collected (0: automatic) and never changes the result."""
        n = len(pattern_set)
        counts = np.zeros(n, np.uint32)
        total = ctypes.c_uint64()
        check(_lib.load().ol_search_many_device(self._ctx, doc.handle, pattern_set.handle, int(max_hits),
                                                int(heavy_min_hits), counts.ctypes.data, ctypes.byref(total),
                                                d_hits), self._ctx)
        return counts, int(total.value)

    def search_many_u64(self, doc: GpuDocument, pattern_set: GpuPatternSet, max_hits: int) -> tuple:
        """``search_many`` in the (pattern id u32, byte offset u64) form: returns
        (counts, total_hits, patterns u32[k], offsets u64[k]), k = min(total, max_hits)."""
        if max_hits < 0:
            raise OnelineError(1, "max_hits must not be negative")
        counts = np.zeros(len(pattern_set), np.uint32)
        total = ctypes.c_uint64()
        pats = np.zeros(max(int(max_hits), 1), np.uint32)
        offs = np.zeros(max(int(max_hits), 1), np.uint64)
        check(_lib.load().ol_search_many_u64(self._ctx, doc.handle, pattern_set.handle, int(max_hits),
                                             counts.ctypes.data, ctypes.byref(total), pats.ctypes.data,
                                             offs.ctypes.data), self._ctx)
        k = min(int(total.value), int(max_hits))
        return counts, int(total.value), pats[:k].copy(), offs[:k].copy()

    def search_many_device_u64(self, doc: GpuDocument, pattern_set: GpuPatternSet, d_patterns: int, d_offsets: int,
                               max_hits: int, *, heavy_min_hits: int = 0) -> tuple[np.ndarray, int]:
        """``search_many_u64`` with the two arrays in device memory; returns (counts, total_hits)."""
        counts = np.zeros(len(pattern_set), np.uint32)
        total = ctypes.c_uint64()
        check(_lib.load().ol_search_many_device_u64(self._ctx, doc.handle, pattern_set.handle, int(max_hits),
                                                    int(heavy_min_hits), counts.ctypes.data, ctypes.byref(total),
                                                    d_patterns, d_offsets), self._ctx)
        return counts, int(total.value)

    # -------------------------------------------------------------- batches

    def upload_batch(self, docs) -> GpuBatch:
        """Uploads and parses many documents as one batch; `docs` is a list of
        byte strings, or (data, offsets) with document i = data[offsets[i]:offsets[i+1]]."""
        if isinstance(docs, tuple):
            data, offs = docs
            data = np.ascontiguousarray(np.frombuffer(data, np.uint8) if isinstance(data, (bytes, bytearray)) else data,
                                        dtype=np.uint8)
            offs = np.ascontiguousarray(offs, dtype=np.uint64)
        else:
            parts = [d.encode("utf-8") if isinstance(d, str) else bytes(d) for d in docs]
            data = np.frombuffer(b"".join(parts), np.uint8) if parts and any(parts) else np.zeros(1, np.uint8)
            offs = np.zeros(len(parts) + 1, np.uint64)
            offs[1:] = np.cumsum([len(p) for p in parts])
        h = ctypes.c_void_p()
        check(_lib.load().ol_batch_upload(self._ctx, data.ctypes.data, offs.ctypes.data, offs.size - 1,
                                          ctypes.byref(h)), self._ctx)
        return GpuBatch(self, h.value)

    def build_batch_trees(self, batch: GpuBatch) -> None:
        check(_lib.load().ol_batch_build_trees(self._ctx, batch.handle), self._ctx)

    def read_batch_doc(self, batch: GpuBatch, i: int, *, tree: bool = True) -> dict:
        """Document i's offsets, kinds and (when built) tree links, all relative to the document."""
        _, _, _, n = batch.doc_info(i)
        out = {"offsets": np.zeros(max(n, 1), np.uint32), "kinds": np.zeros(max(n, 1), np.uint8)}
        names = ("parent", "subtree_end", "first_child", "next_sibling")
        for k in names:
            out[k] = np.zeros(max(n, 1), np.uint32) if tree else None
        ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
        check(_lib.load().ol_batch_read_doc(self._ctx, batch.handle, i, ptr(out["offsets"]), ptr(out["kinds"]),
                                            *[ptr(out[k]) for k in names], n), self._ctx)
        return {k: (v[:n] if v is not None else None) for k, v in out.items()}

    def batch_search_many(self, batch: GpuBatch, pattern_set: GpuPatternSet, d_hits: int, max_hits: int, *,
                          heavy_min_hits: int = 0) -> tuple[np.ndarray, int]:
        """Dictionary search of every document of the batch; hits (device, at d_hits) hold
        offsets in the batch text, in (pattern, document, offset) order. Returns (counts, total)."""
        counts = np.zeros(len(pattern_set), np.uint32)
        total = ctypes.c_uint64()
        check(_lib.load().ol_batch_search_many(self._ctx, batch.handle, pattern_set.handle, int(max_hits),
                                               int(heavy_min_hits), counts.ctypes.data, ctypes.byref(total),
                                               d_hits), self._ctx)
        return counts, int(total.value)

    # ------------------------------------------------------------- pipeline

    def capture_pipeline(self, doc: GpuDocument, tree: GpuTree, patterns, max_matches, d_totals: int,
                         d_outs) -> GpuPipeline:
        """Captures re-parse + tree + search of `patterns` over `doc` as one CUDA graph.
        d_totals (u32 per pattern) and d_outs (one u32 buffer per pattern, room for
        max_matches[i]) are device pointers that must outlive the pipeline."""
        pats = [self._check_pattern(p, None) for p in patterns]
        n = len(pats)
        maxes = np.array([int(max_matches)] * n if np.isscalar(max_matches) else [int(m) for m in max_matches],
                         np.uint32)
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        P = (ctypes.c_void_p * max(n, 1))(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats], np.uint32)
        O = (ctypes.c_void_p * max(n, 1))(*[int(o) for o in d_outs])
        h = ctypes.c_void_p()
        check(_lib.load().ol_pipeline_capture(self._ctx, doc.handle, tree.handle, P, lens.ctypes.data, n,
                                              maxes.ctypes.data, d_totals, O, ctypes.byref(h)), self._ctx)
        return GpuPipeline(self, h.value, (doc, tree))

    # --------------------------------------------------------------- tuning

    @property
    def tuning(self) -> dict:
        t = Tuning()
        check(_lib.load().ol_tuning_get(self._ctx, ctypes.byref(t)), self._ctx)
        return t.as_dict()

    def set_tuning(self, **values) -> None:
        t = Tuning(**{**self.tuning, **values})
        check(_lib.load().ol_tuning_set(self._ctx, ctypes.byref(t)), self._ctx)

    def autotune(self, doc: GpuDocument, pattern_set: "GpuPatternSet | None" = None, patterns=(),
                 path: str | None = None) -> dict:
        """Measures the kernel variants on `doc` (dictionary ones with `pattern_set`,
        substring-search ones with `patterns`), keeps the fastest and records them
        in the file at `path` under this device."""
        pats = [self._check_pattern(p, None) for p in patterns]
        bufs = [np.frombuffer(p, np.uint8) for p in pats]
        P = (ctypes.c_void_p * max(len(pats), 1))(*[b.ctypes.data for b in bufs])
        lens = np.array([len(p) for p in pats] or [0], np.uint32)
        t = Tuning()
        check(_lib.load().ol_autotune(self._ctx, doc.handle, pattern_set.handle if pattern_set else None, P,
                                      lens.ctypes.data, len(pats), path.encode() if path else None, ctypes.byref(t)),
              self._ctx)
        return t.as_dict()

    def tuning_load(self, path: str) -> dict:
        check(_lib.load().ol_tuning_load(self._ctx, path.encode()), self._ctx)
        return self.tuning

    # ------------------------------------------------------------ profiling

    def _profiled(self, fn, *args, **kw):
        """(fn's result, Profile) with the context's profile open around fn."""
        L = _lib.load()
        check(L.ol_profile_begin(self._ctx), self._ctx)
        raw = _Profile()
        try:
            out = fn(*args, **kw)
        finally:
            st = L.ol_profile_end(self._ctx, ctypes.byref(raw))
        check(st, self._ctx)
        return out, Profile._from(raw)

    def profile_upload(self, text) -> tuple[GpuDocument, Profile]:
        """``upload``, with a breakdown of where the time went (waits for the parse)."""
        return self._profiled(self.upload, text)

    def profile_query_document(self, doc: GpuDocument, kind=None, depth=None, max_matches: int = 1 << 20) -> Profile:
        return self._profiled(self.query_document, doc, kind, depth, max_matches)[1]

    def profile_search_document(self, doc: GpuDocument, pattern: bytes, max_matches: int) -> Profile:
        return self._profiled(self.search_document, doc, pattern, max_matches)[1]

    def profile_search_raw(self, text, pattern: bytes, max_matches: int) -> Profile:
        return self._profiled(self.search_raw, text, pattern, max_matches)[1]

    def profile_search_many(self, doc: GpuDocument, pattern_set: "GpuPatternSet", max_hits: int) -> Profile:
        return self._profiled(self.search_many, doc, pattern_set, max_hits)[1]

    def profile_build_tree_reusing(self, doc: GpuDocument, previous: "GpuTree | None") -> tuple["GpuTree", Profile]:
        return self._profiled(self.build_tree_reusing, doc, previous)

    def profile_build_tree(self, doc: GpuDocument) -> Profile:
        tree, prof = self.profile_build_tree_reusing(doc, None)
        tree.free()
        return prof

    def profile_query_raw(self, text, kind=None, depth=None, max_matches: int = 1 << 20) -> Profile:
        return self._profiled(self.query_raw, text, kind, depth, max_matches)[1]

    def dict_stats(self) -> dict:
        """Work of the last dictionary search: positions walked, trie nodes visited,
        bitmap patterns, sorted-key hits, total hits."""
        out = np.zeros(6, np.uint64)
        check(_lib.load().ol_dict_stats(self._ctx, out.ctypes.data), self._ctx)
        keys = ("text_bytes", "walked", "nodes", "heavy_patterns", "light_hits", "total_hits")
        return {k: int(v) for k, v in zip(keys, out)}
