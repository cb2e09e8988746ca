"""The ``.olb`` binary container of a parsed document, on the host:
``save_to_file`` / ``open_mmap`` as the reference plans them for FlatTree
(.agents/tasks/phase4-zero-copy-binary-serialization.md:13-36). The same layout
is written and read on the GPU side by ``ol_doc_save_olb`` / ``ol_doc_load_olb``.

Layout (little-endian): a 64-byte header -- magic ``ONELINE\\0``, version u32
(1), flags u32, text_len u64, line_count u64, text_offset u64, nodes_offset
u64, line_offsets_offset u64, crc32 u64 -- then the text, ``FlatNode[line_count]``
(16 bytes each) and the u32 line offsets, each section on a 64-byte boundary.
crc32 is the zlib CRC-32 of the file's bytes from text_offset to its end.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

from .core import NODE_DTYPE, FlatTree

MAGIC = b"ONELINE\0"
VERSION = 1
HEADER = struct.Struct("<8sIIQQQQQQ")
assert HEADER.size == 64


def _align64(x: int) -> int:
    return (x + 63) & ~63


def layout(text_len: int, line_count: int) -> tuple[int, int, int, int]:
    """(text_offset, nodes_offset, line_offsets_offset, file length)."""
    text_off = 64
    nodes_off = _align64(text_off + text_len)
    offs_off = _align64(nodes_off + 16 * line_count)
    return text_off, nodes_off, offs_off, offs_off + 4 * line_count


def to_bytes(tree: FlatTree) -> bytes:
    """The ``.olb`` file of a parsed document."""
    text = bytes(tree.source)
    nodes = np.ascontiguousarray(tree.nodes, NODE_DTYPE)
    offs = np.ascontiguousarray(tree.line_offsets, np.uint32)
    n, lines = len(text), nodes.size
    t_off, n_off, o_off, total = layout(n, lines)
    body = bytearray(total - 64)
    body[t_off - 64: t_off - 64 + n] = text
    body[n_off - 64: n_off - 64 + 16 * lines] = nodes.tobytes()
    body[o_off - 64: o_off - 64 + 4 * lines] = offs.tobytes()
    header = HEADER.pack(MAGIC, VERSION, 0, n, lines, t_off, n_off, o_off, zlib.crc32(body))
    return header + bytes(body)


def save_to_file(tree: FlatTree, path: str) -> None:
    with open(path, "wb") as f:
        f.write(to_bytes(tree))


def open_mmap(path: str, verify: bool = False) -> FlatTree:
    """A FlatTree whose text, nodes and offsets are views of the mapped file
    (nothing is copied or parsed). Raises ValueError on a malformed file."""
    m = np.memmap(path, dtype=np.uint8, mode="r")
    if m.size < 64:
        raise ValueError(f"{path}: shorter than the 64-byte .olb header")
    magic, version, _flags, n, lines, t_off, n_off, o_off, crc = HEADER.unpack(bytes(m[:64]))
    if magic != MAGIC:
        raise ValueError(f"{path}: not an .olb file (magic)")
    if version != VERSION:
        raise ValueError(f"{path}: unsupported .olb version {version}")
    if not (64 <= t_off and t_off + n <= n_off and n_off + 16 * lines <= o_off and o_off + 4 * lines <= m.size):
        raise ValueError(f"{path}: sections do not fit the file")
    if verify and zlib.crc32(m[t_off:]) != crc:
        raise ValueError(f"{path}: checksum mismatch")
    nodes = m[n_off: n_off + 16 * lines].view(NODE_DTYPE)
    offsets = m[o_off: o_off + 4 * lines].view(np.uint32)
    return FlatTree(memoryview(m[t_off: t_off + n]), nodes, offsets)
