"""Types of crates/oneline-core, mirrored for the Python host side.

* ``NodeKind``                crates/oneline-core/src/lib.rs:39-81
* ``NODE_DTYPE`` / FlatNode   crates/oneline-core/src/lib.rs:86-111 (16 bytes, repr(C))
* ``FlatTree``                crates/oneline-core/src/lib.rs:117-158
* ``TreeLinks`` / ``NONE``    crates/oneline-core/src/links.rs:6-50
* ``MAX_INPUT_LEN`` / ``check_input_len``  crates/oneline-core/src/lib.rs:9-36
"""
from __future__ import annotations

import enum
from dataclasses import dataclass

import numpy as np

NONE = 0xFFFFFFFF
MAX_INPUT_LEN = 0xFFFFFFFF

NODE_DTYPE = np.dtype([("depth", "<u4"), ("kind", "<u4"), ("span_start", "<u4"), ("span_len", "<u4")])


class NodeKind(enum.IntEnum):
    Blank = 0
    Text = 1
    Heading = 2
    Element = 3
    List = 4
    Connect = 5
    OrderedList = 6
    Comment = 7
    Unknown = 99

    @classmethod
    def from_u32(cls, v: int) -> "NodeKind":
        try:
            return cls(v)
        except ValueError:
            return cls.Unknown

    def as_str(self) -> str:
        return {
            0: "blank", 1: "text", 2: "heading", 3: "element", 4: "list", 5: "connect",
            6: "ordered-list", 7: "comment", 99: "unknown",
        }[int(self)]


class InputTooLarge(ValueError):
    def __init__(self, length: int):
        super().__init__(f"input is {length} bytes but 32-bit offsets address at most {MAX_INPUT_LEN} bytes")
        self.len = length


def check_input_len(length: int) -> None:
    if length > MAX_INPUT_LEN:
        raise InputTooLarge(length)


@dataclass
class FlatTree:
    """Parse result: the source (not copied), one 16-byte node and one offset per line."""

    source: bytes
    nodes: np.ndarray  # NODE_DTYPE
    line_offsets: np.ndarray  # uint32

    def content_of(self, i: int) -> bytes:
        n = self.nodes[i]
        s = int(n["span_start"])
        return bytes(self.source[s: s + int(n["span_len"])])

    def dump_tree(self) -> str:
        out = []
        for i, n in enumerate(self.nodes):
            text = self.content_of(i).decode("utf-8", "replace").strip()
            out.append(f"{'  ' * int(n['depth'])}[d:{int(n['depth'])} {NodeKind.from_u32(int(n['kind'])).name}] \"{text}\"")
        return "\n".join(out) + ("\n" if out else "")

    def __eq__(self, other) -> bool:
        return (isinstance(other, FlatTree) and bytes(self.source) == bytes(other.source)
                and np.array_equal(self.nodes, other.nodes) and np.array_equal(self.line_offsets, other.line_offsets))


@dataclass
class TreeLinks:
    """parent / subtree_end of every line (blank lines: NONE and i + 1)."""

    parent: np.ndarray
    subtree_end: np.ndarray

    def __len__(self) -> int:
        return int(self.parent.size)

    def is_empty(self) -> bool:
        return self.parent.size == 0

    def parent_of(self, line: int):
        p = int(self.parent[line])
        return None if p == NONE else p

    def subtree(self, line: int) -> range:
        return range(line, int(self.subtree_end[line]))

    def __eq__(self, other) -> bool:
        return (isinstance(other, TreeLinks) and np.array_equal(self.parent, other.parent)
                and np.array_equal(self.subtree_end, other.subtree_end))
