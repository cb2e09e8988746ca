"""The .olb container on the host (CPU only): the layout of the reference's
plan (.agents/tasks/phase4-zero-copy-binary-serialization.md:13-36), a round
trip through a file with zero-copy views, and refusal of malformed files."""
import struct
import zlib

import numpy as np
import pytest

import oracle
from oneline_b200 import FlatTree, datagen, olb


def tree_of(text: bytes) -> FlatTree:
    offs, nodes = oracle.parse(text)
    return FlatTree(text, nodes, offs)


def test_header_and_sections_follow_the_layout():
    text = datagen.corpus(100_003, 3).tobytes()
    t = tree_of(text)
    raw = olb.to_bytes(t)
    magic, version, flags, n, lines, t_off, n_off, o_off, crc = struct.unpack("<8sIIQQQQQQ", raw[:64])
    assert (magic, version, flags, n, lines) == (b"ONELINE\0", 1, 0, len(text), t.nodes.size)
    assert t_off == 64 and n_off % 64 == 0 and o_off % 64 == 0
    assert n_off >= t_off + n and o_off == (n_off + 16 * lines + 63) // 64 * 64
    assert len(raw) == o_off + 4 * lines and crc == zlib.crc32(raw[64:])
    assert raw[t_off: t_off + n] == text
    assert raw[n_off: n_off + 16 * lines] == t.nodes.tobytes()
    assert raw[o_off:] == t.line_offsets.astype("<u4").tobytes()


def test_round_trip_through_a_mapped_file(tmp_path):
    for text in [b"", b"| a\n|| b\r\n", datagen.corpus(1 << 20, 4).tobytes()]:
        t = tree_of(text)
        path = str(tmp_path / "doc.olb")
        olb.save_to_file(t, path)
        back = olb.open_mmap(path, verify=True)
        assert back == t
        assert isinstance(back.nodes, np.memmap) or back.nodes.size == 0  # a view of the file, not a copy


def test_malformed_files_are_refused(tmp_path):
    raw = bytearray(olb.to_bytes(tree_of(datagen.corpus(20_000, 5).tobytes())))
    cases = {"magic": raw[:1] + b"X" + raw[2:], "version": raw[:8] + b"\x02" + raw[9:], "short": raw[:40],
             "truncated": raw[:-8]}
    flipped = bytearray(raw)
    flipped[100] ^= 1
    for name, data in cases.items():
        p = tmp_path / f"{name}.olb"
        p.write_bytes(bytes(data))
        with pytest.raises(ValueError):
            olb.open_mmap(str(p))
    p = tmp_path / "flipped.olb"
    p.write_bytes(bytes(flipped))
    olb.open_mmap(str(p))  # the checksum is only checked when asked
    with pytest.raises(ValueError, match="checksum"):
        olb.open_mmap(str(p), verify=True)
