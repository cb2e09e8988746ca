"""ol_search_noalloc, the search entry point that allocates nothing, against ol_search.

Some callers cannot call cudaMalloc: a serving process whose own allocator
reserved the GPU's memory up front, or a latency-critical loop that must not
stall the device on cudaMalloc/cudaFree. ol_search_noalloc serves them: it
searches a text the caller already holds on the device and keeps its working
data in one fixed scratch array inside the library. Each test here calls it
through the C ABI two times in a row (with different texts and patterns, so a
result that leaned on what the previous call left in the scratch array would
show) and compares every total and offset, exactly, with ol_search on the same
text and pattern.

This file is collected last, so a run that stops at the first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest

from oneline_b200 import _lib
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu

MAX_TEXT_LEN = 256 << 20  # OL_NOALLOC_MAX_TEXT_LEN
OL_ERR_INVALID_ARG, OL_ERR_INPUT_TOO_LARGE, OL_ERR_BAD_PATTERN = 1, 2, 3


def text_cap(n: int) -> int:
    """OL_NOALLOC_TEXT_CAP(n): whole 16 KiB tiles plus 64 bytes."""
    return (n + 16383) // 16384 * 16384 + 64


def device_text(text: bytes, filler: bytes):
    """The text in a device buffer of text_cap bytes; the bytes past the text
    repeat `filler`, which must never be reported as a match."""
    import torch

    cap = text_cap(len(text))
    host = np.empty(cap, np.uint8)
    host[: len(text)] = np.frombuffer(text, np.uint8)
    pad = (filler * (cap // len(filler) + 1))[: cap - len(text)]
    host[len(text):] = np.frombuffer(pad, np.uint8)
    return torch.from_numpy(host).to("cuda"), cap


def noalloc_search(d_text, n: int, cap: int, pattern: bytes, max_matches: int, ptr_offset: int = 0):
    """One call through the C ABI on torch's current stream; returns (status, total, offsets, message)."""
    import torch

    L = _lib.load()
    d_total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    d_out = torch.full((max(max_matches, 1),), -1, dtype=torch.int32, device="cuda")
    pat = ctypes.create_string_buffer(pattern, max(len(pattern), 1))
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    s = L.ol_search_noalloc(d_text.data_ptr() + ptr_offset, n, cap, pat, len(pattern), max_matches,
                            d_total.data_ptr(), d_out.data_ptr(), stream.cuda_stream, err, len(err))
    if s != 0:
        return s, None, None, err.value.decode()
    stream.synchronize()
    total = int(d_total.cpu().numpy().view(np.uint32)[0])
    k = min(total, max_matches)
    return s, total, d_out[:k].cpu().numpy().view(np.uint32).copy(), ""


def expect(parser, text: bytes, pattern: bytes, max_matches: int):
    """The existing entry point, ol_search on an uploaded document."""
    r = parser.search_document(parser.upload(text), pattern, max_matches)
    return r.total_matches, r.offsets


def check_pair(parser, calls):
    """Runs the calls back to back, then compares each with ol_search."""
    got = []
    for text, pattern, max_matches in calls:
        d_text, cap = device_text(text, pattern)
        s, total, offs, msg = noalloc_search(d_text, len(text), cap, pattern, max_matches)
        assert s == 0, msg
        got.append((total, offs))
    for (text, pattern, max_matches), (total, offs) in zip(calls, got):
        want_total, want_offs = expect(parser, text, pattern, max_matches)
        assert total == want_total, (pattern[:16], total, want_total)
        assert np.array_equal(offs, want_offs), pattern[:16]


def test_two_calls_in_a_row_match_ol_search(parser):
    big = datagen.corpus((6 << 20) + 12_345, 11).tobytes()
    small = datagen.corpus((1 << 20) + 7, 12).tobytes()
    pairs = [
        ((big, b"||", 1 << 21), (small, b"- ", 1 << 20)),
        ((big, big[777_777:777_794], 64), (small, small[-5:], 16)),     # 17 bytes; the text's last bytes
        ((small, small[1000:1064], 8), (big, big[16_380:16_390], 8)),     # 64 bytes; across a tile edge
        ((big, b"|", 100), (big, b"zzzz-absent", 4)),                      # truncated; no match
        ((small, b"\n|", 0), (big, b"\n", 1 << 20)),                       # count only; every line end
    ]
    for first, second in pairs:
        check_pair(parser, [first, second])


def test_largest_text(parser):
    text = datagen.corpus(MAX_TEXT_LEN, 13).tobytes()
    check_pair(parser, [(text, text[-40:], 8), (text, b"|| ", 1 << 22)])


def test_empty_text_and_pattern_longer_than_text(parser):
    import torch

    d_text = torch.zeros(text_cap(3), dtype=torch.uint8, device="cuda")
    for n, pattern in [(0, b"a"), (3, b"abcd")]:
        s, total, offs, msg = noalloc_search(d_text, n, text_cap(n) if n else 0, pattern, 4)
        assert s == 0 and total == 0 and offs.size == 0, msg


def test_refusals_are_clear_and_leave_it_usable(parser):
    import torch

    text = datagen.corpus(1 << 20, 14).tobytes()
    d_text, cap = device_text(text, b"x")
    s, _, _, msg = noalloc_search(d_text, MAX_TEXT_LEN + 1, cap, b"abc", 4)
    assert s == OL_ERR_INPUT_TOO_LARGE and str(MAX_TEXT_LEN) in msg, msg
    s, _, _, msg = noalloc_search(d_text, len(text), cap, b"a" * 65, 4)
    assert s == OL_ERR_BAD_PATTERN and "64" in msg, msg
    s, _, _, msg = noalloc_search(d_text, len(text), cap, b"", 4)
    assert s == OL_ERR_BAD_PATTERN, msg
    s, _, _, msg = noalloc_search(d_text, len(text), cap - 1, b"abc", 4)
    assert s == OL_ERR_INVALID_ARG and str(cap) in msg, msg
    s, _, _, msg = noalloc_search(d_text, len(text) - 64, cap, b"abc", 4, ptr_offset=1)
    assert s == OL_ERR_INVALID_ARG and "16-byte" in msg, msg
    torch.cuda.synchronize()
    check_pair(parser, [(text, b"| ", 1 << 16), (text, text[500:520], 4)])


def test_pinned_pattern_buffer_reused_at_once(parser):
    """The pattern's bytes are taken during the call: a caller that overwrites a
    pinned pattern buffer right after the call returns still gets the results
    of the pattern it passed."""
    import torch

    L = _lib.load()
    text = datagen.corpus((2 << 20) + 99, 15).tobytes()
    d_text, cap = device_text(text, b"#")
    first, second = text[4096:4100], text[70_001:70_013]
    pin = torch.empty(64, dtype=torch.uint8, pin_memory=True)
    stream = torch.cuda.current_stream()
    got = []
    for pattern in (first, second):
        pin.numpy()[: len(pattern)] = np.frombuffer(pattern, np.uint8)
        d_total = torch.zeros(1, dtype=torch.int32, device="cuda")
        d_out = torch.zeros(1 << 16, dtype=torch.int32, device="cuda")
        err = ctypes.create_string_buffer(256)
        s = L.ol_search_noalloc(d_text.data_ptr(), len(text), cap, pin.data_ptr(), len(pattern), 1 << 16,
                                d_total.data_ptr(), d_out.data_ptr(), stream.cuda_stream, err, len(err))
        assert s == 0, err.value.decode()
        pin.numpy()[:] = 0x7E  # overwritten before the GPU has run the search
        stream.synchronize()
        total = int(d_total.cpu().numpy().view(np.uint32)[0])
        got.append((total, d_out[: min(total, 1 << 16)].cpu().numpy().view(np.uint32).copy()))
    for pattern, (total, offs) in zip((first, second), got):
        want_total, want_offs = expect(parser, text, pattern, 1 << 16)
        assert total == want_total and np.array_equal(offs, want_offs), pattern
