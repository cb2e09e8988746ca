"""Substring search on the GPU vs the oracle (every overlapping hit, ascending).

Mirrors crates/oneline-gpu/src/tests.rs:283-448, 655-731.
"""
import numpy as np
import pytest

import oracle
from oneline_b200 import MAX_PATTERN_LEN, OnelineError
from oneline_b200 import datagen
from tests.conftest import to_bytes

pytestmark = pytest.mark.gpu


def assert_search_matches(parser, text: bytes, pattern: bytes, long=False):
    want = oracle.find_all(text, pattern)
    cap = max(len(want), 1)
    kw = {"max_pattern_len": None} if long else {}
    doc = parser.upload(text)
    r = parser.search_document(doc, pattern, cap, **kw)
    assert r.total_matches == len(want), f"resident count for {pattern[:16]!r}"
    assert np.array_equal(r.offsets, want), f"resident offsets for {pattern[:16]!r}"
    r2 = parser.search_raw(text, pattern, cap, **kw)
    assert np.array_equal(r2.offsets, want), f"one-shot offsets for {pattern[:16]!r}"


def test_known_answers(parser, golden):
    for case in golden["kat"]["find_all"]:
        text, pat = to_bytes(case["text"]), to_bytes(case["pattern"])
        r = parser.search_raw(text, pat, 16)
        if "offsets" in case:
            assert r.offsets.tolist() == case["offsets"], case["src"]
        else:
            assert r.total_matches == case["count"], case["src"]


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_generated_documents(parser, profile):
    text = datagen.generate(profile, 3 << 20, 17)
    pats = [p.encode() for p in ["lorem", "SIMD GPU", "naïve", "|", "||", "\n|", "階層 解析", "- ", "zzzz-absent"]]
    for i, n in enumerate([1, 2, 3, 5, 8, 17, 33, 63, 64]):
        at = 1000 + i * 99_991
        pats.append(text[at: at + n])
    for p in pats:
        assert_search_matches(parser, text, p)


def test_alignment_overlap_and_tail(parser, golden):
    for shift in range(8):
        assert_search_matches(parser, b"x" * shift + b"needle" + b"y" * shift + b"needle", b"needle")
    for text, pat in golden["edge_inputs"]["search_cases"] + golden["edge_inputs"]["search_before_text"]:
        assert_search_matches(parser, to_bytes(text), to_bytes(pat))
    text = b"abcq" + b"abc" * 40_000 + b"abcq"
    for p in [b"abcq", b"qabc", b"cabcqabc", b"abcz"]:
        assert_search_matches(parser, text, p)
    assert_search_matches(parser, b"qxyz", b"abcdq")


def test_patterns_across_tile_boundaries_and_long_patterns(parser):
    """Extension: any length (the benchmark uses up to 1024 bytes; > 4096 reads global memory)."""
    text = datagen.corpus(3 << 20, 3).tobytes()
    for n in [4, 8, 16, 32, 64, 65, 128, 255, 256, 1024, 4095, 4096, 4097, 9000]:
        for at in [0, 16384 - n // 2, 3 * 16384 - 1, len(text) - n]:
            assert_search_matches(parser, text, text[at: at + n], long=True)
    with pytest.raises(OnelineError):
        parser.search_raw(text, text[:65], 8)


def test_rejects_bad_patterns_and_stays_usable(parser):
    doc = parser.upload(b"abc")
    with pytest.raises(OnelineError):
        parser.search_document(doc, b"", 8)
    with pytest.raises(OnelineError):
        parser.search_document(doc, b"a" * (MAX_PATTERN_LEN + 1), 8)
    parser.search_document(doc, b"a" * MAX_PATTERN_LEN, 8)
    with pytest.raises(OnelineError):
        parser.search_raw(b"abc", b"", 8)
    assert parser.search_document(doc, b"b", 8).offsets.tolist() == [1]


def test_truncation_reports_the_true_total(parser):
    text = datagen.generate(datagen.MIXED, 2 << 20, 2)
    want = oracle.find_all(text, b"|")
    assert len(want) > 10_000
    doc = parser.upload(text)
    r = parser.search_document(doc, b"|", 100)
    assert r.total_matches == len(want)
    assert np.array_equal(r.offsets, want[:100])  # the lowest 100: a subset, in order
    none = parser.search_document(doc, b"|", 0)
    assert none.total_matches == len(want) and none.offsets.size == 0


def test_empty_document(parser):
    doc = parser.upload(b"")
    assert parser.search_document(doc, b"a", 8).total_matches == 0
    assert parser.search_raw(b"", b"a", 8).total_matches == 0


def test_streaming_upload_places_every_chunk(parser):
    """tests.rs:655-693: 90 MB through the staging ring, twice, plus sizes around the chunk size."""
    record = b"header".ljust(46) + b"MARKER" + b"x".ljust(47) + b"\n"
    assert len(record) == 100
    n = 900_000
    text = record * n + b"end"
    expected = np.arange(n, dtype=np.uint64) * 100 + 46
    for _ in range(2):
        doc = parser.upload(text)
        r = parser.search_document(doc, b"MARKER", n)
        assert r.total_matches == n and np.array_equal(r.offsets, expected.astype(np.uint32))
        assert parser.search_document(doc, b"end", 4).offsets.tolist() == [n * 100]
    chunk = 16 << 20
    for ln in [1, 3, 4, 5, chunk - 1, chunk, chunk + 1, 2 * chunk + 2]:
        t = bytearray(b"." * ln)
        t[0] = ord("A")
        t[-1] = ord("Z")
        doc = parser.upload(bytes(t))
        assert parser.search_document(doc, b"Z", 4).offsets.tolist() == [ln - 1]
        if ln > 1:
            assert parser.search_document(doc, b"A", 4).offsets.tolist() == [0]


def test_multi_pattern_passes_match_single_searches(parser):
    """Up to eight patterns share a pass over the text; each result equals the oracle's."""
    text = datagen.corpus(6 << 20, 7).tobytes()
    arr = np.frombuffer(text, np.uint8)
    pats = datagen.patterns_eight(arr, 7) + [b"|", b"||||", b"- ", b"zzzz-absent", text[100:101], text[5:9],
                                             b"\n", text[16383:16383 + 2000], b"x" * 5000]
    doc = parser.upload(text)
    want = [oracle.find_all(text, p) for p in pats]
    res = parser.search_document_multi(doc, pats, [max(len(w), 1) for w in want])
    for p, w, r in zip(pats, want, res):
        assert r.total_matches == len(w) and np.array_equal(r.offsets, w), p[:16]
    # truncation per pattern keeps the lowest offsets and the true totals
    res = parser.search_document_multi(doc, pats[:8], 3)
    for w, r in zip(want[:8], res):
        assert r.total_matches == len(w) and np.array_equal(r.offsets, w[:3])


def test_planted_occurrences_at_every_offset_around_tile_edges(parser):
    """Occurrences of 5..33-byte patterns planted at every offset from 20
    bytes before to 20 bytes after a 16 KiB tile edge, searched alone and in
    eight-pattern passes that mix every filter (whole-pattern compare up to 4
    bytes, two-byte filter for 5-7, anchor words from 8), including patterns
    that share anchor words."""
    rng = np.random.default_rng(41)
    tile = 16384
    for m in [5, 6, 7, 8, 9, 11, 12, 16, 33]:
        base = rng.integers(33, 127, size=m, dtype=np.uint8).tobytes()
        n_edges = 41
        text = bytearray(rng.integers(33, 127, size=(n_edges + 1) * tile + 777, dtype=np.uint8).tobytes())
        for t, d in enumerate(range(-20, 21), start=1):
            at = t * tile + d
            text[at: at + m] = base
        text[len(text) - m:] = base  # one ending exactly at the end of the text
        text = bytes(text)
        pats = [base, base[1:] + b"~", base[:-1], base[2:], base[:4], base[:5], base[:6], base[:1]]
        doc = parser.upload(text)
        want = [oracle.find_all(text, p) for p in pats]
        assert len(want[0]) == n_edges + 1
        res = parser.search_document_multi(doc, pats, [max(len(w), 1) for w in want])
        for p, w, r in zip(pats, want, res):
            assert r.total_matches == len(w) and np.array_equal(r.offsets, w), (m, p)
        for p, w in zip(pats[:4], want[:4]):
            r = parser.search_document(doc, p, max(len(w), 1), max_pattern_len=None)
            assert r.total_matches == len(w) and np.array_equal(r.offsets, w), (m, p)


def test_patterns_ending_in_nul_do_not_match_the_padding(parser):
    for text, pats in [(b"x" * 40_000 + b"abc", [b"abc\0", b"abc\0\0\0\0", b"bc\0\0\0\0\0\0\0", b"c\0"]),
                       (b"y" * 16_381 + b"abcd\0", [b"abcd\0\0\0\0", b"d\0\0", b"abcd\0"])]:
        doc = parser.upload(text)
        want = [oracle.find_all(text, p) for p in pats]
        res = parser.search_document_multi(doc, pats, 4)
        for p, w, r in zip(pats, want, res):
            assert r.total_matches == len(w) and np.array_equal(r.offsets, w), p


def test_tiles_whose_hits_overflow_the_staging_slot(parser):
    """A tile with more hits than its staging slot holds (8192 for all the
    patterns of a pass) is recomputed in place; the others are copied from
    their slots. Dense runs of one byte put 16,384 hits in a tile."""
    rng = np.random.default_rng(3)
    parts = []
    for i in range(12):
        parts.append(b"a" * int(rng.integers(10_000, 40_000)))
        parts.append(bytes(rng.integers(98, 123, size=int(rng.integers(1_000, 30_000)), dtype=np.uint8)))
    text = b"".join(parts)
    pats = [b"a", b"aa", b"aaaa", b"aaaaaaaaa", b"ab", b"b", b"zz", b"a" * 40]
    doc = parser.upload(text)
    want = [oracle.find_all(text, p) for p in pats]
    for group in (pats[:1], pats[:3], pats):
        res = parser.search_document_multi(doc, group, [len(w) for w in want[:len(group)]])
        for p, w, r in zip(group, want, res):
            assert r.total_matches == len(w) and np.array_equal(r.offsets, w), (len(group), p)
    res = parser.search_document_multi(doc, pats, 1000)  # truncated: the lowest 1000 of each
    for p, w, r in zip(pats, want, res):
        assert r.total_matches == len(w) and np.array_equal(r.offsets, w[:1000]), p
