"""Dictionary search on the GPU vs the oracle: counts, total and every
(pattern, offset) hit, in (pattern, offset) order, duplicates once per id.

Mirrors crates/oneline-gpu/src/tests.rs:754-907 (assert_many_matches_cpu with
duplicate, nested and colliding patterns) against ManyPatterns semantics
(crates/oneline-simd/src/search.rs:259-312).
"""
import numpy as np
import pytest

import oracle
from oneline_b200 import HIT_DTYPE, OnelineError
from oneline_b200 import datagen
from tests.conftest import to_bytes

pytestmark = pytest.mark.gpu


def want_many(text: bytes, pats, fast=False):
    if fast:
        counts, hp, ho, total = oracle.CpuBaseline(threads=8).many(pats).find_all_par(text)
    else:
        counts, hp, ho = oracle.find_many(text, pats)
        total = len(hp)
    return counts.astype(np.uint64), int(total), hp, ho


def assert_many(parser, text: bytes, pats, max_hits=None, fast=False, what=""):
    counts, total, hp, ho = want_many(text, pats, fast)
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats, max_patterns=None)
    cap = total if max_hits is None else max_hits
    r = parser.search_many(doc, ps, cap)
    assert r.total_hits == total, what
    assert np.array_equal(r.counts.astype(np.uint64), counts), what
    k = min(cap, total)
    assert np.array_equal(r.hits["pattern"], hp[:k]), what
    assert np.array_equal(r.hits["offset"], ho[:k]), what
    return r


def assert_many_device(parser, text: bytes, pats, heavy_min_hits, fast=False, what=""):
    import torch

    counts, total, hp, ho = want_many(text, pats, fast)
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats, max_patterns=None)
    buf = torch.full((2 * max(total, 1),), -1, dtype=torch.int32, device="cuda")
    c, t = parser.search_many_device(doc, ps, buf.data_ptr(), total, heavy_min_hits=heavy_min_hits)
    hits = buf.cpu().numpy().view(HIT_DTYPE)[:total]
    assert t == total and np.array_equal(c.astype(np.uint64), counts), what
    assert np.array_equal(hits["pattern"], hp) and np.array_equal(hits["offset"], ho), what


def test_reference_cases(parser, golden):
    for key in ("many_nested", "many_whole_text", "many_longer_than_text"):
        case = golden["edge_inputs"][key]
        assert_many(parser, to_bytes(case["text"]), [to_bytes(p) for p in case["patterns"]], what=key)


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_generated_documents(parser, profile):
    text = datagen.generate(profile, 2 << 20, 31)
    pats = datagen.patterns_dictionary(np.frombuffer(text, np.uint8), 31, n=400)
    pats += [b"||||", b"||||", b"| | ", b"\n|| ", text[:4], text[-4:], text[-64:], b"\x00\x00\x00\x00"]
    assert_many(parser, text, pats, what=f"profile {profile}")


def test_heavy_bitmaps_and_light_keys_give_the_same_hits(parser):
    """Both ways of collecting hits, and the split between them, leave the result unchanged."""
    text = datagen.corpus(3 << 20, 8).tobytes()
    pats = datagen.patterns_dictionary(np.frombuffer(text, np.uint8), 8, n=500)
    for heavy_min_hits in (1, 50, 1 << 30):
        assert_many_device(parser, text, pats, heavy_min_hits, what=f"heavy >= {heavy_min_hits}")


def test_benchmark_dictionary(parser):
    """10,000 patterns (4..64 B, 60% sampled from the text) on the benchmark generator."""
    text = datagen.corpus(4 << 20, 2).tobytes()
    pats = datagen.patterns_dictionary(np.frombuffer(text, np.uint8), 2, n=10_000)
    r = assert_many(parser, text, pats, fast=True)
    assert r.total_hits > 10 * len(text) // 16
    assert_many(parser, text, pats, max_hits=123_457, fast=True, what="truncated")


def test_tile_edges_text_end_and_duplicates(parser):
    text = bytearray(datagen.corpus(1 << 20, 4).tobytes())
    pats = []
    for edge in (16384, 2 * 16384, 5 * 16384, len(text)):
        for n in (4, 5, 17, 63, 64):
            for back in (0, 1, 3, n - 1, n):
                at = edge - back
                if 0 <= at and at + n <= len(text):
                    pats.append(bytes(text[at: at + n]))
    pats += pats[:7]  # duplicates: each id reports every occurrence
    text[-1:] = b"\x00"
    pats += [bytes(text[-3:]) + b"\x00", b"\x00" * 4]  # would only match the zero padding past the end
    assert_many(parser, bytes(text), pats)


def test_truncation_and_count_only(parser):
    text = datagen.generate(datagen.MIXED, 1 << 20, 6)
    pats = [b"||||", b"| | ", b"lorem", b"ipsum dolor", b"\n|||"]
    r = assert_many(parser, text, pats, max_hits=1000)
    assert len(r.hits) == 1000
    doc = parser.upload(text)
    r0 = parser.search_many(doc, parser.compile_patterns(doc, pats), 0)
    assert r0.hits.size == 0 and r0.total_hits == r.total_hits


def test_limits_errors_and_empty_document(parser):
    doc = parser.upload(b"abcdefgh")
    for bad in ([], [b"abc"], [b"a" * 65], [b"abcd"] * 2049):
        with pytest.raises(OnelineError):
            parser.compile_patterns(doc, bad)
    parser.compile_patterns(doc, [b"abcd"] * 2049, max_patterns=None)
    ps = parser.compile_patterns(doc, [b"abcd", b"efgh"])
    assert len(ps) == 2 and not ps.is_empty()
    r = parser.search_many(doc, ps, 10)
    assert r.counts.tolist() == [1, 1] and r.hits.tolist() == [(0, 0), (1, 4)]
    empty = parser.upload(b"")
    r = parser.search_many(empty, ps, 10)
    assert r.total_hits == 0 and r.counts.tolist() == [0, 0]
    r = parser.search_many(parser.upload(b"abc"), ps, 10)
    assert r.total_hits == 0


@pytest.mark.parametrize("heavy_min_hits", [1, 200, 1 << 30])
def test_runs_of_one_byte(parser, heavy_min_hits):
    """Walks that start inside long runs of one byte jump down the trie path of
    that run: patterns c^4..c^64 (some missing, some duplicated, some longer
    than the run), patterns that continue a run with another byte, runs of
    every length from 1 to 90, and runs cut by the text end. Every hit equals
    the oracle's, with all, some or none of the run patterns heavy."""
    rng = np.random.default_rng(7)
    parts = []
    for n in list(range(1, 91)) * 3:
        c = b"|" if rng.random() < 0.7 else b"-"
        parts.append(c * int(n))
        parts.append(bytes(rng.integers(97, 123, size=int(rng.integers(1, 6)), dtype=np.uint8)))
    text = b"".join(parts) + b"|" * 37
    pats = [b"|" * k for k in range(4, 65) if k % 7 != 3]
    pats += [b"-" * k for k in (4, 5, 8, 13, 21, 34, 55)]
    pats += [b"|" * 9, b"|" * 9]  # duplicated ids
    pats += [b"|" * k + b"a" for k in (3, 4, 6, 10, 20, 40, 63)]
    pats += [b"|" * k + b"-" for k in (4, 12)] + [b"a|||", b"||||a|||"]
    assert_many_device(parser, text, pats, heavy_min_hits, what=f"heavy >= {heavy_min_hits}")
    assert_many(parser, text, pats, what="host hits")


def test_injected_wait_timeout_is_reported_and_leaves_the_context_usable(parser):
    """The dictionary kernel's one bounded wait (its filter's bulk copy), made to
    run out on the host's word (ol_ctx_inject), after the copy has landed: the
    call fails with OL_ERR_TIMEOUT and the next search on the same context and
    document is exact. Nothing on the GPU faults or hangs."""
    from oneline_b200 import _lib

    text = datagen.corpus(1 << 20, 21).tobytes()
    pats = [text[1000:1008], b"||||", b"zzzzzz", text[-20:-4]]
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats)
    L = _lib.load()
    assert L.ol_ctx_inject(parser.ctx, 0xFF) == 1  # unknown flags are refused
    assert L.ol_ctx_inject(parser.ctx, 1) == 0
    with pytest.raises(OnelineError) as ei:
        parser.search_many(doc, ps, 1 << 20)
    assert ei.value.status == 7 and "bounded wait" in str(ei.value), ei.value
    assert_many(parser, text, pats, what="after the injected timeout")


def test_u64_offset_form_equals_the_manyhit_form(parser):
    """The (pattern u32, offset u64) hit form: the same hits as ManyHit, host and
    device arrays, truncated and whole."""
    import torch

    text = datagen.corpus(3 << 20, 22).tobytes()
    pats = datagen.patterns_dictionary(np.frombuffer(text, np.uint8), 22, n=500) + [b"||||", b"||||"]
    counts, hp, ho = oracle.find_many(text, pats)
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats)
    total = len(hp)
    for cap in (total, total // 3):
        c, t, pp, oo = parser.search_many_u64(doc, ps, cap)
        assert t == total and np.array_equal(c.astype(np.uint64), counts)
        assert oo.dtype == np.uint64 and np.array_equal(pp, hp[:cap]) and np.array_equal(oo, ho[:cap].astype(np.uint64))
    d_p = torch.full((total,), -1, dtype=torch.int32, device="cuda")
    d_o = torch.full((total,), -1, dtype=torch.int64, device="cuda")
    c, t = parser.search_many_device_u64(doc, ps, d_p.data_ptr(), d_o.data_ptr(), total, heavy_min_hits=1)
    assert t == total
    assert np.array_equal(d_p.cpu().numpy().view(np.uint32), hp)
    assert np.array_equal(d_o.cpu().numpy().view(np.uint64), ho.astype(np.uint64))
