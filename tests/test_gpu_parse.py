"""Parse (newline scan + classification) on the GPU vs the oracle, bit for bit.

Mirrors crates/oneline-gpu/src/tests.rs:27-183, 255-271 and the CPU edge cases
of crates/oneline-simd/src/lib.rs:578-642.
"""
import numpy as np
import pytest

import oracle
from oneline_b200 import NODE_DTYPE, NodeKind, OnelineError
from oneline_b200 import datagen
from tests.conftest import to_bytes

pytestmark = pytest.mark.gpu


def assert_parse_matches(parser, text: bytes, what=""):
    offs, nodes = oracle.parse(text)
    tree = parser.parse_raw(text)
    assert np.array_equal(tree.line_offsets, offs), f"{what}: offsets"
    assert np.array_equal(tree.nodes, nodes), f"{what}: nodes"
    doc = parser.upload(text)
    assert doc.line_count() == len(offs) and doc.text_len() == len(text)
    assert np.array_equal(doc.read_offsets(), offs), f"{what}: resident offsets"
    assert np.array_equal(doc.read_kinds(), nodes["kind"].astype(np.uint8)), f"{what}: resident kinds"
    assert np.array_equal(doc.read_nodes(), nodes), f"{what}: resident nodes"


def test_known_answers(parser, golden):
    for case in golden["kat"]["scan_line_offsets"]:
        assert parser.scan_line_offsets(to_bytes(case["text"])).tolist() == case["offsets"], case["src"]
    for case in golden["kat"]["parse_document"]:
        tree = parser.parse_raw(to_bytes(case["text"]))
        assert [[int(n["depth"]), int(n["kind"])] for n in tree.nodes] == case["depth_kind"], case["src"]
    tree = parser.parse_raw(b"|=[ Header ]\n| Body text\n||:rule(x)\n|| Content.\n")
    assert NodeKind(int(tree.nodes[0]["kind"])) == NodeKind.Heading and int(tree.nodes[3]["depth"]) == 2


def test_grammar_and_edge_cases(parser, golden):
    ins = golden["edge_inputs"]
    for text in ins["simd_edge_cases"] + ins["gpu_grammar_cases"] + ins["gpu_scan_cases"]:
        assert_parse_matches(parser, to_bytes(text), repr(text))


def test_every_short_line_over_a_small_alphabet(parser):
    """All lines of length <= 5 over `| -.:@/\\r` (line.rs:165-181), as one document."""
    import itertools

    lines = [bytes(c) for n in range(6) for c in itertools.product(b"| -.:@/\r", repeat=n)]
    text = b"\n".join(lines) + b"\n"
    assert_parse_matches(parser, text, "short lines")


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_generated_profiles(parser, profile):
    text = datagen.generate(profile, 3 << 20, 11)
    assert_parse_matches(parser, text, f"profile {profile}")


def test_benchmark_corpus(parser):
    assert_parse_matches(parser, datagen.corpus(8 << 20, 0).tobytes(), "corpus")


def test_many_tiles_and_awkward_shapes(parser):
    """> 512 tiles (tests.rs:173-183) and the awkward shapes of lib.rs:618-642."""
    assert_parse_matches(parser, datagen.generate(datagen.MIXED, 9 << 20, 3), "9 MiB mixed")
    for case in [b"a" * 100_000 + b"\n|" + b"b" * 300_000, b"x\r\n" * 300_000, b"\n" * 400_000,
                 b"|" * 1_000_000, b"line\n" * 200_000 + b"tail without newline",
                 b"| " + b"\r" * 70_000 + b"\n| x\n", b"||| \t" * 20_000 + b"- y\n"]:
        assert_parse_matches(parser, case, repr(case[:20]))


def test_tiles_with_more_lines_than_a_slot(parser):
    """Tiles of up to 1024 lines are staged and copied; denser tiles (short or
    empty lines) are parsed again once their first line index is known. Both
    kinds side by side, the dense runs starting and ending at every offset
    around a tile edge."""
    corpus = datagen.corpus(1 << 20, 5).tobytes()
    for cut in [16384 - 3, 16384, 16384 + 1, 3 * 16384 + 7]:
        dense = b"\n" * 5000 + b"|\n" * 3000 + b"| -\n" * 2000
        text = corpus[:cut] + dense + corpus[cut: cut + 100_000] + dense + corpus[:50_000] + b"|" * 17
        assert_parse_matches(parser, text, f"dense at {cut}")


def test_lines_across_tile_and_halo_boundaries(parser):
    """Line ends and prefixes at every distance around the 16 KiB tile and its 256-byte halo."""
    tile = 16384
    for cut in [tile - 2, tile - 1, tile, tile + 1, tile + 255, tile + 256, tile + 257, 2 * tile - 1]:
        head = b"x" * (cut - 1) + b"\n"
        for tail in [b"|| - a\n", b"|" * 300 + b" b\n", b"\r\r\n", b"-. c", b"\n\n"]:
            assert_parse_matches(parser, head + tail + b"| z\n", f"cut {cut} tail {tail[:8]!r}")


def test_empty_and_oversized(parser):
    assert parser.scan_line_offsets(b"").size == 0
    assert parser.parse_raw(b"").nodes.size == 0
    doc = parser.upload(b"")
    assert doc.line_count() == 0 and doc.text_len() == 0
    from oneline_b200.gpu import _check_len, MAX_GPU_INPUT_LEN

    _check_len(MAX_GPU_INPUT_LEN)
    with pytest.raises(OnelineError):
        _check_len(MAX_GPU_INPUT_LEN + 1)


def test_parse_with_given_offsets(parser):
    text = b"|=[ Header ]\n| Body text\n||:rule(x)\n|| Content.\n"
    offs = oracle.scan_line_offsets(text)
    tree = parser.parse(text, offs)
    _, nodes = oracle.parse(text)
    assert np.array_equal(tree.nodes, nodes)
    assert parser.parse(text, np.zeros(0, np.uint32)).nodes.size == 0


def test_reparse_into_the_same_buffers(parser):
    from oneline_b200 import _lib

    text = datagen.corpus(2 << 20, 9).tobytes()
    doc = parser.upload(text)
    before = doc.read_nodes()
    for _ in range(3):
        assert _lib.load().ol_doc_reparse_async(parser.ctx, doc.handle) == 0
    parser.sync()
    assert np.array_equal(doc.read_nodes(), before)
    assert np.array_equal(doc.read_offsets(), oracle.scan_line_offsets(text))


@pytest.mark.parametrize("pinned", [False, True])
def test_upload_overlapped_with_the_parse_across_chunks(parser, pinned):
    """The upload streams the text in chunks (16 MiB ring slots for pageable
    memory, 32 MiB copies for pinned) and the parse runs on each chunk's tiles
    as they land: lines and long lines that straddle chunk edges, and a text
    that ends right after a chunk edge, parse as they do in one piece."""
    import torch

    base = datagen.corpus((70 << 20) + 5, 23).tobytes()
    long_line = b"|| - " + b"x" * 70_000 + b"\n"
    edge = 16 << 20
    text = base[: edge - 30_000] + long_line + base[edge - 30_000: 3 * (32 << 20) + 7]
    for t in (text, text[: 2 * (16 << 20) + 1]):
        want_offs, want_nodes = oracle.CpuBaseline().parse_par(t)
        src = t
        if pinned:
            h = torch.empty(len(t), dtype=torch.uint8, pin_memory=True)
            h.numpy()[:] = np.frombuffer(t, np.uint8)
            src = h.numpy()
        doc = parser.upload(src)
        assert np.array_equal(doc.read_offsets(), want_offs)
        assert np.array_equal(doc.read_nodes(), want_nodes)
