"""Tree links on the GPU vs the oracle: parent, subtree_end, first_child, next_sibling.

Mirrors crates/oneline-gpu/src/tests.rs:452-650, 1065-1125 and the shapes of
crates/oneline-simd/src/links.rs:182-314.
"""
import numpy as np
import pytest

import oracle
from oneline_b200 import OnelineError, TreeLinks
from oneline_b200 import datagen
from tests.conftest import to_bytes

pytestmark = pytest.mark.gpu


def text_from_depths(lines):
    """tests.rs:454-470: one line per (depth, blank); blanks alternate empty and prefix-only."""
    out = []
    for i, (depth, blank) in enumerate(lines):
        s = "|" * depth
        if blank:
            if i % 2 == 0:
                s = ""
        else:
            s += " x"
        out.append(s + "\n")
    return "".join(out).encode()


def assert_tree_matches(parser, text: bytes, what="", strict=True):
    _, nodes = oracle.parse(text)
    want = oracle.full_tree(nodes)
    doc = parser.upload(text)
    tree = parser.build_tree(doc, strict_depth=strict)
    assert tree.line_count() == doc.line_count() == len(nodes)
    got = parser.download_tree(tree)
    for k in ("parent", "subtree_end", "first_child", "next_sibling"):
        if not np.array_equal(got[k], want[k]):
            i = int(np.nonzero(got[k] != want[k])[0][0])
            raise AssertionError(f"{what}: {k} differs at line {i}: gpu {got[k][i]} cpu {want[k][i]}")
    links = parser.download_links(tree)
    assert links == TreeLinks(want["parent"], want["subtree_end"])


def test_known_answer(parser):
    # d 1 2 3 2 (blank) 1 0 (crates/oneline-core/src/links.rs:90-111)
    text = b"| a\n|| b\n||| c\n|| d\n\n| e\nf\n"
    doc = parser.upload(text)
    links = parser.download_links(parser.build_tree(doc))
    N = 0xFFFFFFFF
    assert links.parent.tolist() == [N, 0, 1, 0, N, N, N]
    assert links.subtree_end.tolist() == [5, 3, 3, 5, 5, 6, 7]
    assert links.subtree(0) == range(0, 5) and links.parent_of(3) == 0 and links.parent_of(4) is None


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_generated_documents(parser, profile):
    assert_tree_matches(parser, datagen.generate(profile, 3 << 20, 21), f"profile {profile}")


def test_benchmark_corpus(parser):
    assert_tree_matches(parser, datagen.corpus(16 << 20, 1).tobytes(), "corpus")


def test_run_and_tile_boundaries(parser):
    rng = datagen.Rng(5)
    for n in [1, 2, 15, 16, 17, 31, 32, 33, 255, 256, 257, 1000, 2047, 2048, 2049, 4095, 4096, 4097, 6145,
              8191, 8192, 8193, 12289]:
        lines = [(rng.below(5), rng.chance(15)) for _ in range(n)]
        assert_tree_matches(parser, text_from_depths(lines), f"{n} random lines")


def test_adversarial_shapes(parser):
    n = 4096 * 5 + 77
    shapes = {
        "flat depth 1": [(1, False)] * n,
        "flat depth 0": [(0, False)] * n,
        "header then flat": [(0, False)] + [(1, False)] * (n - 1),
        "flat then header at the end": [(1, False)] * (n - 1) + [(0, False)],
        "strictly increasing to the limit": [(i % 32, False) for i in range(n)],
        "strictly decreasing sawtooth": [(31 - i % 32, False) for i in range(n)],
        "alternating": [(i % 2, False) for i in range(n)],
        "only blanks": [(3, True)] * n,
        "blanks between levels": [(i % 4, i % 3 == 0) for i in range(n)],
        "deepest allowed": [(31, False)] * n,
        "one root far back": [(0, False)] + [(1 + (i % 30), False) for i in range(n)],
    }
    for name, lines in shapes.items():
        assert_tree_matches(parser, text_from_depths(lines), name)


def test_depth_limit_like_the_reference_and_any_depth_when_asked(parser, golden):
    case = golden["kat"]["tree_depth_limit"][0]
    for text in case["ok"]:
        parser.build_tree(parser.upload(to_bytes(text)))
    for text in case["too_deep"]:
        doc = parser.upload(to_bytes(text))
        with pytest.raises(OnelineError) as e:
            parser.build_tree(doc)
        assert "32" in str(e.value)
        # the extension answers instead, and matches the oracle
        assert_tree_matches(parser, to_bytes(text), "too deep, any-depth path", strict=False)
    # still usable after the error
    assert_tree_matches(parser, b"| a\n|| b\n| c\n", "after an error")
    # deep random documents through the any-depth path
    rng = datagen.Rng(77)
    lines = [(rng.below(120), rng.chance(10)) for _ in range(30_000)]
    assert_tree_matches(parser, text_from_depths(lines), "random depths < 120", strict=False)
    lines = [(i % 5000, False) for i in range(20_000)]
    assert_tree_matches(parser, text_from_depths(lines), "staircase to 5000", strict=False)


def test_empty_document(parser):
    doc = parser.upload(b"")
    tree = parser.build_tree(doc)
    assert tree.line_count() == 0
    assert parser.download_links(tree).parent.size == 0


def test_reuse_matches_fresh_builds(parser):
    docs = [datagen.generate(datagen.NESTED, 3 << 20, 1), datagen.generate(datagen.MIXED, 600 << 10, 2),
            datagen.generate(datagen.PROSE, 6 << 20, 3), b"| a\n|| b\n", b"", datagen.generate(datagen.NESTED, 3 << 20, 4)]
    tree = None
    for text in docs:
        doc = parser.upload(text)
        tree = parser.build_tree_reusing(doc, tree)
        _, nodes = oracle.parse(text)
        want = oracle.full_tree(nodes)
        got = parser.download_tree(tree)
        for k in want:
            assert np.array_equal(got[k], want[k]), k
