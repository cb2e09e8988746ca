"""Node queries on the GPU vs the oracle: the lines whose kind and depth match.

Mirrors crates/oneline-gpu/src/tests.rs:86-107 (query_raw) and the filter
semantics of shader.wgsl:152-160 (kind 0 = any, depth 0xFFFFFFFF = any).
"""
import numpy as np
import pytest

import oracle
from oneline_b200 import NodeKind, OnelineError
from oneline_b200 import datagen
from tests.conftest import to_bytes

pytestmark = pytest.mark.gpu


def want(nodes, kind, depth, lo=0, hi=None):
    hi = len(nodes) if hi is None else hi
    m = np.ones(len(nodes), bool)
    if kind:
        m &= nodes["kind"] == kind
    if depth is not None:
        m &= nodes["depth"] == depth
    idx = np.nonzero(m)[0]
    return idx[(idx >= lo) & (idx < hi)].astype(np.uint32)


def test_known_answer(parser, golden):
    case = golden["kat"]["query_raw"][0]
    text = to_bytes(case["text"])
    assert parser.query_raw(text, NodeKind.Element).tolist() == case["kind_element"]
    assert parser.query_raw(text, None, 2).tolist() == case["depth_2"]
    offs, _ = oracle.parse(text)
    assert parser.query(text, offs, NodeKind.Element).tolist() == case["kind_element"]


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_generated_documents(parser, profile):
    text = datagen.generate(profile, 2 << 20, 9)
    offs, nodes = oracle.parse(text)
    doc = parser.upload(text)
    for kind in range(8):
        for depth in (None, 0, 1, 2, 3, 7, 16):
            r = parser.query_document(doc, kind, depth, len(nodes))
            w = want(nodes, kind, depth)
            assert r.total_matches == len(w) and np.array_equal(r.indices, w), (kind, depth)
    assert np.array_equal(parser.query(text, offs, NodeKind.Text, 1), want(nodes, 1, 1))
    assert np.array_equal(parser.query_raw(text, NodeKind.List, None), want(nodes, 4, None))


def test_subtrees(parser):
    text = datagen.corpus(2 << 20, 3).tobytes()
    offs, nodes = oracle.parse(text)
    tree = oracle.full_tree(nodes)
    doc = parser.upload(text)
    gtree = parser.build_tree(doc)
    rng = datagen.Rng(3)
    for _ in range(40):
        root = rng.below(len(nodes))
        for kind, depth in ((0, None), (1, None), (3, int(nodes["depth"][root]) + 1)):
            r = parser.query_subtree(doc, gtree, root, kind, depth, 1 << 20)
            w = want(nodes, kind, depth, root, int(tree["subtree_end"][root]))
            assert r.total_matches == len(w) and np.array_equal(r.indices, w), (root, kind, depth)
    with pytest.raises(OnelineError):
        parser.query_subtree(doc, gtree, len(nodes), 0, None, 8)


def test_truncation_deep_lines_and_empty(parser):
    text = datagen.corpus(1 << 20, 5).tobytes()
    _, nodes = oracle.parse(text)
    doc = parser.upload(text)
    r = parser.query_document(doc, 0, None, 1000)
    assert r.total_matches == len(nodes) and r.indices.tolist() == list(range(1000))
    deep = b"".join(b"|" * d + b" x\n" for d in list(range(0, 300)) + [270, 255, 254, 1000])
    _, dn = oracle.parse(deep)
    ddoc = parser.upload(deep)
    for depth in (0, 254, 255, 256, 270, 299, 1000, 1001):
        assert np.array_equal(parser.query_document(ddoc, NodeKind.Text, depth).indices, want(dn, 1, depth)), depth
    assert parser.query_document(parser.upload(b""), 0, None, 8).total_matches == 0
    assert parser.query_raw(b"", 0, None).size == 0
