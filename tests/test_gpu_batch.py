"""Batches of documents on the GPU: every document's lines, kinds, tree links and
dictionary hits equal the oracle's for that document alone, and no link or hit
crosses a document boundary."""
import numpy as np
import pytest

import oracle
from oneline_b200 import HIT_DTYPE
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu


def make_docs(seed: int, n: int):
    rng = datagen.Rng(seed)
    docs = [b"", b"\n", b"| a", b"||| deep\n|| b\r\n| c\r\n", b"x" * 300, b"|" * 40 + b" y\n" + b"|" * 33 + b"\n",
            b"- item\n\n\n", b"||||"]
    sizes = datagen.lognormal_sizes(seed, n, median=2048, sigma=1.5, lo=0, hi=300_000)
    for i, size in enumerate(sizes):
        d = datagen.generate(datagen.ALL_PROFILES[i % len(datagen.ALL_PROFILES)], int(size), seed + i)[: int(size)]
        if rng.chance(30):
            d = d.rstrip(b"\n")  # no trailing newline
        docs.append(d)
    return docs


def test_lines_kinds_and_trees_per_document(parser):
    docs = make_docs(3, 300)
    b = parser.upload_batch(docs)
    assert len(b) == len(docs)
    parser.build_batch_trees(b)
    for i, d in enumerate(docs):
        offs, nodes = oracle.parse(d)
        start, ln, _, lines = b.doc_info(i)
        assert ln == len(d) and lines == len(offs), i
        got = parser.read_batch_doc(b, i)
        assert np.array_equal(got["offsets"], offs), i
        assert np.array_equal(got["kinds"], nodes["kind"].astype(np.uint8)), i
        want = oracle.full_tree(nodes)
        for k in ("parent", "subtree_end", "first_child", "next_sibling"):
            assert np.array_equal(got[k], want[k]), (i, k)


def test_same_batch_from_packed_buffer(parser):
    docs = make_docs(4, 50)
    data = b"".join(docs)
    offs = np.zeros(len(docs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(d) for d in docs])
    b = parser.upload_batch((data, offs))
    for i, d in enumerate(docs):
        assert np.array_equal(parser.read_batch_doc(b, i, tree=False)["offsets"], oracle.parse(d)[0]), i


@pytest.mark.parametrize("heavy_min_hits", [0, 1])
def test_dictionary_hits_per_document(parser, heavy_min_hits):
    import torch

    docs = make_docs(5, 200)
    corpus = np.frombuffer(b"".join(docs), np.uint8)
    pats = datagen.patterns_dictionary(corpus, 5, n=300)
    # patterns that only occur across a document boundary must not be reported
    for i in range(8, 20):
        if len(docs[i]) >= 3 and len(docs[i + 1]) >= 3:
            pats.append(docs[i][-3:] + docs[i + 1][:3])
    b = parser.upload_batch(docs)
    ps = parser.compile_patterns(None, pats, max_patterns=None)
    want_counts = np.zeros(len(pats), np.uint64)
    per_doc = []
    for d in docs:
        c, hp, ho = oracle.find_many(d, pats)
        want_counts += c.astype(np.uint64)
        per_doc.append((hp, ho))
    total = int(want_counts.sum())
    buf = torch.full((2 * max(total, 1),), -1, dtype=torch.int32, device="cuda")
    counts, t = parser.batch_search_many(b, ps, buf.data_ptr(), total, heavy_min_hits=heavy_min_hits)
    assert t == total and np.array_equal(counts.astype(np.uint64), want_counts)
    hits = buf.cpu().numpy().view(HIT_DTYPE)[:total]
    starts = np.array([b.doc_info(i)[0] for i in range(len(docs))], np.uint64)
    doc_of = np.searchsorted(starts, hits["offset"].astype(np.uint64), side="right") - 1
    # (pattern, document, offset) order
    key = hits["pattern"].astype(np.uint64) << np.uint64(32) | hits["offset"].astype(np.uint64)
    assert np.all(np.diff(key.astype(np.int64)) > 0)
    for i, (hp, ho) in enumerate(per_doc):
        sel = doc_of == i
        assert np.array_equal(hits["pattern"][sel], hp), i
        assert np.array_equal(hits["offset"][sel] - np.uint32(starts[i]), ho), i


def test_same_batch_from_page_locked_buffer(parser):
    """Page-locked input crosses PCIe as it lies and the device lays the
    documents out (separators included): per document the same lines, kinds,
    links and dictionary hits, also when the documents start inside the buffer."""
    import torch

    docs = make_docs(6, 120)
    data = np.frombuffer(b"".join(docs), np.uint8)
    pad = 37
    h = torch.empty(data.size + pad + 5, dtype=torch.uint8, pin_memory=True)
    hv = h.numpy()
    hv[:] = ord("|")
    hv[pad: pad + data.size] = data
    offs = np.zeros(len(docs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(d) for d in docs])
    offs += np.uint64(pad)
    b = parser.upload_batch((hv, offs))
    ref = parser.upload_batch(docs)  # pageable: packed on the host
    assert b.text_len() == ref.text_len()
    parser.build_batch_trees(b)
    for i, d in enumerate(docs):
        offs_i, nodes = oracle.parse(d)
        got = parser.read_batch_doc(b, i)
        assert np.array_equal(got["offsets"], offs_i), i
        assert np.array_equal(got["kinds"], nodes["kind"].astype(np.uint8)), i
        want = oracle.full_tree(nodes)
        for k in ("parent", "subtree_end", "first_child", "next_sibling"):
            assert np.array_equal(got[k], want[k]), (i, k)
    pats = datagen.patterns_dictionary(data, 6, n=200) + [b"\n|||", b"|| \n"]
    ps = parser.compile_patterns(None, pats, max_patterns=None)
    outs = []
    for x in (b, ref):
        counts, total = parser.batch_search_many(x, ps, 0, 0)
        buf = torch.full((2 * max(total, 1),), -1, dtype=torch.int32, device="cuda")
        counts, t = parser.batch_search_many(x, ps, buf.data_ptr(), total)
        assert t == total
        outs.append((counts, buf.cpu().numpy()[: 2 * total]))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
