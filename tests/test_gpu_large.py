"""Parity at the benchmark's sizes: the GPU path against the CPU port of the
reference's engine (oracle/cpu_baseline.cpp, itself checked against the oracle
in test_oracle.py) on the benchmark generators' own inputs, element by element.

* 256 MiB of the 1 GiB parse-and-search document (seed 1), with its eight
  patterns (4..1024 B): offsets, kinds, 16-byte nodes, the four tree arrays and
  every hit;
* 64 MiB of the dictionary document (seed 2) against its 10,000 patterns:
  counts and every (pattern, offset) hit in order;
* the whole batched corpus: 10,000 documents (seeds 3..10002, log-normal
  sizes) with the 1,000-pattern dictionary, per document.

These sizes reach what small inputs do not: tens of thousands of tiles, hit
totals in the hundreds of millions, and the dictionary's bitmap path for its
heavy patterns.
"""
import ctypes

import numpy as np
import pytest

import oracle
from oneline_b200 import HIT_DTYPE, _lib
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu

TREE = ("parent", "subtree_end", "first_child", "next_sibling")


def test_parse_tree_and_eight_patterns_256mib(parser):
    import torch

    big = datagen.corpus(1 << 30, 1)
    pats = datagen.patterns_eight(big, 1)  # the 1 GiB document's own patterns
    text = np.ascontiguousarray(big[: 256 << 20])
    del big
    base = oracle.CpuBaseline()
    offs, nodes = base.parse_par(text)
    tree = base.build_links(nodes)
    doc = parser.upload(text)
    assert doc.line_count() == offs.size
    assert np.array_equal(doc.read_offsets(), offs)
    assert np.array_equal(doc.read_kinds(), nodes["kind"].astype(np.uint8))
    assert np.array_equal(doc.read_nodes(), nodes)
    t = parser.download_tree(parser.build_tree(doc))
    for k in TREE:
        assert np.array_equal(t[k], tree[k]), k
    want = [base.find_all_par(text, x)[1] for x in pats]
    assert want[0].size > 20_000_000  # `||||`: dense
    got = parser.search_document_multi(doc, pats, [max(w.size, 1) for w in want])
    for i, (r, w) in enumerate(zip(got, want)):
        assert r.total_matches == w.size and np.array_equal(r.offsets, w), i
    # the device form the benchmark times (ol_search_multi_async: one pass for all eight)
    L = _lib.load()
    outs = [torch.zeros(max(w.size, 1), dtype=torch.int32, device="cuda") for w in want]
    d_tot = torch.zeros(len(pats), dtype=torch.int32, device="cuda")
    bufs = [np.frombuffer(x, np.uint8) for x in pats]
    P = (ctypes.c_void_p * len(pats))(*[x.ctypes.data for x in bufs])
    lens = np.array([len(x) for x in pats], np.uint32)
    maxes = np.array([w.size for w in want], np.uint32)
    O = (ctypes.c_void_p * len(pats))(*[o.data_ptr() for o in outs])
    assert L.ol_search_multi_async(parser.ctx, doc.handle, P, lens.ctypes.data, len(pats), maxes.ctypes.data,
                                   d_tot.data_ptr(), O) == 0
    parser.sync()
    tots = d_tot.cpu().numpy().view(np.uint32)
    for i, (o, w) in enumerate(zip(outs, want)):
        assert tots[i] == w.size and np.array_equal(o[: w.size].cpu().numpy().view(np.uint32), w), i


def test_dictionary_10k_patterns_64mib(parser):
    big = datagen.corpus(1 << 30, 2)
    pats = datagen.patterns_dictionary(big, 2, n=10_000)  # the 1 GiB document's own dictionary
    text = np.ascontiguousarray(big[: 64 << 20])
    del big
    counts, hp, ho, total = oracle.CpuBaseline().many(pats).find_all_par(text)
    assert total > 100_000_000
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats, max_patterns=None)
    r = parser.search_many(doc, ps, total)
    assert r.total_hits == total
    assert np.array_equal(r.counts.astype(np.uint64), counts)
    assert np.array_equal(r.hits["pattern"], hp)
    assert np.array_equal(r.hits["offset"], ho)
    stats = parser.dict_stats()
    assert stats["heavy_patterns"] > 0  # the bitmap path ran


def test_batched_corpus_10k_documents(parser):
    import torch

    n_docs = 10_000
    sizes = datagen.lognormal_sizes(3, n_docs, 16384.0, 1.5, 256, 64 << 20)
    docs = [datagen.corpus(int(sz), 3 + i) for i, sz in enumerate(sizes)]
    dict_text = datagen.corpus(1 << 30, 2)
    pats = datagen.patterns_dictionary(dict_text, 2, n=10_000)[:1000]
    del dict_text
    offs = np.zeros(n_docs + 1, np.uint64)
    offs[1:] = np.cumsum(sizes)
    b = parser.upload_batch((np.concatenate(docs), offs))
    parser.build_batch_trees(b)
    ps = parser.compile_patterns(None, pats, max_patterns=None)
    base = oracle.CpuBaseline()
    many = base.many(pats)
    keys = []
    for i, d in enumerate(docs):
        o, nodes = base.parse_par(d)
        t = base.build_links(nodes)
        start, ln, _, lines = b.doc_info(i)
        assert ln == d.size and lines == o.size, i
        got = parser.read_batch_doc(b, i)
        assert np.array_equal(got["offsets"], o), i
        assert np.array_equal(got["kinds"], nodes["kind"].astype(np.uint8)), i
        for k in TREE:
            assert np.array_equal(got[k], t[k]), (i, k)
        _, hp, ho, _ = many.find_all_par(d)
        keys.append((hp.astype(np.uint64) << np.uint64(32)) | (ho.astype(np.uint64) + np.uint64(start)))
    # (pattern, document, offset) order: the documents' lists, stably by pattern
    want = np.concatenate(keys)
    want = want[np.argsort((want >> np.uint64(32)).astype(np.uint16), kind="stable")]
    total = want.size
    buf = torch.full((2 * max(total, 1),), -1, dtype=torch.int32, device="cuda")
    counts, t = parser.batch_search_many(b, ps, buf.data_ptr(), total)
    assert t == total
    hits = buf.cpu().numpy().view(HIT_DTYPE)[:total]
    got = (hits["pattern"].astype(np.uint64) << np.uint64(32)) | hits["offset"].astype(np.uint64)
    assert np.array_equal(got, want)
    assert np.array_equal(counts.astype(np.int64), np.bincount(hits["pattern"], minlength=len(pats)))
