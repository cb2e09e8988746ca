"""Kernel variants and the autotuner: every variant gives the oracle's results;
the chosen variants are recorded per device and read back."""
import os

import numpy as np
import pytest

import oracle
from oneline_b200 import GpuParser, HIT_DTYPE
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu

VARIANTS = [dict(dict_slice=256, dict_blocks_per_sm=2, dict_heavy_divisor=128, search_staged=0),
            dict(dict_slice=512, dict_blocks_per_sm=0, dict_heavy_divisor=512, search_staged=1),
            dict(dict_slice=1024, dict_blocks_per_sm=3, dict_heavy_divisor=2048, search_staged=1)]


def test_every_variant_gives_the_same_results(parser):
    import torch

    text = datagen.corpus((3 << 20) + 5, 12).tobytes()
    arr = np.frombuffer(text, np.uint8)
    dict_pats = datagen.patterns_dictionary(arr, 12, n=800)
    counts, hp, ho = oracle.find_many(text, dict_pats)
    search_pats = datagen.patterns_eight(arr, 12) + [b"||||", b"- "]
    want = [oracle.find_all(text, p) for p in search_pats]
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, dict_pats, max_patterns=None)
    keep = parser.tuning
    try:
        for v in VARIANTS:
            parser.set_tuning(**v)
            assert parser.tuning == v
            buf = torch.full((2 * max(len(hp), 1),), -1, dtype=torch.int32, device="cuda")
            c, t = parser.search_many_device(doc, ps, buf.data_ptr(), len(hp))
            hits = buf.cpu().numpy().view(HIT_DTYPE)[: len(hp)]
            assert t == len(hp) and np.array_equal(c.astype(np.uint64), counts.astype(np.uint64)), v
            assert np.array_equal(hits["pattern"], hp) and np.array_equal(hits["offset"], ho), v
            res = parser.search_document_multi(doc, search_pats, [max(len(w), 1) for w in want])
            for w, r in zip(want, res):
                assert r.total_matches == len(w) and np.array_equal(r.offsets, w), v
    finally:
        parser.set_tuning(**keep)


def test_autotune_records_and_loads(tmp_path, monkeypatch):
    text = datagen.corpus(8 << 20, 13).tobytes()
    arr = np.frombuffer(text, np.uint8)
    path = str(tmp_path / "tuning.tsv")
    with open(path, "w") as f:
        f.write("Some Other GPU\t99\t256\t1\t128\t0\n")
    p = GpuParser(0)
    try:
        doc = p.upload(text)
        ps = p.compile_patterns(doc, datagen.patterns_dictionary(arr, 13, n=300), max_patterns=None)
        chosen = p.autotune(doc, ps, datagen.patterns_eight(arr, 13), path=path)
        assert p.tuning == chosen
        lines = open(path).read().splitlines()
        assert lines[0].startswith("Some Other GPU") and len(lines) == 2 and lines[1].startswith(p.adapter_name())
    finally:
        p.close()
    q = GpuParser(0)
    try:
        assert q.tuning_load(path) == chosen
    finally:
        q.close()
    monkeypatch.setenv("OL_TUNING_FILE", path)
    r = GpuParser(0)  # a new context reads the file named by the environment
    try:
        assert r.tuning == chosen
    finally:
        r.close()
