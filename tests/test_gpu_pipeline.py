"""The parse-then-search pipeline as one CUDA graph: every replay leaves the
same offsets, kinds, tree links and search hits as the oracle."""
import numpy as np
import pytest

import oracle
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu


def test_replays_match_the_oracle(parser):
    import torch

    text = datagen.corpus((6 << 20) + 333, 21).tobytes()
    arr = np.frombuffer(text, np.uint8)
    pats = datagen.patterns_eight(arr, 21) + [b"||||", b"- ", text[-7:]]
    want = [oracle.find_all(text, p) for p in pats]
    offs, nodes = oracle.parse(text)
    tree_want = oracle.full_tree(nodes)
    doc = parser.upload(text)
    tree = parser.build_tree(doc)
    d_tot = torch.zeros(len(pats), dtype=torch.int32, device="cuda")
    outs = [torch.full((max(len(w), 1),), -1, dtype=torch.int32, device="cuda") for w in want]
    pipe = parser.capture_pipeline(doc, tree, pats, [max(len(w), 1) for w in want], d_tot.data_ptr(),
                                   [o.data_ptr() for o in outs])
    assert pipe.kernels >= 10
    for _ in range(3):
        for o in outs:
            o.fill_(-1)
        torch.cuda.synchronize()
        pipe.launch()
        pipe.sync()
        assert d_tot.cpu().numpy().tolist() == [len(w) for w in want]
        for w, o in zip(want, outs):
            assert np.array_equal(o.cpu().numpy().view(np.uint32)[: len(w)], w)
        assert np.array_equal(doc.read_offsets(), offs)
        got = parser.download_tree(tree)
        for k in tree_want:
            assert np.array_equal(got[k], tree_want[k]), k
    pipe.free()
