"""The .olb container on the GPU: a resident document saved with
ol_doc_save_olb is byte for byte the host writer's file for the oracle's parse
of the same text, and ol_doc_load_olb makes a file a resident document without
parsing, equal to the uploaded one (offsets, kinds, nodes, tree, searches).
Malformed files are refused and leave the context usable."""
import numpy as np
import pytest

import oracle
from oneline_b200 import FlatTree, OnelineError, datagen, olb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [0, 1000, (3 << 20) + 17])
def test_save_matches_the_host_writer_and_load_skips_the_parse(parser, tmp_path, size):
    text = datagen.corpus(size, 30).tobytes() if size else b""
    offs, nodes = oracle.parse(text)
    doc = parser.upload(text)
    path = str(tmp_path / "doc.olb")
    parser.save_olb(doc, path)
    assert open(path, "rb").read() == olb.to_bytes(FlatTree(text, nodes, offs))
    loaded = parser.load_olb(path, verify=True)
    assert loaded.line_count() == offs.size and loaded.text_len() == len(text)
    if not size:
        return
    assert np.array_equal(loaded.read_offsets(), offs)
    assert np.array_equal(loaded.read_kinds(), nodes["kind"].astype(np.uint8))
    assert np.array_equal(loaded.read_nodes(), nodes)
    assert loaded.max_depth() == doc.max_depth()
    want = oracle.full_tree(nodes)
    got = parser.download_tree(parser.build_tree(loaded))
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    pat = text[len(text) // 2: len(text) // 2 + 10]
    assert parser.search_document(loaded, pat, 64).offsets.tolist() == oracle.find_all(text, pat).tolist()[:64]


def test_malformed_files_are_refused(parser, tmp_path):
    text = datagen.corpus(50_000, 31).tobytes()
    offs, nodes = oracle.parse(text)
    raw = bytearray(olb.to_bytes(FlatTree(text, nodes, offs)))
    _, _, _, _, lines, _, _, o_off, _ = olb.HEADER.unpack(bytes(raw[:64]))
    bad_offsets = bytearray(raw)
    bad_offsets[o_off + 4 * 5: o_off + 4 * 6] = (10 ** 9).to_bytes(4, "little")  # past the text
    flipped = bytearray(raw)
    flipped[200] ^= 4
    cases = [("magic", raw[:2] + b"?" + raw[3:], False), ("short", raw[:63], False), ("truncated", raw[:-3], False),
             ("offsets", bad_offsets, False), ("checksum", flipped, True)]
    for name, data, verify in cases:
        p = tmp_path / f"{name}.olb"
        p.write_bytes(bytes(data))
        with pytest.raises(OnelineError) as ei:
            parser.load_olb(str(p), verify=verify)
        assert ei.value.status == 1, name
    with pytest.raises(OnelineError):
        parser.load_olb(str(tmp_path / "missing.olb"))
    doc = parser.upload(text)  # the context is still usable
    assert np.array_equal(doc.read_offsets(), offs)
