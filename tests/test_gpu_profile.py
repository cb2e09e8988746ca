"""Profiling through the C ABI (ol_profile_begin / ol_profile_end) and the
GpuParser.profile_* methods it backs, mirroring the reference's Profile
(crates/oneline-gpu/src/timing.rs:109-124) and its profile_* calls
(document.rs:136-157, search.rs:143-173, many.rs:401-410, tree.rs:69-82,
query.rs:275): the results equal the unprofiled calls', every GPU pass has a
device time, gpu_total() is their sum, and host steps are in order."""
import ctypes

import numpy as np
import pytest

import oracle
from oneline_b200 import OnelineError, Profile, _lib
from oneline_b200 import datagen

pytestmark = pytest.mark.gpu


def labels(prof: Profile, which="gpu_passes"):
    return [l for l, _ in getattr(prof, which)]


def check_profile(prof: Profile):
    assert prof.gpu_passes and all(d > 0 for _, d in prof.gpu_passes), prof
    assert prof.gpu_total() == pytest.approx(sum(d for _, d in prof.gpu_passes))
    assert prof.host_steps and all(d >= 0 for _, d in prof.host_steps)
    assert prof.wall >= sum(d for _, d in prof.host_steps) * 0.999


def test_profile_upload_search_tree_and_queries(parser):
    text = datagen.corpus(4 << 20, 31).tobytes()
    doc, prof = parser.profile_upload(text)
    check_profile(prof)
    assert {"upload: copy to device", "parse (overlapped with the upload)"} <= set(labels(prof))
    assert labels(prof, "host_steps")[-1] == "upload: wait for parse"
    offs, nodes = oracle.parse(text)
    assert np.array_equal(doc.read_offsets(), offs)

    pat = text[5000:5012]
    prof = parser.profile_search_document(doc, pat, 64)
    check_profile(prof)
    assert "search" in labels(prof)
    assert parser.search_document(doc, pat, 64).offsets.tolist() == oracle.find_all(text, pat).tolist()[:64]
    check_profile(parser.profile_search_raw(text, b"||", 1 << 20))

    prof = parser.profile_build_tree(doc)
    check_profile(prof)
    assert labels(prof) == ["tree"]
    tree, prof = parser.profile_build_tree_reusing(doc, None)
    assert np.array_equal(parser.download_tree(tree)["parent"], oracle.full_tree(nodes)["parent"])

    for prof in (parser.profile_query_document(doc, kind=2), parser.profile_query_raw(text, kind=3, depth=2)):
        check_profile(prof)
        assert "query" in labels(prof)


def test_profile_search_many_lists_the_dictionary_stages(parser):
    text = datagen.corpus(2 << 20, 32).tobytes()
    pats = datagen.patterns_dictionary(np.frombuffer(text, np.uint8), 32, n=200)
    doc = parser.upload(text)
    ps = parser.compile_patterns(doc, pats)
    counts, hp, ho = oracle.find_many(text, pats)
    prof = parser.profile_search_many(doc, ps, len(hp))
    check_profile(prof)
    assert {"dictionary: sample counts", "dictionary: match", "dictionary: emit", "download"} <= set(labels(prof))
    r = parser.search_many(doc, ps, len(hp))
    assert np.array_equal(r.hits["offset"], ho)


def test_profile_through_the_c_abi(parser):
    """The raw entry points: end without begin is refused and leaves the context
    usable; a profile with no work has no passes; profiling stops at end."""
    L = _lib.load()
    raw = ctypes.create_string_buffer(16 + 8 + 2 * 32 * 48)
    assert L.ol_profile_end(parser.ctx, raw) == 1
    assert L.ol_profile_begin(parser.ctx) == 0
    assert L.ol_profile_end(parser.ctx, raw) == 0
    n_host, n_gpu = np.frombuffer(raw.raw[16:24], np.uint32)
    assert n_host == 0 and n_gpu == 0
    doc = parser.upload(b"| a\n|| b\n")
    with pytest.raises(OnelineError):
        parser._profiled(lambda: parser.search_document(doc, b"", 4))
    assert parser.search_document(doc, b"b", 4).offsets.tolist() == [7]
    assert L.ol_profile_end(parser.ctx, raw) == 1  # the failed call's profile was closed
