"""The serving loop: every result equals the oracle's and is the same when the
request runs alone and when it runs among others; the HBM-budgeted store
evicts idle documents and refuses what cannot fit."""
import numpy as np
import pytest

import oracle
from oneline_b200 import datagen
from oneline_b200.serving import GpuServer, parse_digest, search_digest

pytestmark = pytest.mark.gpu

OL_ERR_ADMISSION, OL_ERR_NOT_FOUND = 6, 9


def workload():
    texts = []
    for i, size in enumerate([1 << 10, 5000, 64 << 10, 300 << 10, 1 << 20, 3 << 20, 777, 2 << 20]):
        texts.append(datagen.generate(datagen.ALL_PROFILES[i % len(datagen.ALL_PROFILES)], size, 50 + i))
    searches = []
    for i, t in enumerate(texts):
        arr = np.frombuffer(t, np.uint8)
        for n in (1, 7, 64):
            searches.append((i, datagen.patterns_dictionary(arr, 60 + i * 3 + n, n=n)))
    return texts, searches


def oracle_digests(texts, searches):
    parse, search = [], []
    for t in texts:
        offs, nodes = oracle.parse(t)
        tr = oracle.full_tree(nodes)
        parse.append(parse_digest(offs, nodes["kind"].astype(np.uint8), tr["parent"], tr["subtree_end"],
                                  tr["first_child"], tr["next_sibling"]))
    for i, pats in searches:
        counts, hp, ho = oracle.find_many(texts[i], pats)
        search.append(search_digest(counts, hp, ho, len(hp)))
    return parse, search


def test_each_result_is_the_same_alone_and_in_the_mix():
    texts, searches = workload()
    want_parse, want_search = oracle_digests(texts, searches)
    with GpuServer(workers=1, store_budget=1 << 30) as alone:
        ap = [alone.wait(alone.submit_parse(t)) for t in texts]
        asr = [alone.wait(alone.submit_search(ap[i].doc_id, pats)) for i, pats in searches]
    with GpuServer(workers=6, store_budget=1 << 30) as mix:
        ids = [mix.submit_parse(t) for t in texts]
        mp = [mix.wait(r) for r in ids]
        # searches interleaved with more parse requests of the same texts
        sids, extra = [], []
        for k, (i, pats) in enumerate(searches):
            sids.append(mix.submit_search(mp[i].doc_id, pats))
            if k % 3 == 0:
                extra.append((k % len(texts), mix.submit_parse(texts[k % len(texts)])))
        ms = [mix.wait(r) for r in sids]
        me = [(i, mix.wait(r)) for i, r in extra]
        assert len({r.worker for r in mp + ms}) > 1  # the work was spread over workers
    for r in ap + asr + mp + ms:
        assert r.status == 0
    assert [r.digest for r in ap] == want_parse == [r.digest for r in mp]
    assert [r.digest for r in asr] == want_search == [r.digest for r in ms]
    for i, r in me:
        assert r.status == 0 and r.digest == want_parse[i]


def test_store_budget_evicts_and_refuses():
    t = datagen.corpus(1 << 20, 9).tobytes()
    big = datagen.corpus(24 << 20, 10).tobytes()
    with GpuServer(workers=2, store_budget=8 << 20) as s:
        docs = [s.wait(s.submit_parse(t)) for _ in range(12)]
        assert all(r.status == 0 for r in docs)
        st = s.stats()
        assert st["evictions"] > 0 and st["resident_bytes"] <= 8 << 20
        gone = s.wait(s.submit_search(docs[0].doc_id, [b"||||"]))
        assert gone.status == OL_ERR_NOT_FOUND
        kept = s.wait(s.submit_search(docs[-1].doc_id, [b"||||"]))
        assert kept.status == 0 and kept.total_hits > 0
        r = s.wait(s.submit_parse(big))
        assert r.status == OL_ERR_ADMISSION and s.stats()["refusals"] == 1


def test_queued_requests_share_launches_and_results_reach_the_caller():
    """Continuous batching: requests queued together are served as one step,
    with fewer kernel launches than the same requests served one at a time,
    and every result (arrays in the caller's buffers, and digests) is the same
    both ways and equal to the oracle's."""
    from oneline_b200 import _lib

    L = _lib.load()
    texts, searches = workload()
    want_parse, want_search = oracle_digests(texts, searches)
    runs = {}
    for coalesce in (False, True):
        with GpuServer(workers=1, store_budget=1 << 30, coalesce=coalesce) as s:
            s.pause()
            l0 = L.ol_launch_count()
            pids = [s.submit_parse(t, results=True) for t in texts]
            s.pause(False)
            parsed = [s.wait(r) for r in pids]
            arrays = [s.results(r, res) for r, res in zip(pids, parsed)]
            l1 = L.ol_launch_count()
            s.pause()
            sids = [s.submit_search(parsed[i].doc_id, pats, results=True) for i, pats in searches]
            # a second request on each document, so searches of one document share a pass
            sids2 = [s.submit_search(parsed[i].doc_id, pats) for i, pats in searches]
            s.pause(False)
            found = [s.wait(r) for r in sids]
            found2 = [s.wait(r) for r in sids2]
            hits = [s.results(r, res) for r, res in zip(sids, found)]
            l2 = L.ol_launch_count()
            runs[coalesce] = dict(parse_launches=l1 - l0, search_launches=l2 - l1, steps=s.steps(),
                                  parsed=parsed, arrays=arrays, found=found, found2=found2, hits=hits)
    plain, batched = runs[False], runs[True]
    n_req = len(texts) + 2 * len(searches)
    assert plain["steps"]["largest_step"] == 1 and plain["steps"]["steps"] == n_req
    assert batched["steps"]["steps"] < n_req and batched["steps"]["largest_step"] > 1
    assert batched["parse_launches"] < len(texts) * 2 < plain["parse_launches"]
    assert batched["search_launches"] < plain["search_launches"] / 4
    for run in (plain, batched):
        assert all(r.status == 0 for r in run["parsed"] + run["found"] + run["found2"])
        assert [r.digest for r in run["parsed"]] == want_parse
        assert [r.digest for r in run["found"]] == want_search == [r.digest for r in run["found2"]]
    for t, a in zip(texts, batched["arrays"]):
        offs, nodes = oracle.parse(t)
        tr = oracle.full_tree(nodes)
        assert np.array_equal(a["offsets"], offs) and np.array_equal(a["kinds"], nodes["kind"].astype(np.uint8))
        for k in ("parent", "subtree_end", "first_child", "next_sibling"):
            assert np.array_equal(a[k], tr[k]), k
    for (i, pats), h in zip(searches, batched["hits"]):
        counts, hp, ho = oracle.find_many(texts[i], pats)
        assert np.array_equal(h["counts"], counts.astype(np.uint32))
        assert np.array_equal(h["hits"]["pattern"], hp) and np.array_equal(h["hits"]["offset"], ho)


def test_admission_is_decided_before_any_work_and_counts_requests_in_flight():
    from oneline_b200 import _lib

    L = _lib.load()
    a = datagen.corpus(4 << 20, 11).tobytes()
    b = datagen.corpus(4 << 20, 12).tobytes()
    huge = datagen.corpus(12 << 20, 13).tobytes()
    with GpuServer(workers=1, store_budget=8 << 20) as s:
        l0 = L.ol_launch_count()
        r = s.wait(s.submit_parse(huge))
        assert r.status == OL_ERR_ADMISSION and L.ol_launch_count() == l0  # refused without a kernel
        # a and b fit one at a time, not together: in one step, b is refused
        # because a's reservation counts although a is not yet in the store
        s.pause()
        ra, rb = s.submit_parse(a), s.submit_parse(b)
        s.pause(False)
        res_a, res_b = s.wait(ra), s.wait(rb)
        assert res_a.status == 0 and res_b.status == OL_ERR_ADMISSION
        assert s.stats()["refusals"] == 2 and s.stats()["resident_bytes"] <= 8 << 20
        # alone, b fits (a, idle, is evicted)
        res_b2 = s.wait(s.submit_parse(b))
        assert res_b2.status == 0 and s.stats()["evictions"] == 1


def test_results_into_reused_caller_buffers():
    """A client that keeps its result buffers: each request writes into the
    arrays it is given (`out=`), and a set reused for the next request holds
    that request's result, equal to the oracle's."""
    from oneline_b200 import HIT_DTYPE
    from oneline_b200.serving import LINK_NAMES

    texts, searches = workload()
    room = max(t.count(b"\n") + 2 for t in texts)
    pset = {"offsets": np.full(room, 7, np.uint32), "kinds": np.full(room, 7, np.uint8),
            **{k: np.full(room, 7, np.uint32) for k in LINK_NAMES}}
    sset = {"counts": np.zeros(64, np.uint32), "hits": np.zeros(1 << 16, HIT_DTYPE)}
    with GpuServer(workers=2, store_budget=1 << 30) as s:
        for t in texts:  # one set, reused request after request
            rid = s.submit_parse(t, out=pset)
            res = s.wait(rid)
            a = s.results(rid, res)
            offs, nodes = oracle.parse(t)
            tr = oracle.full_tree(nodes)
            assert res.status == 0
            assert np.array_equal(a["offsets"], offs) and np.array_equal(a["kinds"], nodes["kind"].astype(np.uint8))
            for k in LINK_NAMES:
                assert np.array_equal(a[k], tr[k]), k
            assert np.shares_memory(a["offsets"], pset["offsets"])
            doc = res.doc_id
            for pats in [p for i, p in searches if texts[i] is t]:
                rid = s.submit_search(doc, pats, out=sset)
                r = s.wait(rid)
                h = s.results(rid, r)
                counts, hp, ho = oracle.find_many(t, pats)
                assert r.status == 0 and np.array_equal(h["counts"], counts.astype(np.uint32))
                k = min(hp.size, sset["hits"].size)
                assert np.array_equal(h["hits"]["pattern"], hp[:k]) and np.array_equal(h["hits"]["offset"], ho[:k])
        with pytest.raises(ValueError):
            s.submit_search(doc, [b"abcd"] * 65, out=sset)  # counts has room for 64 patterns
