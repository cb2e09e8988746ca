"""The oracle against the reference's own known answers and differential tests (CPU only)."""
import itertools

import numpy as np
import pytest

import oracle
from oneline_b200 import datagen
from tests.conftest import to_bytes

NONE = 0xFFFFFFFF


def test_scan_line_offsets_known_answers(golden):
    for case in golden["kat"]["scan_line_offsets"]:
        got = oracle.scan_line_offsets(to_bytes(case["text"])).tolist()
        assert got == case["offsets"], case["src"]


def test_parse_line_known_answers(golden):
    for case in golden["kat"]["parse_line"]:
        depth, kind, _, _ = oracle.parse_line(to_bytes(case["line"]), 0)
        assert kind == case["kind"], case["src"]
        if "depth" in case:
            assert depth == case["depth"], case["src"]


def test_parse_document_known_answers(golden):
    for case in golden["kat"]["parse_document"]:
        _, nodes = oracle.parse(to_bytes(case["text"]))
        assert [[int(n["depth"]), int(n["kind"])] for n in nodes] == case["depth_kind"], case["src"]


def test_tree_known_answer(golden):
    for case in golden["kat"]["tree"]:
        nodes = np.zeros(len(case["nodes"]), oracle.NODE_DTYPE)
        for i, (d, k) in enumerate(case["nodes"]):
            nodes[i] = (d, k, 0, 1)
        parent, end = oracle.tree(nodes)
        assert parent.tolist() == case["parent"], case["src"]
        assert end.tolist() == case["subtree_end"], case["src"]
        fc, ns = oracle.tree_children(nodes, parent, end)
        # d 1 2 3 2 (blank) 1 0: line 0 has child 1, 1 has child 2, 1's sibling is 3;
        # the top-level lines 0, 5 and 6 (parent NONE) are siblings of each other
        assert fc.tolist() == [1, 2, NONE, NONE, NONE, NONE, NONE]
        assert ns.tolist() == [5, 3, NONE, NONE, NONE, 6, NONE]


def test_find_all_known_answers(golden):
    for case in golden["kat"]["find_all"]:
        got = oracle.find_all(to_bytes(case["text"]), to_bytes(case["pattern"]))
        if "offsets" in case:
            assert got.tolist() == case["offsets"], case["src"]
        else:
            assert len(got) == case["count"], case["src"]


def test_parse_line_matches_bytewise_oracle_exhaustively():
    """line.rs:165-181: every line of length <= 6 over `| -.:@/\\n`."""
    alphabet = b"| -.:@/\n"
    for n in range(0, 7):
        for combo in itertools.product(alphabet, repeat=n):
            line = bytes(combo)
            assert oracle.parse_line(line, 7) == oracle.parse_line_bytewise(line, 7), line


def test_parse_line_matches_bytewise_oracle_on_random_lines():
    """line.rs:145-162: random lines over a small alphabet (reference seed 4242)."""
    alphabet = b"|| \t=:@->*`0123456789.\r\nxy"
    rng = datagen.Rng(4242)
    for _ in range(60_000):
        n = rng.below(14)
        line = bytes(alphabet[rng.below(len(alphabet))] for _ in range(n))
        start = rng.below(1000)
        assert oracle.parse_line(line, start) == oracle.parse_line_bytewise(line, start), line


def test_edge_cases_are_self_consistent(golden):
    for text in golden["edge_inputs"]["simd_edge_cases"] + golden["edge_inputs"]["gpu_grammar_cases"]:
        t = to_bytes(text)
        offs, nodes = oracle.parse(t)
        assert offs.tolist() == oracle.scan_line_offsets(t).tolist()
        for i, o in enumerate(offs):
            e = int(offs[i + 1]) if i + 1 < len(offs) else len(t)
            assert tuple(int(v) for v in nodes[i]) == oracle.parse_line(t[o:e], int(o))


def test_giant_lines():
    text = b"a" * 100_000 + b"\n|" + b"b" * 300_000
    offs, nodes = oracle.parse(text)
    assert offs.tolist() == [0, 100_001]
    assert tuple(int(v) for v in nodes[1]) == (1, 1, 100_002, 300_000)
    offs, nodes = oracle.parse(b"|" * 1_000_000)
    assert tuple(int(v) for v in nodes[0]) == (1_000_000, 0, 1_000_000, 0)


def test_find_many_matches_per_pattern_find_all(golden):
    """search.rs:291-312: dictionary hits == per-pattern find_all, ordered (pattern, offset)."""
    for key in ("many_nested", "many_whole_text", "many_longer_than_text"):
        case = golden["edge_inputs"][key]
        text = to_bytes(case["text"])
        pats = [to_bytes(p) for p in case["patterns"]]
        counts, hp, ho = oracle.find_many(text, pats)
        at = 0
        for i, p in enumerate(pats):
            want = oracle.find_all(text, p).tolist()
            assert int(counts[i]) == len(want)
            assert hp[at: at + len(want)].tolist() == [i] * len(want)
            assert ho[at: at + len(want)].tolist() == want
            at += len(want)
        assert at == len(hp)


def test_datagen_is_deterministic_and_sized():
    """datagen.rs:255-268."""
    for p in datagen.ALL_PROFILES:
        a = datagen.generate(p, 100_000, 7)
        assert a == datagen.generate(p, 100_000, 7)
        assert len(a) >= 100_000 and a.endswith(b"\n")
    c = datagen.corpus(1 << 20, 0)
    assert c.size == 1 << 20 and c[-1] == ord("\n")
    assert np.array_equal(c, datagen.corpus(1 << 20, 0))


def test_corpus_has_the_stated_shape():
    text = datagen.corpus(4 << 20, 0).tobytes()
    offs, nodes = oracle.parse(text)
    kinds = np.bincount(nodes["kind"], minlength=8) / len(nodes)
    assert 0.04 < kinds[0] < 0.07          # ~5% empty lines
    assert 0.15 < kinds[1] < 0.30          # plain text (30% of non-empty, less markers read as text)
    assert nodes["depth"].max() <= 16
    lens = np.diff(np.append(offs, len(text)))
    assert 40 < lens.mean() < 60


@pytest.mark.parametrize("profile", datagen.ALL_PROFILES)
def test_cpu_baseline_matches_oracle(profile):
    text = datagen.generate(profile, 3 << 20, 41)
    base = oracle.CpuBaseline(threads=4)
    offs, nodes = oracle.parse(text)
    o2, n2 = base.parse_par(text)
    assert np.array_equal(offs, o2) and np.array_equal(nodes, n2)
    tr = oracle.full_tree(nodes)
    got = base.build_links(nodes)
    for k in tr:
        assert np.array_equal(tr[k], got[k]), k
    for pat in [b"|", b"||", b"\n|", b"- ", b"lorem", text[5000:5017]]:
        want = oracle.find_all(text, pat)
        total, got = base.find_all_par(text, pat)
        assert total == len(want) and np.array_equal(got, want), pat


def test_cpu_baseline_dictionary_matches_oracle():
    text = datagen.corpus(2 << 20, 5)
    pats = datagen.patterns_dictionary(text, 5, n=300)
    counts, hp, ho = oracle.find_many(text, pats)
    m = oracle.CpuBaseline(threads=4).many(pats)
    c2, hp2, ho2, total = m.find_all_par(text)
    assert total == len(hp)
    assert np.array_equal(counts, c2) and np.array_equal(hp, hp2) and np.array_equal(ho, ho2)


def test_cpu_baseline_dictionary_digest_matches_the_sorted_hit_list():
    """The order-checking digest (counts + sum of hit_digest over slots), computed
    without building the list, equals the digest of the oracle's sorted list."""
    text = datagen.corpus(1 << 20, 6)
    pats = datagen.patterns_dictionary(text, 6, n=200) + [b"||||", b"||||"]
    counts, hp, ho = oracle.find_many(text, pats)
    m = oracle.CpuBaseline(threads=4).many(pats)
    c2, total, dg = m.digest_par(text)
    assert total == len(hp) and np.array_equal(c2, counts)
    slots = np.arange(len(hp), dtype=np.uint64)
    x = (hp.astype(np.uint64) << np.uint64(32) | ho.astype(np.uint64)) ^ (slots * np.uint64(0x9E3779B97F4A7C15))
    x ^= x >> np.uint64(30)
    x *= np.uint64(0xBF58476D1CE4E5B9)
    x ^= x >> np.uint64(27)
    x *= np.uint64(0x94D049BB133111EB)
    x ^= x >> np.uint64(31)
    assert int(x.sum(dtype=np.uint64)) == dg
    assert oracle.hit_digest(5, int(hp[5]), int(ho[5])) == int(x[5])
    # a swap of two hits changes the digest
    y = np.array([oracle.hit_digest(i, int(hp[i]), int(ho[i])) for i in (0, 1)], np.uint64)
    z = np.array([oracle.hit_digest(i, int(hp[1 - i]), int(ho[1 - i])) for i in (0, 1)], np.uint64)
    assert int(y.sum(dtype=np.uint64)) != int(z.sum(dtype=np.uint64))
