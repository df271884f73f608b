"""The oracle (C restatement, oracle/oracle.c) against golden vectors produced by the reference's own
code (tests/golden/make_golden.py): Hash64, the posting serializer, the filter grammar and evaluator,
and the ground-truth top-K, including its tie-heavy corpora."""
import numpy as np
import pytest

import oracle


def test_hash64_matches_reference(golden):
    g = golden("hash64.npz")
    got = np.array([oracle.hash64(t) for t in g["tokens"]], np.uint64)
    assert (got == g["hashes"]).all()


def _same_posting(a, b):
    a, b = np.frombuffer(a, np.uint8), np.frombuffer(b, np.uint8)
    if a.size != b.size:
        return False
    layout = a[3] >> 4 if a.size >= 4 else None
    if layout == 3:  # id list: the reference writes unordered_set order, the restatement ascending
        return (a[:8] == b[:8]).all() and sorted(a[8:].view(np.uint32)) == sorted(b[8:].view(np.uint32))
    return (a == b).all()


@pytest.mark.parametrize("packed", [False, True])
def test_posting_serializer_matches_reference(golden, packed):
    g = golden("postings.npz")
    layouts = set()
    for i in range(len(g["seg_docs"])):
        want = bytes(g["packed" if packed else "plain"][i])
        got = oracle.posting_serialize(g["ids"][i], int(g["seg_docs"][i]), bool(g["is_matrix"][i]),
                                       float(g["threshold"][i]), packed)
        assert _same_posting(got, want), i
        layouts.add(want[3] >> 4)
    assert layouts == ({0, 2, 3, 4} if packed else {0, 1, 2, 3})


def test_posting_decode_roundtrip(golden):
    g = golden("postings.npz")
    for i in range(0, len(g["seg_docs"]), 3):
        seg_docs = int(g["seg_docs"][i])
        for blob in (g["plain"][i], g["packed"][i]):
            layout, words = oracle.posting_decode(bytes(blob), seg_docs)
            assert layout >= 0
            ids = np.nonzero(np.unpackbits(words.view(np.uint8), bitorder="little"))[0]
            assert (ids == np.sort(g["ids"][i])).all()


def test_filter_grammar_and_eval_match_reference(golden):
    g = golden("filters.json")
    probes = [np.array(p, np.uint64) for p in g["probes"]]
    for case in g["cases"]:
        assert oracle.parse_ok(case["expr"]) == bool(case["ok"]), case["expr"]
        if case["ok"]:
            got = [oracle.eval_bitmap(case["expr"], p) for p in probes]
            assert got == case["eval"], case["expr"]


def test_ground_truth_topk_matches_reference(golden):
    g = golden("topk.npz")
    for name in g["corpora"]:
        vec, bits, q = g[f"{name}__vectors"], g[f"{name}__bits"], g[f"{name}__queries"]
        topks, filters = g[f"{name}__topks"], list(g[f"{name}__filters"])
        scores, ids, counts = oracle.topk(q, filters, topks, vec, bits, threads=2)
        for i in range(len(q)):
            c = counts[i]
            ref_single = set(g[f"{name}__single_ids"][i][:g[f"{name}__single_counts"][i]].tolist())
            ref_batch = set(g[f"{name}__batch_ids"][i][:g[f"{name}__batch_counts"][i]].tolist())
            assert set(ids[i][:c].tolist()) == ref_single == ref_batch, (name, i)
            # ordered by (score desc, id asc)
            s, d = scores[i][:c], ids[i][:c]
            assert all((s[j] > s[j + 1]) or (s[j] == s[j + 1] and d[j] < d[j + 1]) for j in range(c - 1))


def test_ground_truth_scores_are_sequential_fp32():
    rng = np.random.default_rng(0)
    v = rng.standard_normal((300, 40)).astype(np.float32)
    q = rng.standard_normal((3, 40)).astype(np.float32)
    bits = np.full((300, 1), np.uint64(0xFFFFFFFFFFFFFFFF))
    scores, ids, counts = oracle.topk(q, ["", "", ""], 300, v, bits)
    for i in range(3):
        s = np.zeros(300, np.float32)
        for d in range(40):
            s = (s + (v[:, d] * q[i, d]).astype(np.float32)).astype(np.float32)
        assert (scores[i][:counts[i]] == s[ids[i][:counts[i]]]).all()


def test_postfix_evaluator_rejects_malformed_programs():
    ops = [np.array([1], np.uint64), np.array([2], np.uint64)]
    assert oracle.eval_postfix([1, 2, 0], 1, ops, 1) is not None
    assert oracle.eval_postfix([1, 3, 0], 1, ops, 1) is None      # more postings than given
    assert oracle.eval_postfix([1, 1, 1], 1, ops, 1) is None      # stack underflow
    assert oracle.eval_postfix([3, 1, 1], 1, ops, 1) is None      # NOT with two operands
    assert oracle.eval_postfix([1, 1, 0], 1, ops, 1) is None      # a posting left over
    assert oracle.eval_postfix([0, 2, 1, 1], 1, ops, 1) is not None
    assert oracle.eval_postfix([7, 0, 0], 1, ops, 1) is None      # unknown operator
