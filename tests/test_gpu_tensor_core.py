"""The tensor-core candidate pass (tcgen05 + TMA + TMEM) in its three formats -- TF32 over the FP32
rows, a BF16 copy, an FP8 E4M3 copy with per-vector scales -- through the C-ABI.

1. The approximate pass itself: every emitted candidate passes the filter and its approximate score is
   within the query's proven bound eps of the exact FP32 score, and every filtered doc whose exact
   score reaches theta + eps was emitted (nothing the top K could need is missing).
2. End to end: ids bit-exact and in order, scores bit-exact, against the oracle (tolerance 0)."""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import data

pytestmark = pytest.mark.gpu

METHODS = {"tf32": 1, "bf16": 2, "e4m3": 3}


def _seq_scores(q, v):
    s = np.zeros(v.shape[0], np.float32)
    for d in range(v.shape[1]):
        s = (s + (v[:, d] * q[d]).astype(np.float32)).astype(np.float32)
    return s


def _corpus(n=24000, tags=64, seed=31, p=8192):
    mix = data.Mixture(128, tags, (1e-3, 0.5), n_clusters=64, seed=seed)
    vec, bits, _ = mix.corpus(n, seed=seed + 1)
    return mix, vec, bits


@pytest.mark.parametrize("method", list(METHODS))
@pytest.mark.parametrize("nq", [40, 200])
def test_approximate_pass_respects_its_bound(torch_cuda, method, nq):
    mix, vec, bits = _corpus()
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=8192)
    q = mix.queries(nq, seed=32)
    exprs = data.make_filters(mix, nq, n_tags=(1, 3), seed=33)
    exprs[0] = ""
    s = hss.FullRecallSearcher(table, max_batch=256, method=METHODS[method])
    for a, e in zip(q, exprs):
        s.add_query(e, a, 50)
    scores, ids, counts = s.batch_search()
    want = oracle.topk(q, exprs, 50, vec, bits, threads=8)
    for i in range(0, nq, max(1, nq // 12)):
        sc, loc, n, theta, eps = s.last_candidates(i)
        assert n == len(sc), "candidate list overflowed in a small test"
        assert eps > 0 and eps < 0.2
        passing = np.nonzero(np.unpackbits(oracle.filter_bits(exprs[i], bits).view(np.uint8),
                                           bitorder="little")[:vec.shape[0]])[0]
        exact = _seq_scores(q[i], vec[passing])
        ex_of = dict(zip(passing.tolist(), exact.tolist()))
        for a, l in zip(sc, loc):
            assert int(l) in ex_of, "a candidate that fails the filter"
            assert abs(float(a) - ex_of[int(l)]) <= eps, (method, i, float(a), ex_of[int(l)], eps)
        need = set(passing[exact >= theta + eps].tolist())
        assert need <= set(loc.tolist()), (method, i, len(need - set(loc.tolist())))
        c = int(want[2][i])
        assert (ids[i][:c] == want[1][i][:c]).all()
        assert (scores[i][:c].view(np.uint32) == want[0][i][:c].view(np.uint32)).all()


@pytest.mark.parametrize("nq", [96, 256], ids=["one_sm", "sm_pair"])
@pytest.mark.parametrize("method", list(METHODS))
def test_tensor_core_search_is_exact_mixed_k(torch_cuda, method, nq):
    # 40000 docs = 313 tiles of 128: the SM-pair pass (more than 128 queries) ends on a half tile
    mix = data.Mixture(128, 128, (1e-3, 0.6), n_clusters=128, seed=41)
    vec, bits, _ = mix.corpus(40000, seed=42)
    table = hss.DataTable.build(vec, bits, 128, device=0, doc_num_per_segment=16384, sparse_packed=True)
    q = mix.queries(nq, seed=43)
    exprs = data.make_filters(mix, nq, n_tags=(1, 6), seed=44, selectivity_range=(1e-4, 1.0))
    topks = np.array([1, 10, 100, 1000] * (nq // 4))
    s = hss.FullRecallSearcher(table, max_batch=nq, method=METHODS[method])
    for a, e, k in zip(q, exprs, topks):
        s.add_query(e, a, int(k))
    scores, ids, counts = s.batch_search()
    ws, wi, wc = oracle.topk(q, exprs, topks, vec, bits, threads=8)
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c
        assert (ids[i][:c] == wi[i][:c]).all(), (method, i)
        assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), (method, i)


@pytest.mark.parametrize("nq", [24, 160], ids=["one_sm", "sm_pair"])
@pytest.mark.parametrize("method", list(METHODS))
def test_tensor_core_overflow_reruns_are_exact(torch_cuda, method, nq):
    mix = data.Mixture(128, 32, (0.3, 0.9), n_clusters=8, seed=51)
    vec, bits, _ = mix.corpus(50000, seed=52)
    table = hss.DataTable.build(vec, bits, 32, device=0, doc_num_per_segment=8192)
    q = mix.queries(nq, seed=53)
    exprs = [""] * (nq // 2) + ["1 OR 2"] * (nq - nq // 2)
    s = hss.FullRecallSearcher(table, max_batch=nq, candidate_cap=4096, sample_docs=4096, method=METHODS[method])
    for a, e in zip(q, exprs):
        s.add_query(e, a, 3000)
    scores, ids, counts = s.batch_search()
    ws, wi, wc = oracle.topk(q, exprs, 3000, vec, bits, threads=8)
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c
        assert (ids[i][:c] == wi[i][:c]).all(), (method, i)
        assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), (method, i)


@pytest.mark.parametrize("nq", [64, 256], ids=["few_queries", "sm_pair"])
@pytest.mark.parametrize("method", list(METHODS))
def test_long_vectors_are_exact(torch_cuda, method, nq):
    # 768-dim vectors (the precision-form configuration's width): the query tile no longer fits next
    # to a deep stage ring for TF32 (24 k-blocks) and BF16 (12), so those passes stream each query
    # k-block with the doc k-block through the ring on SM pairs, also for a batch of 64; E4M3 (6
    # k-blocks) keeps its queries resident
    mix = data.Mixture(768, 64, (1e-3, 0.6), n_clusters=32, seed=61)
    vec, bits, _ = mix.corpus(30000, seed=62)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=8192)
    q = mix.queries(nq, seed=63)
    exprs = data.make_filters(mix, nq, n_tags=(1, 4), seed=64, selectivity_range=(1e-3, 1.0))
    topks = np.array([1, 10, 100, 500] * (nq // 4))
    s = hss.FullRecallSearcher(table, max_batch=nq, method=METHODS[method])
    for a, e, k in zip(q, exprs, topks):
        s.add_query(e, a, int(k))
    scores, ids, counts = s.batch_search()
    ws, wi, wc = oracle.topk(q, exprs, topks, vec, bits, threads=8)
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c, (method, i)
        assert (ids[i][:c] == wi[i][:c]).all(), (method, i)
        assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), (method, i)


def test_pipeline_wait_runs_out_and_the_searcher_recovers(torch_cuda):
    # The single-SM pass's producer stops before its first corpus stage, so every CTA's MMA issuer
    # waits for a stage that never comes until its bounded wait (about 1 ms of clock here) runs out:
    # the pass records its error bit, drains, frees its tensor memory and returns; the batch reports
    # the error and the same searcher's next batch is exact. Nothing faults: each wait ends by its own
    # budget.
    mix, vec, bits = _corpus()
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=8192)
    nq = 40
    q = mix.queries(nq, seed=71)
    exprs = data.make_filters(mix, nq, n_tags=(1, 3), seed=72)
    s = hss.FullRecallSearcher(table, max_batch=64, method=METHODS["bf16"])
    s.set_pipeline_test(1, 2_000_000)
    for a, e in zip(q, exprs):
        s.add_query(e, a, 50)
    with pytest.raises(hss.HssError) as err:
        s.batch_search()
    assert err.value.code == hss._lib.HSS_ERR_CUDA and "timed out" in str(err.value)
    for a, e in zip(q, exprs):
        s.add_query(e, a, 50)
    scores, ids, counts = s.batch_search()
    ws, wi, wc = oracle.topk(q, exprs, 50, vec, bits, threads=8)
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c
        assert (ids[i][:c] == wi[i][:c]).all() and (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all()
