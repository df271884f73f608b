"""End-to-end parity of the searcher on the GPU, through the C-ABI: every query's doc ids must equal
the oracle's ground truth bit for bit and in order (score descending, doc id ascending), and every
returned score must equal the ground truth's FP32 score bit for bit (tolerance 0; the path's
specification allows 1e-5 relative). Covers one and many segments, all posting layouts, tie-heavy corpora, K above the hit
count, the K limits, empty and match-nothing filters, candidate-list overflow re-runs, a doc-id offset,
the device-resident API and a saved / reloaded index."""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import _lib, data

pytestmark = pytest.mark.gpu


def _check(res, want, nq, offset=0, exact_scores=True):
    scores, ids, counts = res
    ws, wi, wc = want
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c, (i, counts[i], c)
        assert (ids[i][:c] == wi[i][:c] + offset).all(), i
        if exact_scores:
            assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), i


def _run(table, vec, bits, queries, exprs, topks, offset=0, **scfg):
    s = hss.FullRecallSearcher(table, **scfg)
    for q, e, k in zip(queries, exprs, topks):
        s.add_query(e, q, int(k))
    res = s.batch_search()
    want = oracle.topk(queries, exprs, topks, vec, bits, threads=8)
    _check(res, want, len(queries), offset)
    return s, res


def test_cfg1_single_segment_top100(torch_cuda):
    cfg = data.CONFIGS["cfg1"]
    mix = data.Mixture(cfg["dim"], cfg["tag_num"], cfg["p_range"], seed=1)
    vec, bits, _ = mix.corpus(cfg["n"], seed=11)
    table = hss.DataTable.build(vec, bits, cfg["tag_num"], device=0, doc_num_per_segment=131072)
    nq = 64
    q = mix.queries(nq, seed=2)
    exprs = data.make_filters(mix, nq, n_tags=cfg["n_tags"], seed=3)
    _run(table, vec, bits, q, exprs, [100] * nq, max_batch=32)


@pytest.mark.parametrize("in_place", [False, True], ids=["dense_matrix", "in_place"])
@pytest.mark.parametrize("layout", ["bitmap", "packed", "matrix"])
def test_many_segments_mixed_k(torch_cuda, layout, in_place):
    kw = {"bitmap": {}, "packed": {"sparse_packed": True}, "matrix": {"matrix_posting": True}}[layout]
    mix = data.Mixture(64, 96, (1e-3, 0.6), n_clusters=64, seed=4)
    vec, bits, _ = mix.corpus(20000, seed=14)  # 5 segments of 4096, the last one partial
    table = hss.DataTable.build(vec, bits, 96, device=0, doc_num_per_segment=4096, **kw)
    nq = 48
    q = mix.queries(nq, seed=5)
    exprs = data.make_filters(mix, nq, n_tags=(1, 6), seed=6, selectivity_range=(1e-4, 1.0))
    exprs[0], exprs[1], exprs[2], exprs[3] = "", "NOT 3", "3 AND NOT 3", "95"
    topks = np.array([1, 10, 100, 1000] * (nq // 4))
    _run(table, vec, bits, q, exprs, topks, max_batch=48, decode_in_place=in_place)


@pytest.mark.parametrize("levels", [2, 3, 8])
def test_tie_heavy_corpus_orders_by_doc_id(torch_cuda, levels):
    rng = np.random.default_rng(levels)
    n, dim, tags = 9000, 16, 64
    vec = rng.integers(0, levels, (n, dim)).astype(np.float32)
    q = rng.integers(0, levels, (24, dim)).astype(np.float32)
    bits = np.zeros((n, 1), np.uint64)
    hit = rng.random((n, tags)) < 0.3
    for t in range(tags):
        bits[:, 0] |= hit[:, t].astype(np.uint64) << np.uint64(t)
    mix = data.Mixture(dim, tags, (0.1, 0.5), n_clusters=4, seed=7)
    exprs = data.make_filters(mix, 24, n_tags=(1, 3), seed=8)
    table = hss.DataTable.build(vec, bits, tags, device=0, doc_num_per_segment=2048)
    _run(table, vec, bits, q, exprs, [40, 400, 3000] * 8, max_batch=24)


def test_k_above_hits_and_k_limits(torch_cuda):
    mix = data.Mixture(32, 64, (1e-3, 0.2), n_clusters=16, seed=9)
    vec, bits, _ = mix.corpus(8192, seed=19)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=4096)
    q = mix.queries(6, seed=10)
    exprs = ["1 AND 2 AND 3", "", "0", "5 OR 6", "", "7"]
    topks = [5000, _lib.HSS_MAX_TOPK, 1, 4096, 8192, 0]
    s = hss.FullRecallSearcher(table, max_batch=8)
    for a, e, k in zip(q, exprs, topks):
        s.add_query(e, a, k)
    scores, ids, counts = s.batch_search()
    st = s.last_status(6)
    assert st[4] == _lib.QSTATUS_TOPK_TOO_LARGE and counts[4] == 0
    assert counts[5] == 0
    keep = [0, 1, 2, 3]
    want = oracle.topk(q[keep], [exprs[i] for i in keep], [min(topks[i], 4096) for i in keep], vec, bits,
                       out_stride=4096)
    _check((scores[keep], ids[keep], counts[keep]), want, 4)


def test_candidate_overflow_reruns_stay_exact(torch_cuda):
    mix = data.Mixture(32, 32, (0.3, 0.9), n_clusters=8, seed=12)
    vec, bits, _ = mix.corpus(60000, seed=22)
    table = hss.DataTable.build(vec, bits, 32, device=0, doc_num_per_segment=8192)
    nq = 16
    q = mix.queries(nq, seed=13)
    exprs = [""] * 8 + ["1 OR 2"] * 8
    s, _ = _run(table, vec, bits, q, exprs, [3000] * nq, max_batch=nq, candidate_cap=4096, sample_docs=4096)
    s.set_timing(True)


def test_doc_offset_and_device_api(torch_cuda):
    torch = torch_cuda
    mix = data.Mixture(128, 64, (1e-3, 0.5), seed=15)
    vec, bits, _ = mix.corpus(30000, seed=25)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=8192, doc_offset=1_000_000)
    nq = 40
    q = mix.queries(nq, seed=16)
    exprs = data.make_filters(mix, nq, n_tags=(1, 4), seed=17)
    topks = np.array([100] * nq, np.uint32)
    s = hss.FullRecallSearcher(table, max_batch=64)
    f = s.compile_filters(exprs)
    dq = torch.tensor(q, device="cuda")
    stride = 128
    o_sc = torch.zeros((nq, stride), dtype=torch.float32, device="cuda")
    o_id = torch.zeros((nq, stride), dtype=torch.int64, device="cuda")
    o_n = torch.zeros(nq, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = s.search_device(dq.data_ptr(), nq, f, topks, o_sc.data_ptr(), o_id.data_ptr(), o_n.data_ptr(), stride, stream)
    assert rc == _lib.HSS_OK
    torch.cuda.synchronize()
    res = (o_sc.cpu().numpy(), o_id.cpu().numpy(), o_n.cpu().numpy())
    want = oracle.topk(q, exprs, topks, vec, bits, threads=8)
    _check(res, want, nq, offset=1_000_000)
    # the same batch through AddQuery + BatchSearch gives the same answer
    for a, e in zip(q, exprs):
        s.add_query(e, a, 100)
    res2 = s.batch_search(out_stride=stride)
    _check(res2, want, nq, offset=1_000_000)


def test_saved_and_reloaded_index_searches_the_same(torch_cuda, tmp_path):
    mix = data.Mixture(64, 128, (1e-3, 0.5), seed=18)
    vec, bits, _ = mix.corpus(12000, seed=28)
    table = hss.DataTable.build(vec, bits, 128, device=0, doc_num_per_segment=4096, sparse_packed=True)
    table.save(tmp_path)
    loaded = hss.DataTable.load(tmp_path, device=0)
    nq = 20
    q = mix.queries(nq, seed=19)
    exprs = data.make_filters(mix, nq, n_tags=(1, 5), seed=20)
    _run(loaded, vec, bits, q, exprs, [50] * nq, max_batch=nq)


def test_batches_larger_than_max_batch_are_split(torch_cuda):
    mix = data.Mixture(32, 64, (1e-3, 0.5), seed=21)
    vec, bits, _ = mix.corpus(10000, seed=31)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=4096)
    nq = 70
    q = mix.queries(nq, seed=22)
    exprs = data.make_filters(mix, nq, n_tags=(1, 4), seed=23)
    _run(table, vec, bits, q, exprs, [20] * nq, max_batch=16)


def test_bad_filter_is_reported_not_run(torch_cuda):
    mix = data.Mixture(32, 64, (1e-3, 0.5), seed=24)
    vec, bits, _ = mix.corpus(4096, seed=34)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=4096)
    s = hss.FullRecallSearcher(table, max_batch=4)
    with pytest.raises(hss.HssError) as ei:
        s.add_query("1 AND", mix.queries(1)[0], 10)
    assert ei.value.code == _lib.HSS_ERR_PARSE
    with pytest.raises(hss.HssError):
        s.add_query("1", np.zeros(8, np.float32), 10)  # wrong dimension


@pytest.mark.parametrize("method", [0, 2], ids=["simt", "bf16"])
def test_searcher_in_caller_owned_workspace(torch_cuda, method):
    # the reference's ownership model: the caller sizes and owns the device arena; after the table's
    # resident data is prepared, creating the searcher allocates no device memory
    torch = torch_cuda
    mix = data.Mixture(128, 64, (1e-3, 0.5), seed=31)
    vec, bits, _ = mix.corpus(20000, seed=32)
    table = hss.DataTable.build(vec, bits, 64, device=0, doc_num_per_segment=8192)
    nq = 48
    cfg = dict(max_batch=64, candidate_cap=1 << 16, method=method)
    nbytes = hss.FullRecallSearcher.workspace_bytes(table, **cfg)
    assert nbytes > 64 * (1 << 16) * 16
    hss.FullRecallSearcher.prepare_table(table, **cfg)
    arena = torch.empty(nbytes + 256, dtype=torch.uint8, device="cuda:0")
    base = (arena.data_ptr() + 255) // 256 * 256
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    s = hss.FullRecallSearcher(table, workspace=(base, nbytes), **cfg)
    free1, _ = torch.cuda.mem_get_info(0)
    assert free0 - free1 < (4 << 20), (free0, free1)  # no device arena of its own
    q = mix.queries(nq, seed=33)
    exprs = data.make_filters(mix, nq, n_tags=(1, 4), seed=34)
    for a, e in zip(q, exprs):
        s.add_query(e, a, 100)
    res = s.batch_search()
    _check(res, oracle.topk(q, exprs, [100] * nq, vec, bits, threads=8), nq)
    s.close()
    with pytest.raises(hss.HssError):
        hss.FullRecallSearcher(table, workspace=(base, nbytes - 4096), **cfg)  # too small
    with pytest.raises(hss.HssError):
        hss.FullRecallSearcher(table, workspace=(base + 64, nbytes), **cfg)  # misaligned


def test_cross_shard_merge_equals_the_unsharded_search(torch_cuda):
    # three shards holding ascending doc ranges (global ids via doc offsets), each searched alone,
    # their top-K lists merged on the device: the result is the whole corpus's ground truth
    torch = torch_cuda
    mix = data.Mixture(128, 64, (1e-3, 0.5), n_clusters=32, seed=41)
    vec, bits, _ = mix.corpus(30000, seed=42)
    vec[7000] = vec[12000] = vec[25000]  # equal scores across shards: the lower shard (lower id) first
    bounds = [0, 9000, 21000, 30000]
    nq, K = 40, 100
    q = mix.queries(nq, seed=43)
    exprs = data.make_filters(mix, nq, n_tags=(1, 3), seed=44)
    exprs[1] = ""
    d_q = torch.tensor(q, device="cuda:0")
    outs = []
    for s in range(3):
        a, b = bounds[s], bounds[s + 1]
        table = hss.DataTable.build(vec[a:b], bits[a:b], 64, device=0, doc_num_per_segment=4096, doc_offset=a)
        srch = hss.FullRecallSearcher(table, max_batch=nq, method=2 if s == 1 else 0)
        f = srch.compile_filters(exprs)
        sc = torch.zeros((nq, K), dtype=torch.float32, device="cuda:0")
        ids = torch.zeros((nq, K), dtype=torch.int64, device="cuda:0")
        cnt = torch.zeros(nq, dtype=torch.int32, device="cuda:0")
        assert srch.search_device(d_q.data_ptr(), nq, f, [K] * nq, sc.data_ptr(), ids.data_ptr(), cnt.data_ptr(),
                                  K) == 0
        torch.cuda.synchronize()
        outs.append((sc, ids, cnt, table, srch, f))
    m_sc = torch.zeros((nq, K), dtype=torch.float32, device="cuda:0")
    m_id = torch.zeros((nq, K), dtype=torch.int64, device="cuda:0")
    m_n = torch.zeros(nq, dtype=torch.int32, device="cuda:0")
    hss.merge_shards([o[0].data_ptr() for o in outs], [o[1].data_ptr() for o in outs], [o[2].data_ptr() for o in outs],
                     nq, K, K, m_sc.data_ptr(), m_id.data_ptr(), m_n.data_ptr(), K)
    torch.cuda.synchronize()
    want = oracle.topk(q, exprs, [K] * nq, vec, bits, threads=8)
    _check((m_sc.cpu().numpy(), m_id.cpu().numpy(), m_n.cpu().numpy()), want, nq)


@pytest.mark.parametrize("method", [0, 2], ids=["simt", "bf16"])
def test_two_searchers_alternate_batches_on_one_stream(torch_cuda, method):
    # batch i is enqueued on searcher i % 2 before batch i - 1 is finished: every batch must still equal
    # the ground truth, including batches whose candidate lists overflow and re-run in the finish half
    torch = torch_cuda
    mix = data.Mixture(128, 32, (0.05, 0.9), n_clusters=16, seed=51)
    vec, bits, _ = mix.corpus(30000, seed=52)
    table = hss.DataTable.build(vec, bits, 32, device=0, doc_num_per_segment=8192)
    nq, nb = 32, 6
    kk = [50, 50, 2000, 50, 2000, 50]  # K = 2000 with a small candidate cap forces re-runs
    srch = [hss.FullRecallSearcher(table, max_batch=nq, candidate_cap=8192, sample_docs=4096, method=method)
            for _ in range(2)]
    q = mix.queries(nq * nb, seed=53)
    exprs = data.make_filters(mix, nq * nb, n_tags=(1, 2), seed=54)
    d_q = torch.tensor(q, device="cuda:0")
    sc = torch.zeros((nb, nq, 2000), dtype=torch.float32, device="cuda:0")
    ids = torch.zeros((nb, nq, 2000), dtype=torch.int64, device="cuda:0")
    cnt = torch.zeros((nb, nq), dtype=torch.int32, device="cuda:0")
    filt = [srch[0].compile_filters(exprs[b * nq:(b + 1) * nq]) for b in range(nb)]
    sh = torch.cuda.current_stream().cuda_stream
    retries = 0
    for b in range(nb):
        srch[b % 2].search_device_async(d_q[b * nq].data_ptr(), nq, filt[b], [kk[b]] * nq, sc[b].data_ptr(),
                                        ids[b].data_ptr(), cnt[b].data_ptr(), 2000, sh)
        if b > 0:
            assert srch[(b - 1) % 2].finish() == 0
            retries += srch[(b - 1) % 2].last_times()["retries"]
    assert srch[(nb - 1) % 2].finish() == 0
    torch.cuda.synchronize()
    for b in range(nb):
        qb, eb = q[b * nq:(b + 1) * nq], exprs[b * nq:(b + 1) * nq]
        want = oracle.topk(qb, eb, [kk[b]] * nq, vec, bits, threads=8)
        _check((sc[b].cpu().numpy(), ids[b].cpu().numpy(), cnt[b].cpu().numpy()), want, nq)
    # a searcher refuses a second batch before the first is finished
    srch[0].search_device_async(d_q.data_ptr(), nq, filt[0], [50] * nq, sc[0].data_ptr(), ids[0].data_ptr(),
                                cnt[0].data_ptr(), 2000, sh)
    with pytest.raises(hss.HssError):
        srch[0].search_device_async(d_q.data_ptr(), nq, filt[0], [50] * nq, sc[0].data_ptr(), ids[0].data_ptr(),
                                    cnt[0].data_ptr(), 2000, sh)
    assert srch[0].finish() == 0
