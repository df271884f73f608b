"""CUDA-graph replay of a batch's first attempt (hss_searcher_set_graphs), through the C-ABI.

A batch shape (rows rounded up, K rounded up to a power of two, the filters' largest operand count,
the model, the buffers) is captured at its first batch and replayed for the later ones, with each
batch's own filter programs copied in by the graph. Every batch, captured or replayed, must return
the oracle's ids and scores bit for bit (tolerance 0): batch sizes that are padded to their shape
with match-nothing rows, K rounded up, programs of other lengths than the captured batch's,
candidate-overflow re-runs launched after a replay, and the learned threshold's model launches.
"""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import data

pytestmark = pytest.mark.gpu

B, STRIDE = 64, 2048
# (rows, K) of the first pass; the second pass has other rows and K of the same shapes
SHAPES_A = [(1, 10), (3, 100), (17, 100), (40, 2000), (64, 7)]
SHAPES_B = [(1, 12), (4, 128), (32, 65), (48, 1500), (64, 8)]


def _check(sc, ids, cnt, want, nq):
    ws, wi, wc = want
    for i in range(nq):
        c = int(wc[i])
        assert int(cnt[i]) == c, (i, cnt[i], c)
        assert (ids[i][:c] == wi[i][:c]).all(), i
        assert (sc[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), i


def _filters(mix, n, seed):
    # at most three tags each, and one four-tag filter per batch: every batch has the same largest
    # operand count, so the second pass replays the first pass's shapes
    ex = data.make_filters(mix, n, n_tags=(1, 3), seed=seed, selectivity_range=(1e-3, 1.0))
    ex[0] = "1 OR 2 OR 3 OR NOT 4"
    return ex


def _run_pass(torch, s, mix, vec, bits, shapes, seed, stream, bufs):
    d_q, sc, ids, cnt = bufs
    retries = 0
    for j, (nq, k) in enumerate(shapes):
        q = mix.queries(nq, seed=seed + j)
        ex = _filters(mix, nq, seed + 100 + j)
        f = s.compile_filters(ex)
        with torch.cuda.stream(stream):
            d_q[:nq].copy_(torch.from_numpy(q).to("cuda:0"))
        rc = s.search_device(d_q.data_ptr(), nq, f, [k] * nq, sc.data_ptr(), ids.data_ptr(), cnt.data_ptr(),
                             STRIDE, stream.cuda_stream)
        assert rc == 0
        stream.synchronize()
        retries += s.last_times()["retries"]
        want = oracle.topk(q, ex, [k] * nq, vec, bits, threads=8)
        _check(sc.cpu().numpy(), ids.cpu().numpy(), cnt.cpu().numpy(), want, nq)
    return retries


def _world(torch, seed):
    mix = data.Mixture(128, 32, (0.05, 0.9), n_clusters=16, seed=seed)
    vec, bits, _ = mix.corpus(30000, seed=seed + 1)
    table = hss.DataTable.build(vec, bits, 32, device=0, doc_num_per_segment=8192)
    bufs = (torch.zeros((B, 128), dtype=torch.float32, device="cuda:0"),
            torch.zeros((B, STRIDE), dtype=torch.float32, device="cuda:0"),
            torch.zeros((B, STRIDE), dtype=torch.int64, device="cuda:0"),
            torch.zeros(B, dtype=torch.int32, device="cuda:0"))
    return mix, vec, bits, table, bufs


@pytest.mark.parametrize("method", [0, 2], ids=["simt", "bf16"])
def test_replayed_batches_equal_the_ground_truth(torch_cuda, method):
    torch = torch_cuda
    mix, vec, bits, table, bufs = _world(torch, 61)
    s = hss.FullRecallSearcher(table, max_batch=B, candidate_cap=8192, sample_docs=4096, method=method)
    s.set_graphs(True)
    stream = torch.cuda.Stream()
    _run_pass(torch, s, mix, vec, bits, SHAPES_A, 200, stream, bufs)
    st = s.graph_stats()
    assert (st["captures"], st["replays"], st["failed"]) == (len(SHAPES_A), 0, False), st
    _run_pass(torch, s, mix, vec, bits, SHAPES_B, 300, stream, bufs)
    st = s.graph_stats()
    assert (st["captures"], st["replays"], st["failed"]) == (len(SHAPES_A), len(SHAPES_B), False), st
    print("capture and instantiation, ms per shape:", st["capture_ms"] / st["captures"])
    # off again: the same batches launched directly
    s.set_graphs(False)
    _run_pass(torch, s, mix, vec, bits, SHAPES_B, 300, stream, bufs)
    assert s.graph_stats()["replays"] == len(SHAPES_B)


def test_replay_with_a_threshold_model(torch_cuda):
    # an untrained model's predictions, far too high (margin -1: most gated queries miss and re-run,
    # after the replayed graph) and far too low (margin 1.5): results exact either way, through
    # captured model launches
    torch = torch_cuda
    mix, vec, bits, table, bufs = _world(torch, 71)
    s = hss.FullRecallSearcher(table, max_batch=B, method=2)
    model = hss.ThresholdModel(s.feature_dim(), 64, device=0, seed=9)
    s.set_graphs(True)
    stream = torch.cuda.Stream()
    for margin in (-1.0, 1.5):
        s.set_threshold_model(model, margin)  # drops the captured shapes: the margin is in them
        _run_pass(torch, s, mix, vec, bits, SHAPES_A[:3], 400, stream, bufs)
        retries = _run_pass(torch, s, mix, vec, bits, SHAPES_B[:3], 500, stream, bufs)
        if margin < 0:
            assert retries > 0  # threshold misses re-run after replays
    st = s.graph_stats()
    assert (st["captures"], st["replays"], st["failed"]) == (6, 6, False), st


def test_default_stream_falls_back_to_direct_launches(torch_cuda):
    # the legacy default stream cannot be captured: the searcher reports the failed capture, turns
    # graphs off and launches the batch directly, with the same results
    torch = torch_cuda
    mix, vec, bits, table, bufs = _world(torch, 81)
    s = hss.FullRecallSearcher(table, max_batch=B, method=2)
    s.set_graphs(True)
    d_q, sc, ids, cnt = bufs
    nq, k = 20, 50
    q = mix.queries(nq, seed=82)
    ex = _filters(mix, nq, 83)
    d_q[:nq].copy_(torch.from_numpy(q).to("cuda:0"))
    torch.cuda.synchronize()
    f = s.compile_filters(ex)
    assert s.search_device(d_q.data_ptr(), nq, f, [k] * nq, sc.data_ptr(), ids.data_ptr(), cnt.data_ptr(), STRIDE,
                           0) == 0
    torch.cuda.synchronize()
    want = oracle.topk(q, ex, [k] * nq, vec, bits, threads=8)
    _check(sc.cpu().numpy(), ids.cpu().numpy(), cnt.cpu().numpy(), want, nq)
    st = s.graph_stats()
    assert (st["captures"], st["replays"], st["failed"]) == (0, 0, True), st


@pytest.mark.parametrize("method", [0, 2], ids=["simt", "bf16"])
def test_replay_of_edge_batches(torch_cuda, method):
    # match-all and NOT filters, K = 0, K at the output stride over a match-all filter, K above a
    # filter's hits: captured, then replayed with other queries and the filters' order reversed (other
    # program offsets, the same shape); every batch equals the ground truth
    torch = torch_cuda
    mix, vec, bits, table, bufs = _world(torch, 91)
    d_q, sc, ids, cnt = bufs
    s = hss.FullRecallSearcher(table, max_batch=B, candidate_cap=1 << 16, method=method)
    s.set_graphs(True)
    stream = torch.cuda.Stream()
    ex = ["", "NOT 1", "1 OR 2 OR 3 OR NOT 4", "5 AND 6 AND 7", "8", "NOT 9 AND 10", "", "11 OR 12"]
    kk = [0, 1, 7, STRIDE, 100, 2000, 64, 300]
    for j in range(3):
        q = mix.queries(len(ex), seed=92 + j)
        e, k = (ex, kk) if j % 2 == 0 else (ex[::-1], kk[::-1])
        f = s.compile_filters(e)
        with torch.cuda.stream(stream):
            d_q[:len(e)].copy_(torch.from_numpy(q).to("cuda:0"))
        assert s.search_device(d_q.data_ptr(), len(e), f, k, sc.data_ptr(), ids.data_ptr(), cnt.data_ptr(), STRIDE,
                               stream.cuda_stream) == 0
        stream.synchronize()
        want = oracle.topk(q, e, k, vec, bits, threads=8)
        _check(sc.cpu().numpy(), ids.cpu().numpy(), cnt.cpu().numpy(), want, len(e))
    st = s.graph_stats()
    assert (st["captures"], st["replays"], st["failed"]) == (1, 2, False), st
