"""The serving loop (continuous batching) through the C-ABI.

A query's result must not depend on what it is batched with. Every query is run alone (submitted,
then waited for, before the next one is submitted), then all are submitted at once. In the second
run the loop forms mixed batches on several slots, with uneven K and filter selectivity. Both runs
must return the oracle's ids and scores bit for bit (tolerance 0). Open-loop Poisson arrivals must
complete without failures and report latency percentiles.
"""
import threading

import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import data

pytestmark = pytest.mark.gpu


def _world(n=60000, tags=64, seed=121):
    mix = data.Mixture(128, tags, (1e-3, 0.6), n_clusters=64, seed=seed)
    vec, bits, _ = mix.corpus(n, seed=seed + 1)
    table = hss.DataTable.build(vec, bits, tags, device=0, doc_num_per_segment=16384)
    return mix, vec, bits, table


def _requests(mix, n, seed):
    q = mix.queries(n, seed=seed)
    exprs = data.make_filters(mix, n, n_tags=(1, 4), seed=seed + 1, selectivity_range=(1e-3, 1.0))
    rng = np.random.default_rng(seed + 2)
    topks = np.exp(rng.uniform(0, np.log(1000), n)).astype(np.uint32) + 1  # log-uniform K in [1, 1000]
    return q, exprs, topks


def _same(got, want, i):
    sc, ids, _, st = got
    ws, wi, wc = want
    c = int(wc[i])
    assert st == 0 and len(ids) == c, (i, st, len(ids), c)
    assert (ids == wi[i][:c]).all(), i
    assert (sc.view(np.uint32) == ws[i][:c].view(np.uint32)).all(), i


@pytest.mark.parametrize("graphs", [True, False], ids=["graphs", "direct"])
@pytest.mark.parametrize("method", [0, 2], ids=["simt", "bf16"])
def test_results_same_alone_and_in_the_mix(torch_cuda, method, graphs):
    mix, vec, bits, table = _world()
    q, exprs, topks = _requests(mix, 96, 130)
    want = oracle.topk(q, exprs, topks, vec, bits, threads=8)
    srv = hss.Server(table, slots=3, max_batch=32, max_wait_us=2000, method=method, graphs=graphs)
    for i in range(len(q)):  # alone: one query on the GPU at a time
        _same(srv.wait(srv.submit(exprs[i], q[i], int(topks[i]))), want, i)
    assert srv.stats()["mean_batch"] == 1.0
    srv.reset_stats()
    # in the mix: three client threads submit everything at once
    ids = [None] * len(q)

    def client(part):
        for i in part:
            ids[i] = srv.submit(exprs[i], q[i], int(topks[i]))

    threads = [threading.Thread(target=client, args=(range(t, len(q), 3),)) for t in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for i in range(len(q)):
        _same(srv.wait(ids[i]), want, i)
    st = srv.stats()
    assert st["completed"] == len(q) and st["mean_batch"] > 1.0, st
    if graphs:  # batch shapes captured once, replayed for later batches of the same shape
        assert st["graph_captures"] > 0 and st["graph_replays"] > 0, st
    else:
        assert st["graph_captures"] == 0 and st["graph_replays"] == 0, st
    srv.close()


def test_poisson_arrivals_complete_with_latency_percentiles(torch_cuda):
    mix, vec, bits, table = _world(seed=141)
    q, exprs, topks = _requests(mix, 3000, 150)
    srv = hss.Server(table, slots=2, max_batch=128, max_wait_us=300, method=2)
    lat, offered, wall = srv.run_poisson(q, exprs, topks, rate_qps=20000, seed=7)
    assert (lat > 0).all()
    st = srv.stats()
    assert st["completed"] == len(q) and st["p99_ms"] >= st["p50_ms"] > 0, st
    assert offered > 5000, offered
