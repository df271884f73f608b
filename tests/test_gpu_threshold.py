"""The learned threshold predictor through the C-ABI.

1. The CUDA forward pass and gradients equal the CPU restatement (oracle/mlp_ref.py, float64) within
   FP32 tolerance: relative 2e-4 of the gradient's scale, written below.
2. Training with the library's own kernels lowers the loss.
3. A searcher using a trained model returns the oracle's results bit for bit; so do models whose
   thresholds are far too high (every query with more than K passing docs misses the select step's
   check and is re-run at its proven threshold) and far too low.
4. What the model gains: on held-out K = 1000 queries its candidate passes keep far fewer docs than
   the same searcher without it, and few queries' predictions were too high.
"""
import numpy as np
import pytest

import hybridsearchsystem_b200 as hss
import oracle
from hybridsearchsystem_b200 import data
from hybridsearchsystem_b200.threshold import fit_threshold_model
from oracle import mlp_ref

pytestmark = pytest.mark.gpu

GRAD_RTOL = 2e-4  # relative to the largest gradient magnitude (FP32 GEMMs, sums of up to 64 terms)


@pytest.mark.parametrize("tau", [0.0, 0.05], ids=["mse", "pinball"])
def test_mlp_forward_and_gradients_match_cpu(torch_cuda, tau):
    torch = torch_cuda
    rng = np.random.default_rng(71)
    din, h, B = 37, 48, 53
    m = hss.ThresholdModel(din, h, device=0, seed=3)
    m.set_quantile(tau)
    p = m.get_params().astype(np.float64)
    X = rng.standard_normal((B, din)).astype(np.float32)
    t = rng.standard_normal(B).astype(np.float32)
    dX = torch.tensor(X, device="cuda")
    dT = torch.tensor(t, device="cuda")
    dY = torch.zeros(B, dtype=torch.float32, device="cuda")
    m.forward(dX.data_ptr(), B, dY.data_ptr())
    torch.cuda.synchronize()
    y_ref, _ = mlp_ref.forward(p, X, din, h)
    assert np.allclose(dY.cpu().numpy(), y_ref, rtol=1e-4, atol=1e-4 * np.abs(y_ref).max())
    g, loss = m.gradients(dX.data_ptr(), dT.data_ptr(), B)
    loss_ref, g_ref = mlp_ref.loss_and_grad(p, X, t, din, h, tau)
    assert abs(loss - loss_ref) <= 1e-4 * max(1.0, loss_ref)
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= GRAD_RTOL * scale, np.abs(g - g_ref).max() / scale


def test_fused_forward_equals_the_training_forward(torch_cuda):
    # the one-launch inference pass sums in the GEMMs' order, so its outputs match the training pass's
    # (whose loss against a zero target is the mean squared output) to rounding of the loss sum
    torch = torch_cuda
    rng = np.random.default_rng(73)
    for din, h, B in ((37, 48, 53), (396, 256, 256), (844, 256, 7)):
        m = hss.ThresholdModel(din, h, device=0, seed=5)
        X = torch.tensor(rng.standard_normal((B, din)).astype(np.float32), device="cuda")
        dY = torch.zeros(B, dtype=torch.float32, device="cuda")
        m.forward(X.data_ptr(), B, dY.data_ptr())
        zero = torch.zeros(B, dtype=torch.float32, device="cuda")
        _, loss = m.gradients(X.data_ptr(), zero.data_ptr(), B)
        torch.cuda.synchronize()
        y = dY.cpu().numpy().astype(np.float64)
        assert abs(loss - float(np.mean(y * y))) <= 1e-6 * max(1.0, loss), (din, h, B)
        y_ref, _ = mlp_ref.forward(m.get_params().astype(np.float64), X.cpu().numpy(), din, h)
        assert np.allclose(y, y_ref, rtol=1e-4, atol=1e-4 * np.abs(y_ref).max()), (din, h, B)


def test_training_steps_lower_the_loss(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(72)
    din, h, B = 24, 32, 256
    X = rng.standard_normal((B, din)).astype(np.float32)
    w = rng.standard_normal(din).astype(np.float32)
    t = np.tanh(X @ w / 4).astype(np.float32)
    m = hss.ThresholdModel(din, h, device=0, seed=4)
    dX, dT = torch.tensor(X, device="cuda"), torch.tensor(t, device="cuda")
    first = m.train_step(dX.data_ptr(), dT.data_ptr(), B, 3e-3)
    for _ in range(300):
        last = m.train_step(dX.data_ptr(), dT.data_ptr(), B, 3e-3)
    assert last < 0.1 * first


def _world(seed=81, n=80000, tags=64):
    mix = data.Mixture(128, tags, (1e-3, 0.6), n_clusters=64, seed=seed)
    vec, bits, _ = mix.corpus(n, seed=seed + 1)
    table = hss.DataTable.build(vec, bits, tags, device=0, doc_num_per_segment=16384)
    return mix, vec, bits, table


def _queries(mix, n, seed, k=None):
    q = mix.queries(n, seed=seed)
    exprs = data.make_filters(mix, n, n_tags=(1, 4), seed=seed + 1, selectivity_range=(1e-3, 1.0))
    rng = np.random.default_rng(seed + 2)
    topks = (rng.choice([10, 100, 1000], n) if k is None else np.full(n, k)).astype(np.uint32)
    return q, exprs, topks


def _search(s, q, exprs, topks):
    for a, e, k in zip(q, exprs, topks):
        s.add_query(e, a, int(k))
    return s.batch_search()


def _predicted(s, q, exprs, topks, vec, bits):
    """The queries searcher s predicts a threshold for: those whose filter passes more than
    MIN_PASS_FACTOR * K docs (counted by the oracle) and whose doc sample held at least 64 of them
    (the sample's rank-64 feature is present)."""
    import torch
    from hybridsearchsystem_b200.threshold import MIN_PASS_FACTOR
    limit = np.asarray(topks, np.int64) * MIN_PASS_FACTOR
    _, _, c = oracle.topk(q, exprs, int(limit.max()) + 1, vec, bits, threads=8)
    din = s.feature_dim()
    X = torch.zeros((len(q), din), dtype=torch.float32, device="cuda")
    dq = torch.tensor(np.ascontiguousarray(q, np.float32), device="cuda")
    f = s.compile_filters(list(exprs))
    s.features(dq.data_ptr(), len(q), f, np.asarray(topks, np.uint32), X.data_ptr(),
               torch.cuda.current_stream().cuda_stream)
    f.close()
    full = X[:, din - 3].cpu().numpy() != -2.0
    return (np.asarray(c, np.int64) > limit) & full


def _check_exact(res, want, nq):
    scores, ids, counts = res
    ws, wi, wc = want
    for i in range(nq):
        c = int(wc[i])
        assert int(counts[i]) == c, i
        assert (ids[i][:c] == wi[i][:c]).all(), i
        assert (scores[i][:c].view(np.uint32) == ws[i][:c].view(np.uint32)).all(), i


def test_feature_rows_hold_the_sample_order_statistics(torch_cuda):
    # tail of a feature row: log selectivity, log K, 1, the sample's scores at ranks 1, 2, 4, ..., 64
    # (-2 past the sample's size), its K-th best (-2 when absent), log10(sample docs + 1) / 5
    torch = torch_cuda
    mix, vec, bits, table = _world(seed=85, n=60000)
    s = hss.FullRecallSearcher(table, max_batch=64, method=2)
    q, ex, k = _queries(mix, 64, 97)
    din = s.feature_dim()
    assert din == 128 + table.info["posting_rows"] + 12
    X = torch.zeros((64, din), dtype=torch.float32, device="cuda")
    dq = torch.tensor(q, device="cuda")
    f = s.compile_filters(ex)
    s.features(dq.data_ptr(), 64, f, k, X.data_ptr(), torch.cuda.current_stream().cuda_stream)
    tail = X.cpu().numpy()[:, din - 12:]
    assert np.isfinite(tail).all()
    assert (tail[:, 2] == 1.0).all()
    ranks, kth, logn = tail[:, 3:10], tail[:, 10], tail[:, 11]
    n = np.rint(10 ** (logn * 5) - 1).astype(np.int64)
    for i in range(64):
        have = (1 << np.arange(7)) <= n[i]
        assert (ranks[i][~have] == -2.0).all(), i
        r = ranks[i][have]
        assert (np.diff(r) <= 0).all(), (i, r)  # best first
        if n[i] >= k[i]:
            assert kth[i] <= r[0], i
            if k[i] <= 64:
                assert kth[i] <= r[int(np.log2(k[i]))], i
        else:
            assert kth[i] == -2.0, i


@pytest.mark.parametrize("method", [2, 1], ids=["bf16", "tf32"])
def test_learned_threshold_search_is_exact(torch_cuda, method):
    mix, vec, bits, table = _world()
    s = hss.FullRecallSearcher(table, max_batch=256, method=method)
    qt, et, kt = _queries(mix, 3072, 90)
    model, margin, report = fit_threshold_model(s, qt, et, kt, hidden=128, steps=600, seed=1)
    assert report["loss_last_epoch"] < report["loss_first_epoch"]
    qv, ev, kv = _queries(mix, 200, 95)
    want = oracle.topk(qv, ev, kv, vec, bits, threads=8)
    gated = _predicted(s, qv, ev, kv, vec, bits)
    for m in (margin, -1.0, 1.5):  # calibrated, far too high a threshold, far too low
        s.set_threshold_model(model, m)
        _check_exact(_search(s, qv, ev, kv), want, len(qv))
        assert (s.last_status(len(qv)) == 0).all()
        miss = s.last_threshold_misses(len(qv))
        assert not miss[~gated].any()  # their proven thresholds stand
        if m == -1.0:  # far too high: the queries the prediction applies to miss
            assert miss[gated].mean() > 0.9, miss.mean()
        if m == 1.5:
            assert not miss.any()


def test_learned_threshold_prunes_the_candidates(torch_cuda):
    # 400k docs, K = 1000: without a model the doc sample grows with K and the two-part pass keeps the
    # docs above the sample's (then pass A's) proven threshold; with the model the passes prune at the
    # predicted K-th score less the margin, so far fewer docs reach the select step, and few
    # predictions were too high (re-runs)
    mix, vec, bits, table = _world(seed=83, n=400000)
    s = hss.FullRecallSearcher(table, max_batch=256, method=2, sample_docs=4096)
    qt, et, kt = _queries(mix, 8192, 96)
    # the margin at the 0.99 quantile of the held-out residuals: about 1 % misses, each re-run exactly
    model, margin, report = fit_threshold_model(s, qt, et, kt, hidden=128, steps=3000, seed=2, quantile=0.99)
    qv, ev, kv = _queries(mix, 256, 99, k=1000)
    want = oracle.topk(qv, ev, kv, vec, bits, threads=8)
    _search(s, qv, ev, kv)
    without = s.last_candidate_counts(len(qv)).astype(np.int64)
    s.set_threshold_model(model, margin)
    _check_exact(_search(s, qv, ev, kv), want, len(qv))
    learned = s.last_candidate_counts(len(qv)).astype(np.int64)
    miss = s.last_threshold_misses(len(qv))
    many = _predicted(s, qv, ev, kv, vec, bits)  # the queries the prediction applies to
    pruned = 1.0 - learned[many & ~miss].sum() / max(1, without[many & ~miss].sum())
    print("learned threshold: candidates", without[many].sum(), "->", learned[many].sum(), "pruned", pruned,
          "miss rate", miss[many].mean(), report)
    assert pruned > 0.3, (pruned, miss.mean(), report)
    assert miss[many].mean() < 0.15, (pruned, miss.mean(), report)
