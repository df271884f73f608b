"""Training of the learned threshold predictor on the GPU.

With a model set, a searcher's candidate passes prune at max(doc sample's proven threshold,
prediction - margin - error bound), and its select step checks each such query: the K-th best exact
score must clear that threshold by the error bound, else the query is re-run at a proven threshold
(a miss). So the label of a query is its exact K-th best score, from the searcher's own exact path
(no model set). The searcher predicts only for queries whose filter passes more than
MIN_PASS_FACTOR * K docs (the others have few candidates whatever the threshold) and whose doc sample
held at least 64 of them (every sample rank feature present); the queries trained and calibrated on
are those.

The network predicts the standardised label with the library's own forward / backward / Adam kernels
(ThresholdModel.train_step). With tau > 0 it is trained on the pinball loss of the tau-quantile, so it
predicts a low conditional quantile of the K-th score: low where the features say little (a wide
margin for that query alone), close where they pin it down. It keeps the parameters with the lowest
held-out loss. The margin is a quantile of (prediction - label) over the held-out queries: a query
predicted above its label by more than the margin is a miss, so that quantile sets the miss rate
(quantile 1.0: the largest held-out residual).
"""
import numpy as np

from .api import ThresholdModel

MIN_PASS_FACTOR = 4  # kLearnedMinPass of the searcher's prediction step


def label_and_features(searcher, queries, exprs, topks, batch=None, min_pass_factor=MIN_PASS_FACTOR):
    """(X [n][din] device tensor, labels [n] float32 numpy): the feature rows and each query's exact
    K-th best score (NaN where its filter passes fewer than min(min_pass_factor * K, HSS_MAX_TOPK)
    docs, or where its doc sample held fewer than 64 of them)."""
    import torch
    from ._lib import HSS_MAX_TOPK
    dev = torch.device("cuda", searcher.table.device)
    B = batch or searcher.max_batch
    din = searcher.feature_dim()
    topks = np.asarray(topks, dtype=np.uint32)
    ranks = np.minimum(topks.astype(np.int64) * max(1, min_pass_factor), HSS_MAX_TOPK).astype(np.uint32)
    R = int(ranks.max())
    n = len(queries)
    X = torch.zeros((n, din), dtype=torch.float32, device=dev)
    labels = np.full(n, np.nan, np.float32)
    q = torch.zeros((B, queries.shape[1]), dtype=torch.float32, device=dev)
    sc = torch.zeros((B, R), dtype=torch.float32, device=dev)
    ids = torch.zeros((B, R), dtype=torch.int64, device=dev)
    cnt = torch.zeros(B, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for b0 in range(0, n, B):
        nb = min(B, n - b0)
        q[:nb].copy_(torch.from_numpy(np.ascontiguousarray(queries[b0:b0 + nb], np.float32)))
        f = searcher.compile_filters(list(exprs[b0:b0 + nb]))
        searcher.features(q.data_ptr(), nb, f, topks[b0:b0 + nb], X[b0:b0 + nb].data_ptr(), stream)
        rk = ranks[b0:b0 + nb]
        rc = searcher.search_device(q.data_ptr(), nb, f, rk, sc.data_ptr(), ids.data_ptr(), cnt.data_ptr(), R, stream)
        assert rc == 0, searcher.last_status(nb)
        s_h = sc[:nb].cpu().numpy()
        c_h = cnt[:nb].cpu().numpy()
        # the sample's rank-64 feature (-2 when its sample held fewer than 64 filtered docs)
        full = X[b0:b0 + nb, din - 3].cpu().numpy() != -2.0
        for i in range(nb):
            k = int(topks[b0 + i])
            if k > 0 and c_h[i] >= int(rk[i]) and full[i]:
                labels[b0 + i] = s_h[i, k - 1]
        f.close()
    return X, labels


def fit_threshold_model(searcher, queries, exprs, topks, hidden=256, steps=2000, batch=512, lr=2e-3, seed=0,
                        val_fraction=0.15, quantile=0.999, slack=0.0, n_val=None, tau=0.02):
    """Trains a ThresholdModel for `searcher` (which must have no model set) on the given queries,
    holding out n_val of them (or val_fraction) for the early stop and the margin; tau is the quantile
    the network is trained to predict (0: the mean, by squared error). Returns (model, margin, report)."""
    import torch
    topks = np.asarray(topks, np.uint32)
    X, labels = label_and_features(searcher, queries, exprs, topks)
    keep = np.nonzero(np.isfinite(labels))[0]
    rng = np.random.default_rng(seed)
    rng.shuffle(keep)
    nval = max(1, min(len(keep) - 1, n_val) if n_val else int(len(keep) * val_fraction))
    val, tr = keep[:nval], keep[nval:]
    mu, sd = float(labels[tr].mean()), float(labels[tr].std() + 1e-6)
    dev = X.device
    T = torch.from_numpy(np.nan_to_num((labels - mu) / sd).astype(np.float32)).to(dev)
    din = X.shape[1]
    model = ThresholdModel(din, hidden, device=dev.index or 0, seed=seed)
    model.set_output_scale(sd, mu)
    model.set_quantile(tau)

    def held_out_loss(res):  # the training loss over residuals (prediction - label), in score units
        return float(np.mean(res * res)) if tau <= 0 else float(np.mean(np.where(res > 0, (1 - tau) * res, -tau * res)))

    stream = torch.cuda.current_stream(dev).cuda_stream
    tr_t = torch.from_numpy(tr.astype(np.int64)).to(dev)
    xb = torch.zeros((batch, din), dtype=torch.float32, device=dev)
    tb = torch.zeros(batch, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    def predict(idx):
        y = torch.zeros(len(idx), dtype=torch.float32, device=dev)
        xs = X.index_select(0, torch.from_numpy(idx.astype(np.int64)).to(dev)).contiguous()
        model.forward(xs.data_ptr(), len(idx), y.data_ptr(), stream)
        return y.cpu().numpy() * sd + mu

    # minibatch Adam with cosine decay; the parameters kept are those with the lowest held-out loss
    # (checked every `check_every` steps), which stops the network from memorising the training queries
    losses = []
    batch = min(batch, len(tr))
    steps_per_epoch = max(1, len(tr) // batch)
    check_every = max(25, steps // 40)
    best = (np.inf, model.get_params(), 0)
    step = 0
    while step < steps:
        perm = tr_t[torch.randperm(len(tr), device=dev, generator=gen)]
        ep_loss, n_ep = 0.0, 0
        for s in range(steps_per_epoch):
            if step >= steps:
                break
            idx = perm[s * batch:(s + 1) * batch]
            nb = idx.numel()
            xb[:nb].copy_(X.index_select(0, idx))
            tb[:nb].copy_(T.index_select(0, idx))
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / steps))
            ep_loss += model.train_step(xb.data_ptr(), tb.data_ptr(), nb, float(cur), stream)
            n_ep += 1
            step += 1
            if step % check_every == 0 or step == steps:
                err = held_out_loss(predict(val) - labels[val])
                if err < best[0]:
                    best = (err, model.get_params(), step)
        losses.append(ep_loss / max(1, n_ep))
    model.set_params(best[1])

    res_val = predict(val) - labels[val]
    res_tr = predict(tr) - labels[tr]
    margin = float(np.quantile(res_val, quantile)) + slack
    report = {"train_queries": int(len(tr)), "val_queries": int(len(val)), "label_mean": mu, "label_std": sd,
              "loss_first_epoch": losses[0], "loss_last_epoch": losses[-1],
              "val_abs_err_median": float(np.median(np.abs(res_val))),
              "val_rmse": float(np.sqrt(np.mean(res_val ** 2))), "train_rmse": float(np.sqrt(np.mean(res_tr ** 2))),
              "margin": margin, "val_overshoot_rate_at_margin": float(np.mean(res_val > margin)),
              "val_residual_quantiles": {str(q): float(np.quantile(res_val, q)) for q in (0.5, 0.9, 0.99, 0.999, 1.0)},
              "val_residual_quantiles_by_k": {
                  f"K{int(k)}": {str(q): float(np.quantile(res_val[topks[val] == k], q)) for q in (0.99, 0.999, 1.0)}
                  for k in np.unique(topks[val])},
              "tau": tau, "labelled_fraction": float(len(keep) / max(1, len(labels))),
              "steps": steps, "best_step": best[2]}
    return model, margin, report
