#!/usr/bin/env python
"""Benchmark of the filtered full-recall path: QPS of batched filtered top-K search on the 10M x 128
FP32 corpus (256 tags, densities log-uniform in [1e-4, 0.6], filters of 1-6 tags whose selectivity
spreads over 1e-4..1, K = 100, batches of 256 queries), one resident index per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one batch of queries through the whole path (filter -> candidate scoring -> exact
rescoring + top-K). `value` is whole-job QPS with queries and index resident in HBM (device-timed,
max over ranks); `e2e` is the same through the public C-ABI with the batch's queries copied from pinned
host memory and its results copied back inside the timed region. Under torchrun every rank holds a
full replica and serves its own batches (weak scaling, no data-path collective).

--impl reference times the reference's own CPU ground-truth scan (CpuTopKBatch, compiled from the
reference sources into oracle/_ref) on this host's cores for the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS & p99 at 10M x128 filtered top-100, recall 1.0: chosen form vs plain FP32"
METHODS = {"simt": 0, "tf32": 1, "bf16": 2, "e4m3": 3}
FORMS = {"simt": "plain FP32 (SIMT FFMA candidate pass + exact FP32 rescoring)",
         "tf32": "plain FP32 (TF32 tensor-core candidate pass over the FP32 rows + exact FP32 rescoring)",
         "bf16": "BF16 copy (tensor-core candidate pass + exact FP32 rescoring)",
         "e4m3": "FP8 E4M3 copy with per-vector scales (tensor-core candidate pass + exact FP32 rescoring)"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--docs", type=int, default=10_000_000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--topk", type=int, default=100)
    ap.add_argument("--queries", type=int, default=2048, help="query pool the steps cycle through")
    ap.add_argument("--cpu-queries", type=int, default=0, help="CPU baseline sample size (0: 2 per thread)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cand-cap", type=int, default=1 << 18, help="per-query candidate capacity")
    ap.add_argument("--sample-docs", type=int, default=32768, help="docs of the threshold sample per batch")
    ap.add_argument("--method", default="bf16", choices=list(METHODS),
                    help="the chosen form's candidate pass: simt (FP32 FFMA), tf32 (tensor cores over the FP32 "
                         "rows), bf16, e4m3")
    ap.add_argument("--learned", action="store_true", help="the chosen form uses the learned threshold")
    ap.add_argument("--train-queries", type=int, default=32768, help="training queries of the learned threshold")
    ap.add_argument("--no-learned-form", dest="learned_form", action="store_false",
                    help="skip measuring the chosen format with the learned threshold beside it")
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip measuring the plain FP32 (TF32) form beside the chosen one")
    ap.add_argument("--no-serve", dest="serve", action="store_false", help="skip the serving-loop latency sweep")
    ap.add_argument("--no-batch64", dest="batch64", action="store_false",
                    help="skip measuring the chosen (and plain) form at batches of 64 queries")
    ap.add_argument("--serve-requests", type=int, default=40000)
    ap.add_argument("--serve-rates", default="1000,10000,50000,100000,150000,200000",
                    help="offered Poisson rates (QPS) of the serving sweep")
    ap.add_argument("--serve-wait-us", type=int, default=300)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def max_over_ranks(ms, device):
    """The slowest rank's time: every rank's number, all-reduced with MAX (one collective, taken by
    every rank in the same order)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_qps(world, steps, batch, t_max_ms):
    """Weak scaling: every rank serves `steps` batches of `batch` queries; the job takes the slowest
    rank's time."""
    return world * steps * batch / (t_max_ms / 1e3)


def workload(args, device):
    from hybridsearchsystem_b200 import data
    mix = data.Mixture(128, 256, (1e-4, 0.6), n_clusters=1024, sigma=0.3, n_corr=16, seed=1)
    if device is not None:
        vec, bits = mix.corpus_torch(args.docs, device=device, seed=11)
    else:
        vec, bits, _ = mix.corpus(args.docs, seed=11)
    queries = mix.queries(args.queries, seed=2)
    exprs = data.make_filters(mix, args.queries, n_tags=(1, 6), seed=3, selectivity_range=(1e-4, 1.0))
    return mix, vec, bits, queries, exprs


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while running. Entering waits until
    the first sample has been written (nvidia-smi takes a while to start); that sample predates the
    timed region and is dropped from the summary."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", self.gpu_id], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        t0 = time.time()
        while self.proc and time.time() - t0 < 10 and os.path.getsize(self.out.name) == 0:
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        self.out.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines()[1:]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.out.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(vec, bits, queries, exprs, topk, nq_sample):
    """The reference's CpuTopKBatch (oracle/_ref, compiled from its sources) on all host threads, or the
    oracle's restatement of it when the reference build is absent. Returns (record, ids, counts)."""
    import ctypes

    import oracle
    threads = os.cpu_count() or 1
    nq = nq_sample or 2 * threads
    nq = min(nq, len(queries))
    q = np.ascontiguousarray(queries[:nq], np.float32)
    ex = exprs[:nq]
    topks = np.full(nq, topk, np.int32)
    t0 = time.perf_counter()
    if oracle.ref_available():
        r = oracle.ref()
        arr = (ctypes.c_char_p * nq)(*[e.encode() for e in ex])
        ids = np.full((nq, topk), -1, np.int64)
        counts = np.zeros(nq, np.int32)
        rc = r.ref_cpu_topk_batch(q.ctypes.data, nq, q.shape[1], arr, topks.ctypes.data, vec.ctypes.data,
                                  bits.ctypes.data, bits.shape[1] * 64, vec.shape[0], 0, 1, threads, topk,
                                  ids.ctypes.data, counts.ctypes.data)
        assert rc == 0
        kind = "reference"
    else:
        _, ids, counts = oracle.topk(q, ex, topks, vec, bits, threads=threads, out_stride=topk)
        kind = "port"
    dt = time.perf_counter() - t0
    rec = {"value": nq / dt, "unit": "QPS", "cores": threads, "kind": kind,
           "sample": f"{nq} queries (filtered top-{topk}) over the full {vec.shape[0]}-doc corpus, "
                     f"CpuTopKBatch in {threads} query slices, fp32 mode"}
    return rec, ids, counts


def run_reference(args):
    rank, local, world = dist_env()
    if rank != 0:
        return
    import torch
    device = "cuda" if torch.cuda.is_available() else None
    _, vec, bits, queries, exprs = workload(args, device)
    threads = os.cpu_count() or 1
    nq = args.cpu_queries or 2 * threads
    for _ in range(args.warmup):
        cpu_baseline(vec, bits, queries, exprs, args.topk, max(1, nq // 4))
    total_q, total_t = 0, 0.0
    rec = None
    for s in range(args.steps):
        t0 = time.perf_counter()
        rec, _, _ = cpu_baseline(vec, bits, queries, exprs, args.topk, nq)
        total_t += time.perf_counter() - t0
        total_q += min(nq, len(queries))
    v = total_q / total_t
    rec = dict(rec, value=v)
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "QPS", "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic (seeded cluster mixture, HYDSET2 shapes)",
                      "config": config_of(args, world), "cpu_baseline": rec,
                      "e2e": {"value": v, "unit": "QPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def config_of(args, world):
    return {"workload": f"filtered top-{args.topk}, {args.docs} docs x 128 FP32, 256 tags, batch {args.batch}",
            "docs": args.docs, "dim": 128, "tags": 256, "batch": args.batch, "topk": args.topk,
            "doc_num_per_segment": 131072, "filters": "1-6 tags AND/OR/NOT, est. selectivity 1e-4..1",
            "parallelism": f"replica x{world}",
            "l2": "inputs larger than L2: every step reads the whole corpus copy (FP32 5.1 GB, BF16 2.6 GB, "
                  "E4M3 1.3 GB)"}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def measure_form(args, ctx, method, learned=False):
    """One form of the path (candidate-pass method, with or without the learned threshold) over the
    workload: device-resident QPS (CUDA events, max over ranks), end-to-end QPS through the C-ABI,
    stage times and the candidate stage's roofline."""
    import torch

    import hybridsearchsystem_b200 as hss
    from hybridsearchsystem_b200.threshold import fit_threshold_model
    rank, world, dev, table = ctx["rank"], ctx["world"], ctx["dev"], ctx["table"]
    queries, exprs, barrier = ctx["queries"], ctx["exprs"], ctx["barrier"]
    B, K = args.batch, args.topk
    searcher = hss.FullRecallSearcher(table, max_batch=B, candidate_cap=args.cand_cap, method=METHODS[method],
                                      sample_docs=args.sample_docs)
    report = None
    if learned:
        # trained on its own queries (seeded apart from the measured ones), labels from the exact path
        tq = ctx["mix"].queries(args.train_queries, seed=20)
        te = data_filters(ctx["mix"], args.train_queries, 21)
        tk = np.random.default_rng(22).choice([10, 100, 1000], args.train_queries).astype(np.uint32)
        model, margin, report = fit_threshold_model(searcher, tq, te, tk, hidden=256, steps=2000, seed=3)
        searcher.set_threshold_model(model, margin)
    searcher.set_timing(True)
    nb = max(1, len(queries) // B)
    filters = [searcher.compile_filters(exprs[i * B:(i + 1) * B]) for i in range(nb)]
    topks = np.full(B, K, np.uint32)
    d_q = torch.tensor(np.ascontiguousarray(queries[:nb * B]).reshape(nb, B, -1), device=dev)
    o_sc = torch.zeros((B, K), dtype=torch.float32, device=dev)
    o_id = torch.zeros((B, K), dtype=torch.int64, device=dev)
    o_n = torch.zeros(B, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    def step(i):
        j = (rank * 7919 + i) % nb
        rc = searcher.search_device(d_q[j].data_ptr(), B, filters[j], topks, o_sc.data_ptr(), o_id.data_ptr(),
                                    o_n.data_ptr(), K, sh)
        assert rc == 0, searcher.last_status(B)
        return searcher.last_times()

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # device-resident leg
    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    cand_ms, launches, stage_ms = [], 0, []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_id) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(args.steps):
            t = step(args.warmup + i)
            cand_ms.append(t["candidates_ms"])
            stage_ms.append([t["filter_ms"], t["sample_ms"], t["candidates_ms"], t["select_ms"], t["total_ms"]])
            launches += t["launches"]
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    clocks = clk.summary()
    t_max = max_over_ranks(ev0.elapsed_time(ev1), dev)
    value = whole_job_qps(world, args.steps, B, t_max)

    # end-to-end leg through the C-ABI: pinned host queries in, results out, every step. Each step
    # is one batch through hss_filters_compile + hss_searcher_search_device with its host->device
    # query copy and device->host result copy, on one searcher and stream. A second host thread
    # compiles the next batch's filters (host-only work, table read-only) while this batch is on the
    # GPU; the ctypes calls release the interpreter lock.
    from concurrent.futures import ThreadPoolExecutor
    h_q = torch.tensor(np.ascontiguousarray(queries[:nb * B]).reshape(nb, B, -1)).pin_memory()
    h_sc = torch.zeros((B, K), dtype=torch.float32).pin_memory()
    h_id = torch.zeros((B, K), dtype=torch.int64).pin_memory()
    h_n = torch.zeros(B, dtype=torch.int32).pin_memory()
    d_stage = torch.zeros((B, 128), dtype=torch.float32, device=dev)

    def batch_of(i):
        return (rank * 7919 + args.warmup + i) % nb

    def e2e_run(steps, pool):
        fut = pool.submit(lambda: searcher.compile_filters(exprs[batch_of(0) * B:(batch_of(0) + 1) * B]))
        for i in range(steps):
            j = batch_of(i)
            f = fut.result()
            if i + 1 < steps:
                jn = batch_of(i + 1)
                fut = pool.submit(lambda jn=jn: searcher.compile_filters(exprs[jn * B:(jn + 1) * B]))
            d_stage.copy_(h_q[j], non_blocking=True)
            rc = searcher.search_device(d_stage.data_ptr(), B, f, topks, o_sc.data_ptr(), o_id.data_ptr(),
                                        o_n.data_ptr(), K, sh)
            assert rc == 0
            h_sc.copy_(o_sc, non_blocking=True)
            h_id.copy_(o_id, non_blocking=True)
            h_n.copy_(o_n, non_blocking=True)
            stream.synchronize()
            f.close()

    with ThreadPoolExecutor(1) as pool:
        e2e_run(2, pool)  # warm-up of the compile thread
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        e2e_run(args.steps, pool)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    e2e = whole_job_qps(world, args.steps, B, max_over_ranks(e0.elapsed_time(e1), dev))

    # roofline of the dominant stage, the candidate passes: algorithmic bytes per batch = the corpus
    # rows the passes read (docs x 128 x element bytes, +4 B scale for E4M3; a learned form's
    # estimation pass re-reads a quarter) + the batch's filter bitmaps (B x docs/8 B)
    info = table.info
    words = info["segment_num"] * info["doc_num_per_segment"] // 64
    elem = {"simt": 4, "tf32": 4, "bf16": 2, "e4m3": 1}[method]
    reads = 1.25 if learned else 1.0
    alg_bytes = reads * args.docs * (128 * elem + (4 if method == "e4m3" else 0)) + B * words * 8
    cand_avg = float(np.mean(cand_ms))
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (cand_avg / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "cand_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(method)
    kernel = "cand_simt_kernel" if method == "simt" else ("tc2_cand_kernel" if B > 128 else "tc_cand_kernel")
    # the tensor side of the same stage: 2 d flops per (query, doc) pair of every pass, against the
    # pipe's peak (measured BF16 GEMM rate; TF32 and E4M3 by the nominal dense ratios 1/2 and 2)
    flops = reads * 2.0 * 128 * args.docs * B
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    tpeak = {"simt": None, "tf32": bf16_peak / 2, "bf16": bf16_peak, "e4m3": bf16_peak * 2}[method]
    t_s = cand_avg / 1e3
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": traffic, "kernel": kernel, "avg_ms": cand_avg,
            "peak_source": "measured" if peaks else "fallback",
            "tensor": None if tpeak is None else {
                "achieved_tflops": flops / t_s / 1e12, "peak_tflops": tpeak, "frac": flops / t_s / 1e12 / tpeak,
                "peak_note": "measured BF16 GEMM" + ("" if method == "bf16" else " x nominal dense ratio")},
            "bound_frac": (max(alg_bytes / (hbm * 1e9), 0.0 if tpeak is None else flops / (tpeak * 1e12)) / t_s)}
    out = {"value": value, "t_max_ms": t_max, "e2e": e2e, "batch": B, "roofline": roof, "clocks": clocks, "launches": launches,
           "stages_ms": dict(zip(["filter", "sample", "candidates", "select", "total"],
                                 [round(float(x), 4) for x in np.mean(np.array(stage_ms), axis=0)])),
           "form": FORMS[method] + (" + learned threshold" if learned else ""), "method": method,
           "learned": learned, "searcher": searcher, "filters": filters, "d_q": d_q,
           "out": (o_sc, o_id, o_n, topks, sh)}
    if report:
        out["model"], out["margin"] = model, margin
        out["learned_report"] = {k: (round(v, 5) if isinstance(v, float) else v) for k, v in report.items()}
        # what the model does on this workload: its estimation pass against the same pass at the doc
        # sample's proven threshold (margin 1e9 turns the prediction into -inf), over the measured batches
        at_sample, at_model, kk = [], [], []
        for j in range(min(nb, 8)):
            for m, sink in ((1e9, at_sample), (margin, at_model)):
                searcher.set_threshold_model(model, m)
                rc = searcher.search_device(d_q[j].data_ptr(), B, filters[j], topks, o_sc.data_ptr(), o_id.data_ptr(),
                                            o_n.data_ptr(), K, sh)
                assert rc == 0
                sink.append(searcher.last_estimate_counts(B).astype(np.int64))
            kk.append(topks.astype(np.int64))
        at_sample, at_model, kk = np.concatenate(at_sample), np.concatenate(at_model), np.concatenate(kk)
        searcher.set_threshold_model(model, margin)
        out["learned_report"].update({
            "estimation_pass_docs_at_sample_threshold": int(at_sample.sum()),
            "estimation_pass_docs_at_model_threshold": int(at_model.sum()),
            "pruned_fraction": round(1.0 - at_model.sum() / max(1, at_sample.sum()), 4),
            "miss_rate": round(float(np.mean(at_model < kk)), 4), "queries": int(len(kk))})
    return out


def data_filters(mix, n, seed):
    from hybridsearchsystem_b200 import data
    return data.make_filters(mix, n, n_tags=(1, 6), seed=seed, selectivity_range=(1e-4, 1.0))


def measure_serving(args, ctx, method, rates, model=None, margin=0.0):
    """p50/p99 latency of single queries through the serving loop (continuous batching) at open-loop
    Poisson arrival rates. Requests mix the workload's filters (selectivity log-uniform in
    [1e-4, 1]) with per-request K log-uniform in [1, 1000]."""
    import hybridsearchsystem_b200 as hss
    srv = hss.Server(ctx["table"], slots=2, max_batch=args.batch, max_wait_us=args.serve_wait_us,
                     method=METHODS[method], candidate_cap=args.cand_cap)
    if model is not None:
        srv.set_threshold_model(model, margin)
    q, ex = ctx["queries"], ctx["exprs"]
    kk = np.exp(np.random.default_rng(77).uniform(0.0, np.log(1000.0), len(q))).astype(np.uint32) + 1
    kk = np.minimum(kk, 1000)
    out = []
    for rate in rates:
        n = int(min(args.serve_requests, max(2000, rate * 0.5)))
        idx = np.arange(n) % len(q)
        srv.reset_stats()
        lat, offered, wall = srv.run_poisson(q[idx], [ex[i] for i in idx], kk[idx], rate, seed=int(rate))
        st = srv.stats()
        out.append({"offered_qps": round(offered), "completed_qps": round(n / wall), "p50_ms": round(st["p50_ms"], 3),
                    "p99_ms": round(st["p99_ms"], 3), "mean_batch": round(st["mean_batch"], 1)})
    srv.close()
    return {"form": FORMS[method] + (" + learned threshold" if model is not None else ""), "slots": 2,
            "max_wait_us": args.serve_wait_us, "topk": "log-uniform in [1, 1000] per request", "rates": out}


def run_ours(args):
    import torch
    import torch.distributed as dist

    import hybridsearchsystem_b200 as hss
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = f"cuda:{local}"
    mix, vec, bits, queries, exprs = workload(args, dev)
    table = hss.DataTable.build(vec, bits, 256, device=local, doc_num_per_segment=131072)

    def barrier():
        if world > 1:
            dist.barrier()

    ctx = {"rank": rank, "world": world, "dev": dev, "table": table, "queries": queries, "exprs": exprs,
           "barrier": barrier, "mix": mix}
    B, K = args.batch, args.topk
    chosen = measure_form(args, ctx, args.method, learned=args.learned)
    forms = {"chosen": chosen}
    if args.learned_form and not args.learned:
        # the chosen format with the learned threshold, measured beside it
        forms["chosen_learned"] = measure_form(args, ctx, args.method, learned=True)
    if args.plain:
        # the two plain FP32 forms (both read the FP32 rows): TF32 tensor cores, and SIMT FFMA
        if not (args.method == "tf32" and not args.learned):
            forms["plain_fp32"] = measure_form(args, ctx, "tf32")
        forms["plain_fp32_simt"] = measure_form(args, ctx, "simt")
    if args.batch64 and args.batch != 64:
        # the configuration's other batch size: 64 queries per batch (one SM per 128-doc tile)
        import copy
        a64 = copy.copy(args)
        a64.batch = 64
        forms["chosen_batch64"] = measure_form(a64, ctx, args.method)
        if args.plain:
            forms["plain_fp32_batch64"] = measure_form(a64, ctx, "tf32")
    serving = None
    if rank == 0 and world == 1 and args.serve:
        rates = [float(r) for r in args.serve_rates.split(",")]
        serving = {"chosen": measure_serving(args, ctx, args.method, rates, chosen.get("model"),
                                             chosen.get("margin", 0.0))}
        if "chosen_learned" in forms:
            serving["chosen_learned"] = measure_serving(args, ctx, args.method, rates, forms["chosen_learned"]["model"],
                                                        forms["chosen_learned"]["margin"])
        if args.plain:
            serving["plain_fp32"] = measure_serving(args, ctx, "tf32", rates)

    def summary(f):
        d = {"value": f["value"], "e2e_qps": f["e2e"], "ms_per_step": f["t_max_ms"] / args.steps,
             "stages_ms": f["stages_ms"], "roofline_frac": f["roofline"]["frac"], "form": f["form"],
             "batch": f["batch"]}
        if "learned_report" in f:
            d["learned_report"] = f["learned_report"]
        return d

    rec = {"metric": METRIC, "value": chosen["value"], "unit": "QPS", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": chosen["t_max_ms"] / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": {"simt": "f32", "tf32": "f32", "bf16": "bf16",
                                                             "e4m3": "e4m3"}[args.method] + "+f32 rescore",
           "data": "synthetic (seeded cluster mixture, HYDSET2 shapes)",
           "config": dict(config_of(args, world), form=chosen["form"], method=args.method, learned=args.learned),
           "e2e": {"value": chosen["e2e"], "unit": "QPS", "h2d_bytes_per_step": B * 128 * 4,
                   "d2h_bytes_per_step": B * K * (4 + 8) + B * 4,
                   "path": "hss_filters_compile (next batch, compile thread) + hss_searcher_search_device "
                           "per batch, pinned host queries in and results out"},
           "roofline": chosen["roofline"], "clocks": chosen["clocks"], "gpu_launches": chosen["launches"],
           "stages_ms": chosen["stages_ms"], "forms": {k: summary(v) for k, v in forms.items()}}
    if "plain_fp32" in forms:
        rec["chosen_over_plain"] = chosen["value"] / forms["plain_fp32"]["value"]
    if serving:
        rec["serving"] = serving

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, ref_ids, ref_counts = cpu_baseline(vec, bits, queries, exprs, K, args.cpu_queries)
        rec["cpu_baseline"] = cb
        # parity at full scale, for the CPU sample's queries. The reference's ground truth is a set
        # (CpuTopK returns an unordered_set, recall_ref.cpp:18-48; the reference build hands it back
        # sorted by id), so ids are compared as sets; the order (score desc, id asc) and the scores are
        # checked against the ground truth's own arithmetic: an FP32 sum over d ascending, each product
        # and sum rounded to FP32.
        searcher, filters, d_q = chosen["searcher"], chosen["filters"], chosen["d_q"]
        o_sc, o_id, o_n, topks, sh = chosen["out"]
        nq = len(ref_counts)
        set_ok = order_ok = score_ok = True
        err_abs, err_rel = [], []
        for j in range((nq + B - 1) // B):
            rc = searcher.search_device(d_q[j].data_ptr(), B, filters[j], topks, o_sc.data_ptr(), o_id.data_ptr(),
                                        o_n.data_ptr(), K, sh)
            torch.cuda.synchronize()
            assert rc == 0
            g_id, g_n, g_sc = o_id.cpu().numpy(), o_n.cpu().numpy(), o_sc.cpu().numpy()
            for i in range(B):
                qi = j * B + i
                if qi >= nq:
                    break
                c = int(ref_counts[qi])
                if int(g_n[i]) != c or set(g_id[i][:c].tolist()) != set(ref_ids[qi][:c].tolist()):
                    set_ok = False
                    continue
                ids, sc = g_id[i][:c], g_sc[i][:c]
                acc = np.zeros(c, np.float32)
                qv, dv = queries[qi].astype(np.float32), vec[ids].astype(np.float32)
                for d in range(qv.shape[0]):
                    acc = (acc + (qv[d] * dv[:, d]).astype(np.float32)).astype(np.float32)
                if not (acc.view(np.uint32) == sc.view(np.uint32)).all():
                    score_ok = False
                exact64 = dv.astype(np.float64) @ qv.astype(np.float64)
                err_abs.append(np.abs(sc.astype(np.float64) - exact64))
                err_rel.append(np.abs(sc.astype(np.float64) - exact64) / np.maximum(np.abs(exact64), 1e-30))
                if c > 1 and not all(sc[r] > sc[r + 1] or (sc[r] == sc[r + 1] and ids[r] < ids[r + 1])
                                     for r in range(c - 1)):
                    order_ok = False
        rec["parity_full_scale"] = {"queries": nq, "against": cb["kind"], "id_sets_match": set_ok,
                                    "scores_bit_exact": score_ok, "order_score_desc_id_asc": order_ok}
        if err_abs:
            ea, er = np.concatenate(err_abs), np.concatenate(err_rel)
            # the returned FP32 scores against an FP64 dot product of the same vectors
            rec["parity_full_scale"]["score_error_vs_fp64"] = {
                "max_abs": float(ea.max()), "median_abs": float(np.median(ea)),
                "max_rel": float(er.max()), "median_rel": float(np.median(er))}
    if rank == 0:
        print(json.dumps(rec))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
